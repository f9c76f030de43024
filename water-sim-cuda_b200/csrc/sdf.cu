// Signed distance field of the obstacle triangles on the simulation grid
// (makeSDF, kernels.cu:282-300; Engine::initSDF, engine.cu:105-114).
//
// One thread per node at integer coordinates, a CTA per brick of 8 x 8 x 4
// nodes, in two passes over the triangles:
//
//  1. the winding number: every triangle, in the order given (the sign of
//     the SDF needs all of them).  The CTA streams the list through shared
//     memory in tiles of 256 triangles: one thread issues a bulk async copy
//     (cp.async.bulk, the 1-D TMA path) of the next tile into the second
//     buffer while the CTA evaluates the current one, completion tracked by
//     an mbarrier.  Each node also keeps the least squared distance to a
//     triangle's first vertex, a point on the mesh, hence an upper bound of
//     its distance to the mesh.
//  2. the distance: the triangles again, in a copy sorted by the Morton code
//     of their centroids, whose 256-triangle tiles carry bounding boxes.  A
//     tile whose box lies farther from the brick than the brick's largest
//     bound cannot hold any node's nearest triangle and is skipped by the
//     whole CTA; within a loaded tile, a node skips a triangle whose
//     bounding box lies farther than its distance so far.  The minimum is
//     taken over the same per-pair values as a pass over every triangle, so
//     the result is the same.
//
// Each wait gives up after a fixed time, records kStatusTimeout and drains
// the copies still in flight before the CTA returns, so a lost completion
// cannot hang the device.
//
// Per node-triangle pair the kernel adds the signed solid angle
// (Van Oosterom & Strackee, 1983) and keeps the minimum squared distance to
// the triangle (closest point by Voronoi regions, Ericson, "Real-Time
// Collision Detection" 5.1.5), in triangle order like the reference.  The
// node is inside when the winding number, the solid-angle sum divided by
// 4 * 3.1415 (the reference's constant, kernels.cu:298), exceeds 0.5.
#include <algorithm>
#include <utility>
#include <vector>

#include "kernels.h"

namespace mpm {
namespace {

constexpr int kSdfThreads = 256;
constexpr int kTriTile = 256;                 // triangles per stage
constexpr int kTriFloats = 9;
// Floats rounded up to a 16-byte multiple (bulk copies start 16-byte aligned).
constexpr size_t align_floats16(size_t n) { return (n + 3) & ~(size_t)3; }
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s per wait
constexpr unsigned long long kSdfTestWaitNs = 20000000ull;  // the test hook's expiring wait: 20 ms
// Test hooks (the engine's wait test, the values of kWaitTest* in
// corrector_tc.cuh), acted on at the first tile after its copy has landed.
constexpr uint32_t kSdfTestGiveUp = 1u, kSdfTestExpire = 2u;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void proxy_fence_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of `bar`; false after limit_ns.
__device__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned long long limit_ns = kWaitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
    return true;
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return ax * bx + ay * by + az * bz;
}

// Signed solid angle of triangle (a, b, c) seen from the origin, the vertices
// already relative to the node (calculateSolidAngle, common.cuh:310-323).
__device__ __forceinline__ float solid_angle(float ax, float ay, float az, float bx, float by, float bz, float cx,
                                             float cy, float cz) {
    const float la = norm3df(ax, ay, az), lb = norm3df(bx, by, bz), lc = norm3df(cx, cy, cz);
    const float det = ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx);
    const float div = la * lb * lc + dot3(ax, ay, az, bx, by, bz) * lc + dot3(ax, ay, az, cx, cy, cz) * lb +
                      dot3(bx, by, bz, cx, cy, cz) * la;
    return 2.0f * atan2f(det, div);
}

// Squared distance from P to triangle (a, b, c) (pointTriangleDistanceSq,
// common.cuh:325-378).
__device__ __forceinline__ float tri_dist2(float px, float py, float pz, const float* t) {
    const float ax = t[0], ay = t[1], az = t[2];
    const float abx = t[3] - ax, aby = t[4] - ay, abz = t[5] - az;
    const float acx = t[6] - ax, acy = t[7] - ay, acz = t[8] - az;
    const float apx = px - ax, apy = py - ay, apz = pz - az;
    const float d1 = dot3(abx, aby, abz, apx, apy, apz), d2 = dot3(acx, acy, acz, apx, apy, apz);
    if (d1 <= 0.0f && d2 <= 0.0f) return dot3(apx, apy, apz, apx, apy, apz);
    const float bpx = px - t[3], bpy = py - t[4], bpz = pz - t[5];
    const float d3 = dot3(abx, aby, abz, bpx, bpy, bpz), d4 = dot3(acx, acy, acz, bpx, bpy, bpz);
    if (d3 >= 0.0f && d4 <= d3) return dot3(bpx, bpy, bpz, bpx, bpy, bpz);
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        const float v = d1 / (d1 - d3);
        const float qx = px - (ax + v * abx), qy = py - (ay + v * aby), qz = pz - (az + v * abz);
        return dot3(qx, qy, qz, qx, qy, qz);
    }
    const float cpx = px - t[6], cpy = py - t[7], cpz = pz - t[8];
    const float d5 = dot3(abx, aby, abz, cpx, cpy, cpz), d6 = dot3(acx, acy, acz, cpx, cpy, cpz);
    if (d6 >= 0.0f && d5 <= d6) return dot3(cpx, cpy, cpz, cpx, cpy, cpz);
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        const float w = d2 / (d2 - d6);
        const float qx = px - (ax + w * acx), qy = py - (ay + w * acy), qz = pz - (az + w * acz);
        return dot3(qx, qy, qz, qx, qy, qz);
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        const float qx = px - (t[3] + w * (t[6] - t[3])), qy = py - (t[4] + w * (t[7] - t[4])),
                    qz = pz - (t[5] + w * (t[8] - t[5]));
        return dot3(qx, qy, qz, qx, qy, qz);
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    const float qx = px - (ax + abx * v + acx * w), qy = py - (ay + aby * v + acy * w),
                qz = pz - (az + abz * v + acz * w);
    return dot3(qx, qy, qz, qx, qy, qz);
}

constexpr int kBrickX = 8, kBrickY = 8, kBrickZ = 4;  // kSdfThreads nodes per CTA
static_assert(kBrickX * kBrickY * kBrickZ == kSdfThreads, "one node per thread");
constexpr int kBoxFloats = 8;  // tile box: min x, y, z, max x, y, z, 2 unused

// Squared distance between two boxes (0 when they overlap).
__device__ __forceinline__ float box_dist2(float ax0, float ay0, float az0, float ax1, float ay1, float az1,
                                           const float* b) {
    const float dx = fmaxf(0.0f, fmaxf(b[0] - ax1, ax0 - b[3]));
    const float dy = fmaxf(0.0f, fmaxf(b[1] - ay1, ay0 - b[4]));
    const float dz = fmaxf(0.0f, fmaxf(b[2] - az1, az0 - b[5]));
    return dx * dx + dy * dy + dz * dz;
}

__global__ void __launch_bounds__(kSdfThreads) sdf_build_kernel(SimParams p, const float* __restrict__ tris,
                                                                const float* __restrict__ sorted,
                                                                const float* __restrict__ boxes, int t_count,
                                                                float* __restrict__ sdf,
                                                                uint32_t* __restrict__ status, uint32_t wait_test) {
    __shared__ __align__(128) float s_tri[2][kTriTile * kTriFloats];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ float s_red[kSdfThreads / 32];

    const int nbx = (p.sx + kBrickX - 1) / kBrickX, nby = (p.sy + kBrickY - 1) / kBrickY;
    const int bxi = blockIdx.x % nbx, byi = (blockIdx.x / nbx) % nby, bzi = blockIdx.x / (nbx * nby);
    const int t = threadIdx.x;
    const int x = bxi * kBrickX + t % kBrickX, y = byi * kBrickY + (t / kBrickX) % kBrickY,
              z = bzi * kBrickZ + t / (kBrickX * kBrickY);
    const bool valid = x < p.sx && y < p.sy && z < p.sz;
    const float px = x * 1.0f, py = y * 1.0f, pz = z * 1.0f;
    const int ntiles = (t_count + kTriTile - 1) / kTriTile;

    if (threadIdx.x == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();

    auto issue = [&](const float* src, int tile, int b) {
        const int cnt = min(kTriTile, t_count - tile * kTriTile);
        const uint32_t bytes = (uint32_t)((cnt * kTriFloats * 4 + 15) & ~15);
        proxy_fence_shared();
        mbar_expect_tx(&s_bar[b], bytes);
        bulk_copy_g2s(s_tri[b], src + (size_t)tile * kTriTile * kTriFloats, bytes, &s_bar[b]);
    };

    // Pass 1: winding number over every triangle in order, and an upper bound
    // of the distance (first vertices).
    if (threadIdx.x == 0 && ntiles > 0) issue(tris, 0, 0);
    float wsum = 0.0f, ub2 = 1e30f;
    bool aborted = false;
    int tile = 0;
    for (; tile < ntiles; ++tile) {
        const int b = tile & 1;
        if (threadIdx.x == 0 && tile + 1 < ntiles) issue(tris, tile + 1, (tile + 1) & 1);
        bool ok = mbar_wait_bounded(&s_bar[b], (uint32_t)((tile >> 1) & 1));
        if (ok && tile == 0 && wait_test) {
            // Test hooks, with tile 0's copy landed: report a give-up, or
            // wait for the barrier's next phase, which no copy completes yet
            // (tile 2 is issued only at the next iteration), until the short
            // limit runs out.
            if (wait_test & kSdfTestGiveUp) ok = false;
            else if (wait_test & kSdfTestExpire) ok = mbar_wait_bounded(&s_bar[b], 1u, kSdfTestWaitNs);
        }
        if (__syncthreads_or(!ok)) {
            aborted = true;
            break;
        }
        const int cnt = min(kTriTile, t_count - tile * kTriTile);
        const float* st = s_tri[b];
        for (int k = 0; k < cnt; ++k) {
            const float* tr = st + k * kTriFloats;
            const float ax = tr[0] - px, ay = tr[1] - py, az = tr[2] - pz;
            wsum += solid_angle(ax, ay, az, tr[3] - px, tr[4] - py, tr[5] - pz, tr[6] - px, tr[7] - py, tr[8] - pz);
            ub2 = fminf(ub2, ax * ax + ay * ay + az * az);
        }
        __syncthreads();
    }
    if (aborted) {
        // Drain: the copy of `tile` and possibly `tile + 1` may still land.
        if (threadIdx.x == 0) {
            atomicOr(status, kStatusTimeout);
            mbar_wait_bounded(&s_bar[tile & 1], (uint32_t)((tile >> 1) & 1));
            if (tile + 1 < ntiles) mbar_wait_bounded(&s_bar[(tile + 1) & 1], (uint32_t)(((tile + 1) >> 1) & 1));
        }
        __syncthreads();
        return;
    }
    // The brick's bound: no node of it is farther from the mesh than this,
    // with a margin for the rounding of the bound and of the box distances.
    float bound = valid ? ub2 : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bound = fmaxf(bound, __shfl_xor_sync(0xffffffffu, bound, o));
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = bound;
    __syncthreads();
    bound = s_red[0];
#pragma unroll
    for (int w = 1; w < kSdfThreads / 32; ++w) bound = fmaxf(bound, s_red[w]);
    bound = bound * 1.0001f + 1e-6f;
    const float bx0 = bxi * kBrickX, by0 = byi * kBrickY, bz0 = bzi * kBrickZ;
    const float bx1 = bx0 + (kBrickX - 1), by1 = by0 + (kBrickY - 1), bz1 = bz0 + (kBrickZ - 1);

    // Pass 2: distance over the sorted tiles that can hold a nearest
    // triangle, one tile at a time through buffer 0, whose barrier has
    // completed (ntiles + 1) / 2 phases in pass 1.
    uint32_t phase = (uint32_t)(((ntiles + 1) / 2) & 1);
    float dmin2 = 1e30f;
    for (int k = 0; k < ntiles; ++k) {
        if (box_dist2(bx0, by0, bz0, bx1, by1, bz1, boxes + (size_t)k * kBoxFloats) > bound) continue;
        if (threadIdx.x == 0) issue(sorted, k, 0);
        const bool ok = mbar_wait_bounded(&s_bar[0], phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicOr(status, kStatusTimeout);
                mbar_wait_bounded(&s_bar[0], phase ^ 1u);  // drain the copy
            }
            __syncthreads();
            return;
        }
        const int cnt = min(kTriTile, t_count - k * kTriTile);
        const float* st = s_tri[0];
        for (int q = 0; q < cnt; ++q) {
            const float* tr = st + q * kTriFloats;
            const float lo[3] = {fminf(tr[0], fminf(tr[3], tr[6])), fminf(tr[1], fminf(tr[4], tr[7])),
                                 fminf(tr[2], fminf(tr[5], tr[8]))};
            const float hi[3] = {fmaxf(tr[0], fmaxf(tr[3], tr[6])), fmaxf(tr[1], fmaxf(tr[4], tr[7])),
                                 fmaxf(tr[2], fmaxf(tr[5], tr[8]))};
            const float dx = fmaxf(0.0f, fmaxf(lo[0] - px, px - hi[0]));
            const float dy = fmaxf(0.0f, fmaxf(lo[1] - py, py - hi[1]));
            const float dz = fmaxf(0.0f, fmaxf(lo[2] - pz, pz - hi[2]));
            if ((dx * dx + dy * dy + dz * dz) * 0.9999f > dmin2) continue;
            const float d2 = tri_dist2(px, py, pz, tr);
            if (d2 < dmin2) dmin2 = d2;
        }
        __syncthreads();
    }
    if (valid) {
        const float wn = wsum / (4.0f * 3.1415f);
        sdf[node_index(p, x, y, z)] = (wn > 0.5f ? -1.0f : 1.0f) * sqrtf(dmin2);
    }
}

}  // namespace

// Morton code of a point in [0, 1)^3, 10 bits per axis.
static uint32_t morton10(float x, float y, float z) {
    auto spread = [](uint32_t v) {
        v = (v * 0x00010001u) & 0xFF0000FFu;
        v = (v * 0x00000101u) & 0x0F00F00Fu;
        v = (v * 0x00000011u) & 0xC30C30C3u;
        v = (v * 0x00000005u) & 0x49249249u;
        return v;
    };
    auto q = [](float f) { return (uint32_t)std::min(1023.0f, std::max(0.0f, f * 1024.0f)); };
    return (spread(q(z)) << 2) | (spread(q(y)) << 1) | spread(q(x));
}

size_t sdf_aux_floats(int t) {
    const size_t tiles = (size_t)(t + kTriTile - 1) / kTriTile;
    return align_floats16((size_t)t * kTriFloats) + tiles * kBoxFloats;
}

void sdf_prepare_host(const float* tris, int t, float* aux) {
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < t; ++i)
        for (int k = 0; k < 9; ++k) {
            lo[k % 3] = std::min(lo[k % 3], tris[i * 9 + k]);
            hi[k % 3] = std::max(hi[k % 3], tris[i * 9 + k]);
        }
    std::vector<std::pair<uint32_t, int>> key((size_t)t);
    for (int i = 0; i < t; ++i) {
        float c[3];
        for (int a = 0; a < 3; ++a) {
            const float mid = (tris[i * 9 + a] + tris[i * 9 + 3 + a] + tris[i * 9 + 6 + a]) / 3.0f;
            const float ext = hi[a] - lo[a];
            c[a] = ext > 0.0f ? (mid - lo[a]) / ext : 0.0f;
        }
        key[i] = {morton10(c[0], c[1], c[2]), i};
    }
    std::stable_sort(key.begin(), key.end());
    float* sorted = aux;
    float* boxes = aux + align_floats16((size_t)t * kTriFloats);
    for (int i = 0; i < t; ++i) std::copy(tris + (size_t)key[i].second * 9, tris + (size_t)key[i].second * 9 + 9, sorted + (size_t)i * 9);
    const int tiles = (t + kTriTile - 1) / kTriTile;
    for (int k = 0; k < tiles; ++k) {
        float* b = boxes + (size_t)k * kBoxFloats;
        b[0] = b[1] = b[2] = 1e30f;
        b[3] = b[4] = b[5] = -1e30f;
        b[6] = b[7] = 0.0f;
        for (int i = k * kTriTile; i < std::min(t, (k + 1) * kTriTile); ++i)
            for (int v = 0; v < 9; ++v) {
                b[v % 3] = std::min(b[v % 3], sorted[(size_t)i * 9 + v]);
                b[3 + v % 3] = std::max(b[3 + v % 3], sorted[(size_t)i * 9 + v]);
            }
    }
}

int launch_sdf_build(const SimParams& p, const float* tris, const float* aux, int t, float* sdf, uint32_t* status,
                     cudaStream_t st, uint32_t wait_test) {
    if (p.g <= 0) return 0;
    const int bricks = ((p.sx + kBrickX - 1) / kBrickX) * ((p.sy + kBrickY - 1) / kBrickY) *
                       ((p.sz + kBrickZ - 1) / kBrickZ);
    const float* sorted = aux;
    const float* boxes = aux + align_floats16((size_t)t * kTriFloats);
    sdf_build_kernel<<<bricks, kSdfThreads, 0, st>>>(p, tris, sorted, boxes, t, sdf, status, wait_test);
    return 1;
}

}  // namespace mpm
