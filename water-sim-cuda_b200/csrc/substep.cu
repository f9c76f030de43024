// One MLS-MPM substep on the device: particle binning, P2G scatter, grid
// update, G2P gather, plus the kernels that move state across the boundary.
//
// Layout (HBM):
//  - particle state: particle-major, 24 floats per particle (device_math.cuh),
//    double-buffered, ordered by cell of the last binning so that the
//    particles of one stencil base cell are contiguous;
//  - cells: every stencil base cell of the grid, numbered bin * kBinCells +
//    the cell's index in its bin (kBinX x kBinY x kBinZ cells).  Two counter
//    sets alternate: the substep from parity p orders the particles by set p
//    (filled by the previous G2P or by an import) and its G2P files every
//    particle into set 1-p (cell count, bin count, and the list of bins that
//    received particles);
//  - grid: one float4 per node, (mass, x, y, z).  `accum` receives the P2G
//    sums with 16-byte vector reductions (red.global.add.v4.f32); the grid
//    update turns it into `vgrid` (mass, velocity) and leaves `accum` zero
//    for the next substep, so no separate clear pass is needed;
//  - sdf: one float per node.
#include <algorithm>
#include <climits>
#include <cstdint>

#include "kernels.h"

namespace mpm {
namespace {

__device__ __forceinline__ void red_add_v4(float4* addr, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// A 16-byte asynchronous copy of a particle record's vector into shared
// memory, marked evict-first in L2: each record is read once per pass, and
// leaving L2 to the grid arrays the P2G reductions and the grid update work
// on measured 5 % off P2G on the 2M dam break (early and late states).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
                 "l"(gmem), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Programmatic dependent launch: the substep's kernels are launched with
// programmatic stream serialisation (launch_dep), so that a kernel's CTAs are
// scheduled while its predecessor drains; each such kernel waits here, before
// touching memory, until its predecessor has completed and its writes are
// visible (griddepcontrol.wait; a no-op for an ordinary launch).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Files this lane's particle under global cell `gcell` (global bin `gbin`,
// bin `bin` of scene `scene`, whose bin entries start at `boff`) of a counter
// set: one reduction per distinct cell of the warp (no value comes back, so
// no lane waits on it) and one atomic per distinct bin, whose leader appends
// the bin to its scene's list when it is the bin's first particle.  The
// particle's place within its cell is drawn later, by the ordering's scatter.
// Every lane of the warp must call it; lanes with gcell < 0 take part without
// counting.
__device__ __forceinline__ void file_particle(int gcell, int gbin, int bin, int scene, long long boff,
                                              const BinSet& set) {
    const int lane = threadIdx.x & 31;
    const uint32_t peers = __match_any_sync(0xffffffffu, gcell);
    if (gcell >= 0 && lane == __ffs(peers) - 1) atomicAdd(set.ccount + gcell, (uint32_t)__popc(peers));
    const uint32_t bpeers = __match_any_sync(0xffffffffu, gbin);
    if (gbin >= 0 && lane == __ffs(bpeers) - 1) {
        if (atomicAdd(set.bcount + gbin, (uint32_t)__popc(bpeers)) == 0u)
            set.blist[boff + atomicAdd(set.nlist + scene, 1u)] = bin;
    }
}

// Scene lookup for the per-particle and per-node kernels.  With one scene
// (kBatch false) the parameters are the kernel argument p0, read from the
// parameter bank.  With several, a CTA whose indices are [i0, i1) needs only
// the scenes that range touches (usually one or two): the first threads find
// its first and last scene in one parallel test, and the CTA stages just those
// records and first indices in shared memory.  Each thread then finds its
// scene there.  Beyond kTableScenes scenes the lookup searches the global
// table.
constexpr int kTableScenes = 64;

template <bool kBatch>
struct SceneLookup {
    const SimParams* prm;
    const long long* first;
    int count;
    int lo = 0;  // global index of prm[0] / first[0]

    // Must be reached by every thread of the CTA (it may synchronize).
    // s_range: two ints of shared memory.
    __device__ __forceinline__ SceneLookup(const SceneTable& sc, const long long* first_global, SimParams* s_prm,
                                           long long* s_first, int* s_range, long long i0, long long i1)
        : prm(sc.prm), first(first_global), count(sc.count) {
        if constexpr (kBatch) {
            if (count <= kTableScenes) {
                // Scene s holds index i when it is the last with first[s] <= i
                // (first[0] = 0, non-decreasing): exactly one thread matches.
                const int t = threadIdx.x;
                if (t < count) {
                    const long long f0 = first_global[t];
                    const long long f1 = t + 1 < count ? first_global[t + 1] : LLONG_MAX;
                    if (f0 <= i0 && i0 < f1) s_range[0] = t;
                    if (f0 <= i1 - 1 && i1 - 1 < f1) s_range[1] = t;
                }
                __syncthreads();
                lo = s_range[0];
                const int n = s_range[1] - lo + 1;
                if (t < n) s_prm[t] = sc.prm[lo + t];
                if (t <= n) s_first[t] = first_global[lo + t];
                __syncthreads();
                prm = s_prm;
                first = s_first;
                count = n;
            }
        }
    }

    // Global scene index of index i (i in the CTA's range).
    __device__ __forceinline__ int scene(long long i) const {
        if constexpr (!kBatch) return 0;
        int a = 0, b = count - 1;
        while (a < b) {
            const int mid = (a + b + 1) >> 1;
            if (first[mid] <= i) a = mid;
            else b = mid - 1;
        }
        return lo + a;
    }

    __device__ __forceinline__ const SimParams& params(int scene) const { return prm[scene - lo]; }
};

// ------------------------------------------------------------------ P2G ----
// P2G (p2GTransferScatter, kernels.cu:6-142).  Persistent single-warp CTAs
// take work items from a counter; a listed bin (8 x 4 x 4 base cells) has
// kBinZ items, and item g takes positions 32 g .. 32 g + 31 of the bin's cell
// order (cell_order: occupied cells by count class, largest first), so the
// lanes of a warp hold cells of similar counts and no empty ones.  The
// counter hands out every bin's item 0 before any item 1, and so on, so the
// longest items start first.  Lane =
// cell: all particles of a cell scatter to the same 27 nodes, so the lane sums
// them in registers, reading them through a ring of kRing particles fetched
// ahead with 16-byte cp.async copies (the gather through gidx costs no
// registers).  The lane then adds its 27 sums to the warp's footprint, the
// bin's 10 x 6 x 6 nodes in shared memory: the lanes' cells are distinct, so
// for one stencil offset their nodes differ and a plain read-add-write per
// offset is race-free.  A lane sums at most `cap` particles of its cell (a
// launch parameter; 0 = chosen per work item by item_cap); the rest of a
// crowded cell (this Tait law resists only expansion, so compressed fluid
// piles up) goes to a list in chunks of kCrowdChunk particles, which a
// second launch spreads over all warps (the count order gathers a bin's
// crowded cells in one item, and one warp working through all of their
// particles would hold up the kernel).  The footprint's z-planes that the
// item reached go to global memory with one vector reduction per touched
// node.  Unlike the reference, no partial sum
// is dropped (it drops shared-tile cells whose partial mass is <= 1e-9,
// kernels.cu:132).
constexpr int kP2GWarpsPerSM = 12;
constexpr int kRing = 2;
constexpr int kGidxStage = 256;   // gather indices of a bin staged in shared memory
constexpr int kCellCap = 12;      // particles of a cell its own lane sums; the rest: the crowded-cell list
constexpr int kCrowdChunk = 256;  // particles of a crowded cell per list entry
constexpr int kTX = kBinX + 2, kTY = kBinY + 2;
constexpr int kFootPlane = kTX * kTY;              // 60 nodes of one z-plane
constexpr int kFootNodes = kFootPlane * (kBinZ + 2);  // 360: a bin's stencil footprint
static_assert(kBinX * kBinY == 32 && kBinZ == 4, "a bin is 128 cells: four items of 32");

// Spline weights of nodes 0, 1, 2 of one axis at fractional offset f = pos -
// base, times m.  For f in [0.5, 1.5) (every particle at pos >= 0.5) the
// branch of bspline_weight is known per node and the same roundings are
// written out; otherwise the general form.
__device__ __forceinline__ void axis_weights(float f, float m, float* w) {
    if (f >= 0.5f && f < 1.5f) {
        const float t0 = __fsub_rn(1.5f, f);
        const float x1 = __fsub_rn(f, 1.0f);
        const float t2 = __fsub_rn(1.5f, __fsub_rn(2.0f, f));
        w[0] = m * __fmul_rn(__fmul_rn(t0, t0), 0.5f);
        w[1] = m * __fsub_rn(0.75f, __fmul_rn(x1, x1));
        w[2] = m * __fmul_rn(__fmul_rn(t2, t2), 0.5f);
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) w[a] = m * bspline_weight(f - (float)a);
    }
}

// Per-particle part of P2G from the particle's 96-byte record: the spline
// weights (mass folded into wx) and the affine momentum at stencil node
// (0,0,0), u = v - C' f, with C' the stress-augmented affine matrix.  Node
// o of the stencil then gets w_o (u + C' o).
struct P2GParticle {
    float wx[3], wy[3], wz[3];
    float u0, u1, u2;
    float C[9];
    int bx, by, bz;  // stencil base cell
};

__device__ __forceinline__ P2GParticle p2g_particle(const SimParams& p, float4 q0, float4 q1, float4 q2, float4 q3,
                                                    float4 q4, float4 q5) {
    P2GParticle r;
    const float px = q0.x, py = q0.y, pz = q0.z;
    const float F[9] = {q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
    float* C = r.C;
    C[0] = q3.w;
    C[1] = q4.x;
    C[2] = q4.y;
    C[3] = q4.z;
    C[4] = q4.w;
    C[5] = q5.x;
    C[6] = q5.y;
    C[7] = q5.z;
    C[8] = q5.w;
    // Tait pressure from the clamped det F and the APIC + stress affine
    // matrix C' = C + (4 DT V p / m) I (kernels.cu:20-35).
    float J = det3(F);
    J = fmaxf(0.9f, fminf(J, 1.1f));
    // J^gamma - 1 > 0 only for J > 1 (gamma > 0) or J < 1 (gamma < 0); the
    // clamp below zeroes every other case, so powf runs only where it counts.
    float pressure = 0.0f;
    if ((p.gamma > 0.0f && J > 1.0f) || (p.gamma < 0.0f && J < 1.0f))
        pressure = p.compression * (powf(J, p.gamma) - 1.0f);
    if (pressure < 0.0f) pressure = 0.0f;
    const float multi = 4.0f * p.dt * (p.pvol * J) * pressure / p.pmass;
    C[0] += multi;
    C[4] += multi;
    C[8] += multi;
    // f = pos - base is exact for |pos| < 2^24, so f - o equals the
    // reference's pos - (base + o) bit for bit.
    r.bx = stencil_base(px);
    r.by = stencil_base(py);
    r.bz = stencil_base(pz);
    const float fx = px - (float)r.bx, fy = py - (float)r.by, fz = pz - (float)r.bz;
    axis_weights(fx, p.pmass, r.wx);
    axis_weights(fy, 1.0f, r.wy);
    axis_weights(fz, 1.0f, r.wz);
    r.u0 = q3.x - (C[0] * fx + C[1] * fy + C[2] * fz);
    r.u1 = q3.y - (C[3] * fx + C[4] * fy + C[5] * fz);
    r.u2 = q3.z - (C[6] * fx + C[7] * fy + C[8] * fz);
    return r;
}

// The 27 contributions w_o (u + C' o) of one particle, o = (a, b, c), handed
// to emit(k, a, b, c, m, mx, my, mz) in order k = (c * 3 + b) * 3 + a.
template <typename Emit>
__device__ __forceinline__ void p2g_stencil(const P2GParticle& r, Emit emit) {
    float tz0 = r.u0, tz1 = r.u1, tz2 = r.u2;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float ty0 = tz0, ty1 = tz1, ty2 = tz2;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float wyz = r.wy[b] * r.wz[c];
            float t0 = ty0, t1 = ty1, t2 = ty2;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float w = r.wx[a] * wyz;
                emit((c * 3 + b) * 3 + a, a, b, c, w, w * t0, w * t1, w * t2);
                t0 += r.C[0];
                t1 += r.C[3];
                t2 += r.C[6];
            }
            ty0 += r.C[1];
            ty1 += r.C[4];
            ty2 += r.C[7];
        }
        tz0 += r.C[2];
        tz1 += r.C[5];
        tz2 += r.C[8];
    }
}

// The crowded-cell threshold of one work item, from the counts of its 32
// cells (`full`, one per lane): for each candidate cap the loop costs
// min(max count, cap) iterations with every lane, plus, per cell above the
// cap, ceil((count - cap) / 32) whole-warp iterations and one reduce-scatter
// (about 1.3 iterations) in the crowded-cell launch; the cheapest candidate
// wins.  Every cap gives the same sums.  Caps stop at 32: a larger one makes a
// few long items that hold up the kernel while other warps idle, whereas the
// list spreads the rest of a crowded cell over all warps.
__device__ __forceinline__ int item_cap(int full) {
    const int maxc = __reduce_max_sync(0xffffffffu, (unsigned)full);
    int best = kCellCap;
    float best_cost = 1e30f;
#pragma unroll
    for (int cand : {8, 12, 16, 24, 32}) {
        const int over = full > cand ? (full - cand + 31) / 32 : 0;
        const int passes = (int)__reduce_add_sync(0xffffffffu, (unsigned)over);
        const int cells = __popc(__ballot_sync(0xffffffffu, full > cand));
        const float cost = (float)min(maxc, cand) + (float)passes + 1.3f * (float)cells;
        if (cost < best_cost) best_cost = cost, best = cand;
    }
    return best;
}

__global__ void __launch_bounds__(32, kP2GWarpsPerSM) p2g_kernel(SceneTable sc, const float* __restrict__ P,
                                                                  const int32_t* __restrict__ gidx,
                                                                  const int32_t* __restrict__ cstart, BinSet set,
                                                                  const uint8_t* __restrict__ corder,
                                                                  const long long* __restrict__ itemoff,
                                                                  uint32_t* __restrict__ work,
                                                                  float4* __restrict__ accum_all, int4* __restrict__ crowd,
                                                                  int crowd_cap, uint32_t* __restrict__ status, int cap) {
    pdl_wait();
    __shared__ __align__(16) float4 s_ring[kRing][6][32];
    __shared__ float4 s_foot[kFootNodes];
    __shared__ int32_t s_gidx[kGidxStage];
    const int lane = threadIdx.x;
    const long long nitems = *reinterpret_cast<volatile const long long*>(itemoff + sc.count);
    for (int q = lane; q < kFootNodes; q += 32) s_foot[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (;;) {
        int item = 0;
        if (lane == 0) item = (int)atomicAdd(work, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= nitems) return;
        // Items: kBinZ per listed bin, scene after scene, group-major within a scene.
        const int scene = sc.count == 1 ? 0 : scene_of(itemoff, sc.count, item);
        const SimParams p = sc.prm[scene];
        // Group-major: every listed bin's group 0 (its most crowded cells) comes
        // before any group 1, and so on, so that the long items start first.
        const int local = item - (int)__ldg(itemoff + scene);
        const int nl = (int)((__ldg(itemoff + scene + 1) - __ldg(itemoff + scene)) / kBinZ);
        const int bin = __ldg(set.blist + p.boff + local % nl), group = local / nl;
        if (bin >= p.nb) continue;  // the overflow bin reaches no node
        float4* accum = accum_all + p.goff;
        const int bxi = bin % p.nbx, byi = (bin / p.nbx) % p.nby, bzi = bin / (p.nbx * p.nby);
        // Node origin of the footprint = base cell of the bin's first cell.
        const int ox = bxi * kBinX - 2, oy = byi * kBinY - 2, oz = bzi * kBinZ - 2;
        const size_t cb = (size_t)p.coff + (size_t)bin * kBinCells;
        // This lane's cell (z * 32 + y * 8 + x in the bin), 0xFF for none.
        const int tcell = __ldg(corder + cb + group * 32 + lane);
        if (__ballot_sync(0xffffffffu, tcell != 0xFF) == 0u) continue;
        const bool own = tcell != 0xFF;
        const int cs = own ? __ldg(cstart + cb + tcell) : 0;
        const int full = own ? (int)__ldg(set.ccount + cb + tcell) : 0;
        // The bin's slots (its cells are consecutive in the particle order).
        const int l0 = __ldg(cstart + cb);
        const int l1 = __ldg(cstart + cb + kBinCells - 1) + (int)__ldg(set.ccount + cb + kBinCells - 1);
        const bool staged = l1 - l0 <= kGidxStage;
        if (staged)
            for (int q = lane; q < l1 - l0; q += 32) s_gidx[q] = __ldg(gidx + l0 + q);
        __syncwarp();
        // Each lane sums its cell's first `icap` particles; the rest of a
        // crowded cell goes to the crowded-cell list in chunks, which
        // p2g_crowd_kernel spreads over all warps.
        const int icap = cap > 0 ? cap : item_cap(full);
        for (int off = icap; off < full; off += kCrowdChunk) {
            const uint32_t e = atomicAdd(work + 2, 1u);
            if (e < (uint32_t)crowd_cap)
                crowd[e] = make_int4(scene, bin * kBinCells + tcell, cs + off, min(kCrowdChunk, full - off));
            else
                atomicOr(status, kStatusCrowdList);
        }
        const int cnt = min(full, icap);
        const int maxc = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
        float am[27], ax[27], ay[27], az[27];
        auto src_of = [&](int s) -> const float4* {
            const int slot = cs + s;
            const int g = staged ? s_gidx[slot - l0] : __ldg(gidx + slot);
            return reinterpret_cast<const float4*>(P + (size_t)g * kAFloats);
        };
#pragma unroll
        for (int k = 0; k < 27; ++k) am[k] = ax[k] = ay[k] = az[k] = 0.f;
#pragma unroll
        for (int d = 0; d < kRing - 1; ++d) {
            if (d < cnt) {
                const float4* src = src_of(d);
#pragma unroll
                for (int v = 0; v < 6; ++v) cp_async16(&s_ring[d][v][lane], src + v);
            }
            cp_async_commit();
        }
        for (int s = 0; s < maxc; ++s) {
            const int pf = s + kRing - 1;
            if (pf < cnt) {
                const float4* src = src_of(pf);
#pragma unroll
                for (int v = 0; v < 6; ++v) cp_async16(&s_ring[pf % kRing][v][lane], src + v);
            }
            cp_async_commit();
            cp_async_wait<kRing - 1>();
            __syncwarp();
            if (s < cnt) {
                const int sl = s % kRing;
                const P2GParticle r = p2g_particle(p, s_ring[sl][0][lane], s_ring[sl][1][lane], s_ring[sl][2][lane],
                                                   s_ring[sl][3][lane], s_ring[sl][4][lane], s_ring[sl][5][lane]);
                // Filed under this lane's cell by construction; a mismatch is
                // recorded, never scattered to a wrong node.
                if (r.bx - ox != tcell % kBinX || r.by - oy != (tcell / kBinX) % kBinY || r.bz - oz != tcell / 32) {
                    atomicOr(status, kStatusBinning);
                } else {
                    p2g_stencil(r, [&](int k, int, int, int, float m, float mx, float my, float mz) {
                        am[k] += m;
                        ax[k] += mx;
                        ay[k] += my;
                        az[k] += mz;
                    });
                }
            }
            __syncwarp();
        }
        cp_async_wait<0>();
        // One lane per cell: distinct nodes for each stencil offset.
        {
            const int tx = tcell % kBinX, ty = (tcell / kBinX) % kBinY, tz = (tcell / 32) & (kBinZ - 1);
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int b = 0; b < 3; ++b)
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const int k = (c * 3 + b) * 3 + a;
                        float4* d = &s_foot[((tz + c) * kTY + ty + b) * kTX + tx + a];
                        __syncwarp();
                        if (own) {
                            float4 v = *d;
                            v.x += am[k];
                            v.y += ax[k];
                            v.z += ay[k];
                            v.w += az[k];
                            *d = v;
                        }
                    }
        }
        __syncwarp();
        // The z-planes the group's cells reach: zmin .. zmax + 2.
        const int zmin = (int)__reduce_min_sync(0xffffffffu, own ? (unsigned)(tcell / 32) : 0xFFu);
        const int zmax = (int)__reduce_max_sync(0xffffffffu, own ? (unsigned)(tcell / 32) : 0u);
        for (int q = zmin * kFootPlane + lane; q < (zmax + 3) * kFootPlane; q += 32) {
            const int x = ox + q % kTX, y = oy + (q / kTX) % kTY, z = oz + q / kFootPlane;
            const float4 v = s_foot[q];
            s_foot[q] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (node_in_grid(p, x, y, z) && (v.x != 0.f || v.y != 0.f || v.z != 0.f || v.w != 0.f))  // NaN counts
                red_add_v4(accum + node_index(p, x, y, z), v.x, v.y, v.z, v.w);
        }
        __syncwarp();
    }
}

// The crowded-cell list: each entry (scene, bin * 128 + cell, first slot,
// count <= kCrowdChunk) is the next chunk of a crowded cell's particles.  All
// 32 lanes take its particles (slot first + lane + 32 s), sum their 27 x 4
// contributions in registers, reduce-scatter them across the warp (five
// shuffle steps, each halving the 128 padded sums, so lane l ends with node
// l's totals) and add them to global memory.
__global__ void __launch_bounds__(32, kP2GWarpsPerSM) p2g_crowd_kernel(SceneTable sc, const float* __restrict__ P,
                                                                        const int32_t* __restrict__ gidx,
                                                                        const int4* __restrict__ crowd, int crowd_cap,
                                                                        uint32_t* __restrict__ work,
                                                                        float4* __restrict__ accum_all,
                                                                        uint32_t* __restrict__ status) {
    pdl_wait();
    __shared__ __align__(16) float4 s_ring[kRing][6][32];
    const int lane = threadIdx.x;
    const int total = (int)min(*reinterpret_cast<volatile const uint32_t*>(work + 2), (uint32_t)crowd_cap);
    for (;;) {
        int item = 0;
        if (lane == 0) item = (int)atomicAdd(work + 3, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) return;
        const int4 e = crowd[item];
        const SimParams p = sc.prm[e.x];
        const int bin = e.y / kBinCells, cell = e.y % kBinCells;
        const int bxi = bin % p.nbx, byi = (bin / p.nbx) % p.nby, bzi = bin / (p.nbx * p.nby);
        const int bx = bxi * kBinX - 2 + cell % kBinX, by = byi * kBinY - 2 + (cell / kBinX) % kBinY;
        const int bz = bzi * kBinZ - 2 + cell / 32;
        const int first = e.z + lane, cnt = max(0, (e.w - lane + 31) / 32), maxc = (e.w + 31) / 32;
        float am[27], ax[27], ay[27], az[27];
#pragma unroll
        for (int k = 0; k < 27; ++k) am[k] = ax[k] = ay[k] = az[k] = 0.f;
        auto src_of = [&](int s) -> const float4* {
            return reinterpret_cast<const float4*>(P + (size_t)__ldg(gidx + first + 32 * s) * kAFloats);
        };
#pragma unroll
        for (int d = 0; d < kRing - 1; ++d) {
            if (d < cnt) {
                const float4* src = src_of(d);
#pragma unroll
                for (int v = 0; v < 6; ++v) cp_async16(&s_ring[d][v][lane], src + v);
            }
            cp_async_commit();
        }
        for (int s = 0; s < maxc; ++s) {
            const int pf = s + kRing - 1;
            if (pf < cnt) {
                const float4* src = src_of(pf);
#pragma unroll
                for (int v = 0; v < 6; ++v) cp_async16(&s_ring[pf % kRing][v][lane], src + v);
            }
            cp_async_commit();
            cp_async_wait<kRing - 1>();
            __syncwarp();
            if (s < cnt) {
                const int sl = s % kRing;
                const P2GParticle r = p2g_particle(p, s_ring[sl][0][lane], s_ring[sl][1][lane], s_ring[sl][2][lane],
                                                   s_ring[sl][3][lane], s_ring[sl][4][lane], s_ring[sl][5][lane]);
                if (r.bx != bx || r.by != by || r.bz != bz) {
                    atomicOr(status, kStatusBinning);
                } else {
                    p2g_stencil(r, [&](int k, int, int, int, float m, float mx, float my, float mz) {
                        am[k] += m;
                        ax[k] += mx;
                        ay[k] += my;
                        az[k] += mz;
                    });
                }
            }
            __syncwarp();
        }
        cp_async_wait<0>();
        __syncwarp();
        float v[128];
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            v[4 * k + 0] = k < 27 ? am[k < 27 ? k : 0] : 0.f;
            v[4 * k + 1] = k < 27 ? ax[k < 27 ? k : 0] : 0.f;
            v[4 * k + 2] = k < 27 ? ay[k < 27 ? k : 0] : 0.f;
            v[4 * k + 3] = k < 27 ? az[k < 27 ? k : 0] : 0.f;
        }
#pragma unroll
        for (int d = 16, h = 64; d >= 1; d >>= 1, h >>= 1) {
            const bool upper = (lane & d) != 0;
#pragma unroll
            for (int i = 0; i < h; ++i) {
                const float send = upper ? v[i] : v[i + h];
                const float keep = upper ? v[i + h] : v[i];
                v[i] = keep + __shfl_xor_sync(0xffffffffu, send, d);
            }
        }
        if (lane < 27) {
            const int x = bx + lane % 3, y = by + (lane / 3) % 3, z = bz + lane / 9;
            if (node_in_grid(p, x, y, z) && (v[0] != 0.f || v[1] != 0.f || v[2] != 0.f || v[3] != 0.f))
                red_add_v4(accum_all + p.goff + node_index(p, x, y, z), v[0], v[1], v[2], v[3]);
        }
        __syncwarp();
    }
}

// -------------------------------------------------------------- binning ----
// Files the particles of an imported state (slot order) into a counter set.
__global__ void __launch_bounds__(256) bin_count_kernel(SceneTable sc, long long n, const float* __restrict__ P,
                                                        int32_t* __restrict__ pcell, BinSet set) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool valid = j < n;
    int gcell = -1, gbin = -1, bin = -1, scene = 0;
    long long boff = 0;
    if (valid) {
        scene = scene_of(sc.poff, sc.count, j);
        const SimParams p = sc.prm[scene];
        const float4 q = __ldg(reinterpret_cast<const float4*>(P + (size_t)j * kAFloats));
        const int cell = cell_of(p, q.x, q.y, q.z, &bin);
        gcell = (int)p.coff + cell;
        gbin = (int)p.boff + bin;
        boff = p.boff;
    }
    file_particle(gcell, gbin, bin, scene, boff, set);
    if (valid) pcell[j] = gcell;
}

// Bin starts in two launches over (scene, chunk of kScanChunk bins) CTAs, no
// CTA waiting on another: bin_sum_kernel writes each chunk's count sum to
// bpart[scene * chunks + chunk]; bin_scan_kernel adds the sums of the
// scene's earlier chunks to poff and scans its own chunk, so that
// bstart[i] = poff + sum of bcount[0..i) over the scene's nbins = nb + 1
// bins and bstart[nbins] = poff + its particle count (global slots).  The
// scan also zeroes the chunk's bin counters of the other set, and CTA (0, 0)
// the P2G and G2P work counters and writes the per-scene prefixes of the
// listed bins (itemoff, in P2G items, for the current set; clroff for the set
// to clear).  Per chunk: coalesced loads into shared
// memory, a contiguous run of kScanPer counters per thread, a block scan of
// the run sums, coalesced stores.
constexpr int kScanThreads = 256;
constexpr int kScanWarps = kScanThreads / 32;
constexpr int kScanPer = 8;
constexpr int kScanChunk = kScanThreads * kScanPer;

// Sum of v over the CTA, returned to every thread (s_red: kScanWarps ints).
__device__ __forceinline__ int scan_block_sum(int v, int* s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    int total = 0;
#pragma unroll
    for (int w = 0; w < kScanWarps; ++w) total += s_red[w];
    return total;
}

__global__ void __launch_bounds__(kScanThreads) bin_sum_kernel(SceneTable sc, const uint32_t* __restrict__ bcount_all,
                                                               int32_t* __restrict__ bpart) {
    pdl_wait();
    __shared__ int s_red[kScanWarps];
    const int scene = blockIdx.x, chunk = blockIdx.y;
    const int nbins = sc.prm[scene].nb + 1;
    const int c0 = chunk * kScanChunk;
    if (c0 >= nbins) return;
    const uint32_t* bcount = bcount_all + sc.prm[scene].boff + c0;
    const int m = min(kScanChunk, nbins - c0);
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int i = k * kScanThreads + threadIdx.x;
        if (i < m) sum += (int)bcount[i];
    }
    sum = scan_block_sum(sum, s_red);
    if (threadIdx.x == 0) bpart[(long long)scene * gridDim.y + chunk] = sum;
}

__global__ void __launch_bounds__(kScanThreads) bin_scan_kernel(SceneTable sc, const uint32_t* __restrict__ bcount_all,
                                                                uint32_t* __restrict__ bclear_all,
                                                                const int32_t* __restrict__ bpart,
                                                                int32_t* __restrict__ bstart_all,
                                                                uint32_t* __restrict__ work,
                                                                const uint32_t* __restrict__ cur_nlist,
                                                                const uint32_t* __restrict__ clear_nlist,
                                                                long long* __restrict__ itemoff,
                                                                long long* __restrict__ clroff,
                                                                uint32_t* __restrict__ tstamp) {
    pdl_wait();
    __shared__ int s_val[kScanChunk];
    __shared__ int s_red[kScanWarps];
    __shared__ int s_warp[kScanWarps];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int scene = blockIdx.x, chunk = blockIdx.y;
    if (scene == 0 && chunk == 0 && t == 0) {
        work[0] = 0u;  // P2G items
        work[1] = 0u;  // G2P items
        work[2] = 0u;  // crowded-cell list length
        work[3] = 0u;  // crowded-cell entries taken
        if (tstamp) *tstamp += 1u;  // this ordering's tile stamp
        // Per-scene prefixes: P2G items (kBinZ per listed bin of the current
        // set) and the listed bins of the set to clear.
        long long run = 0, runc = 0;
        for (int s2 = 0; s2 < sc.count; ++s2) {
            itemoff[s2] = run;
            clroff[s2] = runc;
            run += (long long)cur_nlist[s2] * kBinZ;
            runc += (long long)clear_nlist[s2];
        }
        itemoff[sc.count] = run;
        clroff[sc.count] = runc;
    }
    const SimParams& p = sc.prm[scene];
    const int nbins = p.nb + 1;
    const int c0 = chunk * kScanChunk;
    if (c0 >= nbins) return;
    const long long boff = p.boff;
    const uint32_t* bcount = bcount_all + boff + c0;
    uint32_t* bclear = bclear_all + boff + c0;
    int32_t* bstart = bstart_all + boff + c0;
    const int m = min(kScanChunk, nbins - c0);
    // Particles of the scene's earlier chunks.
    int pre = 0;
    for (int i = t; i < chunk; i += kScanThreads) pre += bpart[(long long)scene * gridDim.y + i];
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int i = k * kScanThreads + t;
        s_val[i] = i < m ? (int)bcount[i] : 0;
        if (i < m) bclear[i] = 0u;
    }
    const int carry = (int)p.poff + scan_block_sum(pre, s_red);  // its barrier also publishes s_val
    int v[kScanPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = s_val[t * kScanPer + k];
        sum += v[k];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    int before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kScanWarps; ++w) {
        const int x = s_warp[w];
        before += w < warp ? x : 0;
        total += x;
    }
    int run = carry + before + incl - sum;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        s_val[t * kScanPer + k] = run;
        run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int i = k * kScanThreads + t;
        if (i < m) bstart[i] = s_val[i];
    }
    if (t == 0 && c0 + m == nbins) bstart[m] = carry + total;
}

// The P2G order of a bin's cells (one warp; lane holds the counts of cells
// 4 lane .. 4 lane + 3): occupied cells by count class (floor(log2 count),
// 7 for 128 and more), largest class first, by cell index within a class;
// order[p] = the cell at position p, 0xFF past the occupied cells.  P2G's
// item g of the bin takes positions 32 g .. 32 g + 31, so a warp's lanes hold
// cells of similar counts.  Class counts travel as the bytes of two words
// (classes 0..3 and 4..7; a byte holds at most 128): one warp scan gives the
// cells of each class in lower lanes, and multiplying the totals by
// 0x01010101 gives byte-wise running sums, hence each class's first position.
__device__ __forceinline__ void cell_order(uint4 c, uint8_t* __restrict__ order) {
    const int lane = threadIdx.x & 31;
    const uint32_t cnt[4] = {c.x, c.y, c.z, c.w};
    int cls[4];
    uint32_t lo = 0u, hi = 0u;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        cls[j] = cnt[j] == 0u ? -1 : min(7, 31 - __clz((int)cnt[j]));
        const uint32_t one = cls[j] < 0 ? 0u : 1u << (8 * (cls[j] & 3));
        if (cls[j] < 4) lo += one;
        else hi += one;
    }
    uint32_t ilo = lo, ihi = hi;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t a = __shfl_up_sync(0xffffffffu, ilo, o), b = __shfl_up_sync(0xffffffffu, ihi, o);
        if (lane >= o) ilo += a, ihi += b;
    }
    const uint32_t clo = __shfl_sync(0xffffffffu, ilo, 31) * 0x01010101u;  // byte k: cells of classes <= k
    const uint32_t chi = __shfl_sync(0xffffffffu, ihi, 31) * 0x01010101u + (clo >> 24) * 0x01010101u;
    const int total = (int)(chi >> 24);
    uint32_t seen_lo = ilo - lo, seen_hi = ihi - hi;  // cells of each class in lower lanes, then earlier here
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (cls[j] < 0) continue;
        const int sh = 8 * (cls[j] & 3);
        const bool h = cls[j] >= 4;
        const int upto = (int)(((h ? chi : clo) >> sh) & 0xFFu);  // cells of classes <= cls
        const int ex = (int)(((h ? seen_hi : seen_lo) >> sh) & 0xFFu);
        // First position of the class = cells of larger classes = total - upto.
        order[total - upto + ex] = (uint8_t)(4 * lane + j);
        if (h) seen_hi += 1u << sh;
        else seen_lo += 1u << sh;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (4 * lane + j >= total) order[4 * lane + j] = 0xFFu;
}

// One warp per listed bin of each scene: cstart of its 128 cells = bstart of
// the bin + the exclusive scan of their counts (also written to ccur, the
// cursors the scatter draws slots from).  Then clears the cell
// counters of the other set for the bins on that set's lists (the cells it
// last filled).
__global__ void __launch_bounds__(128) cell_scan_kernel(SceneTable sc, BinSet set, const int32_t* __restrict__ bstart,
                                                        int32_t* __restrict__ cstart, int32_t* __restrict__ ccur,
                                                        uint8_t* __restrict__ corder,
                                                        BinSet clear, const long long* __restrict__ itemoff,
                                                        const long long* __restrict__ clroff,
                                                        const uint32_t* __restrict__ tstamp,
                                                        uint32_t* __restrict__ tmark) {
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const uint32_t stamp = tmark ? *tstamp : 0u;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    // Listed bins of all scenes, one after another (itemoff counts kBinZ items per bin).
    const long long nbins = itemoff[sc.count] / kBinZ;
    for (long long it = gw; it < nbins; it += nw) {
        const int scene = sc.count == 1 ? 0 : scene_of(itemoff, sc.count, it * kBinZ);
        const long long coff = sc.prm[scene].coff, boff = sc.prm[scene].boff;
        const int bin = set.blist[boff + it - itemoff[scene] / kBinZ];
        const size_t c0 = (size_t)coff + (size_t)bin * kBinCells + lane * 4;
        const uint4 c = *reinterpret_cast<const uint4*>(set.ccount + c0);
        const int sum = (int)(c.x + c.y + c.z + c.w);
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int e0 = bstart[boff + bin] + incl - sum;
        int4 st;
        st.x = e0;
        st.y = e0 + (int)c.x;
        st.z = st.y + (int)c.y;
        st.w = st.z + (int)c.z;
        *reinterpret_cast<int4*>(cstart + c0) = st;
        *reinterpret_cast<int4*>(ccur + c0) = st;  // the scatter's cursors start at the cells' first slots
        cell_order(c, corder + (size_t)coff + (size_t)bin * kBinCells);
        // The grid-update tiles this bin's particles reach: tiles bin + (dx,
        // dy, dz), d in {0, 1}^3, lane d.
        const SimParams& ps = sc.prm[scene];
        if (tmark && lane < 8 && bin < ps.nb) {
            const int tx = bin % ps.nbx + (lane & 1), ty = (bin / ps.nbx) % ps.nby + ((lane >> 1) & 1),
                      tz = bin / (ps.nbx * ps.nby) + (lane >> 2);
            if (tx < ps.nbx && ty < ps.nby && tz < ps.nbz) tmark[boff + ((long long)tz * ps.nby + ty) * ps.nbx + tx] = stamp;
        }
    }
    const long long nclear = clroff[sc.count];
    for (long long it = gw; it < nclear; it += nw) {
        const int scene = sc.count == 1 ? 0 : scene_of(clroff, sc.count, it);
        const long long coff = sc.prm[scene].coff, boff = sc.prm[scene].boff;
        const int bin = clear.blist[boff + it - clroff[scene]];
        *reinterpret_cast<uint4*>(clear.ccount + (size_t)coff + (size_t)bin * kBinCells + lane * 4) =
            make_uint4(0u, 0u, 0u, 0u);
    }
}

// gidx[slot] = j: the order by cell, each particle taking the next slot of
// its cell from the cursor ccur[cell] (one atomic per distinct cell of a warp;
// the lanes sharing a cell take consecutive slots in lane order).  A thread
// files kScatterPer particles (block b: particles b * kScatterPer * blockDim
// .. + kScatterPer * blockDim, one blockDim-wide slice per pass), so that the
// cursor atomics of its passes are in flight together.  Thread 0 also resets
// the other set's lists, which cell_scan_kernel has just cleared.
constexpr int kScatterPer = 4;

__global__ void __launch_bounds__(256) bin_scatter_kernel(long long n, int scenes, const int32_t* __restrict__ pcell,
                                                          int32_t* __restrict__ ccur, int32_t* __restrict__ gidx,
                                                          uint32_t* __restrict__ clear_nlist) {
    pdl_wait();
    const long long j0 = blockIdx.x * (long long)blockDim.x * kScatterPer + threadIdx.x;
    if (j0 == 0)
        for (int s2 = 0; s2 < scenes; ++s2) clear_nlist[s2] = 0u;
    const int lane = threadIdx.x & 31;
    int cell[kScatterPer], base[kScatterPer];
    uint32_t peers[kScatterPer];
#pragma unroll
    for (int k = 0; k < kScatterPer; ++k) {
        const long long j = j0 + (long long)k * blockDim.x;
        cell[k] = j < n ? __ldg(pcell + j) : -1;
    }
#pragma unroll
    for (int k = 0; k < kScatterPer; ++k) {
        peers[k] = __match_any_sync(0xffffffffu, cell[k]);
        base[k] = 0;
        if (cell[k] >= 0 && lane == __ffs(peers[k]) - 1) base[k] = atomicAdd(ccur + cell[k], __popc(peers[k]));
    }
#pragma unroll
    for (int k = 0; k < kScatterPer; ++k) {
        const int b = __shfl_sync(0xffffffffu, base[k], __ffs(peers[k]) - 1);
        if (cell[k] >= 0) gidx[b + __popc(peers[k] & lanemask_lt())] = (int32_t)(j0 + (long long)k * blockDim.x);
    }
}

// ---------------------------------------------------------- grid update ----
// Grid update (gridUpdate, kernels.cu:144-196): v = p/m, gravity, SDF
// projection where sdf < 0, PADDING walls.  Writes (mass, v) to vgrid and
// zeroes accum for the next P2G.  The wall tests use the reference's
// unsigned arithmetic (SimConfig fields are uint32_t): x < PADDING and
// x > SIZE-1-PADDING with wrap-around.
// One node at (x, y, z): (mass, v) for the velocity grid from its
// accumulated (mass, momentum) `a`; `inside`: the node's SDF is negative.
__device__ __forceinline__ float4 update_node(const SimParams& p, int x, int y, int z, float4 a, bool inside,
                                             const float* __restrict__ sdf) {
    float4 out = make_float4(a.x, 0.f, 0.f, 0.f);
    if (a.x > 1e-9f) {
        float vx = a.y / a.x;
        float vy = a.z / a.x - p.gravity * p.dt;
        float vz = a.w / a.x;
        if (inside) {
            const float3 nrm = sdf_node_normal(p, sdf, x, y, z);
            const float vdn = vx * nrm.x + vy * nrm.y + vz * nrm.z;
            if (vdn < 0.0f) {
                vx -= nrm.x * vdn;
                vy -= nrm.y * vdn;
                vz -= nrm.z * vdn;
            }
        }
        const uint32_t pad = (uint32_t)p.padding;
        if ((uint32_t)x < pad && vx < 0.f) vx = 0.f;
        if ((uint32_t)y < pad && vy < 0.f) vy = 0.f;
        if ((uint32_t)z < pad && vz < 0.f) vz = 0.f;
        if ((uint32_t)x > (uint32_t)p.sx - 1u - pad && vx > 0.f) vx = 0.f;
        if ((uint32_t)y > (uint32_t)p.sy - 1u - pad && vy > 0.f) vy = 0.f;
        if ((uint32_t)z > (uint32_t)p.sz - 1u - pad && vz > 0.f) vz = 0.f;
        out = make_float4(a.x, vx, vy, vz);
    }
    // Sign bit of the mass: the node's SDF is negative (G2P's obstacle test).
    if (inside) out.x = -out.x;
    return out;
}

// Every node of every scene, one thread per node.
template <bool kBatch>
__global__ void __launch_bounds__(256) grid_update_kernel(SceneTable sc, SimParams p0, long long g_total,
                                                          float4* __restrict__ accum, float4* __restrict__ vgrid,
                                                          const float* __restrict__ sdf_all) {
    pdl_wait();
    __shared__ SimParams s_prm[kBatch ? kTableScenes : 1];
    __shared__ long long s_first[kBatch ? kTableScenes + 1 : 1];
    __shared__ int s_range[2];
    const long long gi = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const SceneLookup<kBatch> look(sc, sc.goff, s_prm, s_first, s_range, blockIdx.x * (long long)blockDim.x,
                                   min((blockIdx.x + 1) * (long long)blockDim.x, g_total));
    if (gi >= g_total) return;
    const SimParams& p = kBatch ? look.params(look.scene(gi)) : p0;
    const int idx = (int)(gi - p.goff);
    const float* sdf = sdf_all + p.goff;
    const float4 a = accum[gi];
    const bool inside = __ldg(sdf + idx) < 0.0f;
    const int x = idx % p.sx, y = (idx / p.sx) % p.sy, z = idx / (p.sx * p.sy);
    vgrid[gi] = update_node(p, x, y, z, a, inside, sdf);
    if (a.x != 0.f || a.y != 0.f || a.z != 0.f || a.w != 0.f) accum[gi] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// One warp per node tile (TileMarks; global bin entries, the scene found by
// binary search over the scenes' first entries): lane l takes the nodes
// (x0 + l % 8, y0 + l / 8, z0 + c), c = 0..3.  A tile marked by this
// substep's ordering is updated like grid_update_kernel; a tile updated
// before but not marked now holds no accumulated mass any more and is reset to
// zero; every other tile is already zero and is skipped.  Every node the
// substep's particles reach lies in a marked tile, and G2P reads no other.
template <bool kBatch>
__global__ void __launch_bounds__(256) grid_tiles_kernel(SceneTable sc, SimParams p0, TileMarks tiles,
                                                         float4* __restrict__ accum_all, float4* __restrict__ vgrid_all,
                                                         const float* __restrict__ sdf_all) {
    pdl_wait();
    const long long gt = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gt >= tiles.count) return;  // warp-uniform
    int scene = 0;
    if constexpr (kBatch) {
        int lo = 0, hi = sc.count - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(&sc.prm[mid].boff) <= gt) lo = mid;
            else hi = mid - 1;
        }
        scene = lo;
    }
    const SimParams& p = kBatch ? sc.prm[scene] : p0;
    const int t = (int)(gt - p.boff);
    if (t >= p.nb) return;  // the overflow bin's entries hold no tile
    float4* accum = accum_all + p.goff;
    float4* vgrid = vgrid_all + p.goff;
    const float* sdf = sdf_all + p.goff;
    const bool act = tiles.mark[gt] == *tiles.stamp;
    const bool dirty = tiles.dirty[gt] != 0;
    if (!act && !dirty) return;
    __syncwarp();  // every lane has read the flag lane 0 rewrites below
    const int x = (t % p.nbx) * kBinX - 2 + (lane & 7);
    const int y = ((t / p.nbx) % p.nby) * kBinY - 2 + (lane >> 3);
    const int z0 = (t / (p.nbx * p.nby)) * kBinZ - 2;
    const bool xy = (unsigned)x < (unsigned)p.sx && (unsigned)y < (unsigned)p.sy;
    if (act) {
        float4 a[kBinZ];
        bool inside[kBinZ];
#pragma unroll
        for (int c = 0; c < kBinZ; ++c) {
            const bool ok = xy && (unsigned)(z0 + c) < (unsigned)p.sz;
            const int i = ok ? node_index(p, x, y, z0 + c) : 0;
            a[c] = ok ? accum[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            inside[c] = ok && __ldg(sdf + i) < 0.0f;
        }
#pragma unroll
        for (int c = 0; c < kBinZ; ++c) {
            if (!xy || (unsigned)(z0 + c) >= (unsigned)p.sz) continue;
            const int i = node_index(p, x, y, z0 + c);
            vgrid[i] = update_node(p, x, y, z0 + c, a[c], inside[c], sdf);
            if (a[c].x != 0.f || a[c].y != 0.f || a[c].z != 0.f || a[c].w != 0.f)
                accum[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    } else {
#pragma unroll
        for (int c = 0; c < kBinZ; ++c)
            if (xy && (unsigned)(z0 + c) < (unsigned)p.sz)
                vgrid[node_index(p, x, y, z0 + c)] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncwarp();
    if (lane == 0 && act != dirty) tiles.dirty[gt] = act ? 1 : 0;
}

// ------------------------------------------------------------------ G2P ----
// G2P (g2PTransfer, kernels.cu:199-280).  Thread j reads the particle at
// slot gidx[j] of the old state and writes slot j of the new one, so the
// state ends up ordered by cell.  It also files the new position into the
// counter set of the next substep.
// G2P modes: the plain substep; the uncorrected large step; the learned
// large step (features -> MLP -> velocity correction before advection); the
// collection probe (the uncorrected large step, recording each particle's
// features and final velocity by original index).  Large steps advect with
// v_old + blend (v_new - v_old), blend = (R + 1) / (2R) for R plain substeps:
// R substeps under a constant acceleration move a particle by exactly that.
enum G2PMode : int { kG2PPlain = 0, kG2PLearned = 1, kG2PCollect = 2, kG2PLarge = 3, kG2PLearnedTc = 4 };

// Particles per thread of a G2P instantiation: two for the batched plain
// mode (records staged in dynamic shared memory, kPer x 3 x blockDim float4),
// one otherwise.  Measured per substep on the 64-scene batch, two per thread
// cut G2P by 5-8 %; on one scene (fewer registers, more warps per SM) two
// per thread cost 5 % and four 20 %.
__host__ __device__ constexpr int g2p_per_thread(bool batch, int mode, bool wide) {
    return (mode == 0 && !wide && batch) ? 2 : 1;
}

// CTAs per SM: the learned tcgen05 mode fits four (64 registers, 128 TMEM
// columns and about 45 KB of shared memory each), so one CTA's MMA waits
// overlap the other three's work; mma.sync learned, collect and batched
// modes need more registers.
// kWide: 256-thread CTAs free to use up to 255 registers (one CTA per SM,
// every node load of a particle in flight at once) instead of 64 registers
// and four CTAs per SM; chosen by the autotuner.
template <bool kBatch, int kMode, bool kWide = false>
__global__ void __launch_bounds__(256, kWide ? 1 : (kMode == 1 ? 2 : ((kBatch || kMode == 2) ? 3 : 4))) g2p_kernel(SceneTable sc, SimParams p0, long long n_total, const float* __restrict__ Pin,
                                                  float* __restrict__ Pout, const int32_t* __restrict__ gidx,
                                                  const int32_t* __restrict__ sig_in, int32_t* __restrict__ sig_out,
                                                  const float4* __restrict__ vgrid_all, const float* __restrict__ sdf_all,
                                                  int32_t* __restrict__ pcell, BinSet next,
                                                  uint32_t* __restrict__ health, LearnArgs la) {
    pdl_wait();
    __shared__ SimParams s_prm[kBatch ? kTableScenes : 1];
    __shared__ long long s_first[kBatch ? kTableScenes + 1 : 1];
    __shared__ int s_range[2];
    __shared__ __align__(16) unsigned char s_mlp_raw[kMode == kG2PLearned ? sizeof(MlpPacked) : 16];
    __shared__ uint32_t s_stage[kMode == kG2PLearned ? 8 * 32 * kMlpStageStride : 1];
    extern __shared__ __align__(1024) unsigned char s_dyn[];  // MlpTcSmem in the tcgen05 mode
    if constexpr (kMode == kG2PLearned) {
        const uint4* src = reinterpret_cast<const uint4*>(la.mlp);
        uint4* dst = reinterpret_cast<uint4*>(s_mlp_raw);
        for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) dst[i] = __ldg(src + i);
        __syncthreads();
    }
    if constexpr (kMode == kG2PLearnedTc) {
        MlpTcSmem& ts = *reinterpret_cast<MlpTcSmem*>(s_dyn);
        const uint4* src = reinterpret_cast<const uint4*>(la.mlp_tc);
        uint4* dst = reinterpret_cast<uint4*>(&ts.w);
        for (int i = threadIdx.x; i < (int)(sizeof(MlpTc) / 16); i += blockDim.x) dst[i] = __ldg(src + i);
        mlp_tc_begin(ts, la.wait_test);  // TMEM columns and the mbarrier; synchronises the CTA
    }
    constexpr int kPer = g2p_per_thread(kBatch, kMode, kWide);
    const long long cta0 = (long long)blockIdx.x * kPer * blockDim.x;  // this CTA's particles: [cta0, cta1)
    const SceneLookup<kBatch> look(sc, sc.poff, s_prm, s_first, s_range, cta0,
                                   min(cta0 + (long long)kPer * blockDim.x, n_total));
    // The plain mode takes kPer particles per thread (block b: particles
    // b * kPer * blockDim .. + kPer * blockDim, one blockDim-wide slice per
    // pass) and requests all their positions and F up front, into shared
    // memory with cp.async, so that a record's load overlaps the passes
    // before it.  Every lane makes all kPer passes: filing is warp-wide.
    float4* s_rec = reinterpret_cast<float4*>(s_dyn);  // [kPer][3][blockDim] when kPer > 1
    if constexpr (kPer > 1) {
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const long long jk = ((long long)blockIdx.x * kPer + k) * blockDim.x + threadIdx.x;
            if (jk < n_total) {
                const float4* qk = reinterpret_cast<const float4*>(Pin + (size_t)__ldg(gidx + jk) * kAFloats);
#pragma unroll
                for (int v = 0; v < 3; ++v) cp_async16(s_rec + (k * 3 + v) * blockDim.x + threadIdx.x, qk + v);
            }
        }
        cp_async_commit();
    }
#pragma unroll 1
    for (int k = 0; k < kPer; ++k) {
    const long long jj = ((long long)blockIdx.x * kPer + k) * blockDim.x + threadIdx.x;
    const bool valid = jj < n_total;
    const long long j = valid ? jj : n_total - 1;  // idle lanes redo the last particle and store nothing
    const int scene = look.scene(j);
    const SimParams& p = kBatch ? look.params(scene) : p0;
    const float4* vgrid = vgrid_all + p.goff;
    const float* sdf = sdf_all + p.goff;
    const int src = __ldg(gidx + j);
    const float4* q = reinterpret_cast<const float4*>(Pin + (size_t)src * kAFloats);
    float4 q0, q1, q2;
    if constexpr (kPer > 1) {
        if (k == 0) cp_async_wait<0>();  // every record of this thread has arrived
        const float4* r = s_rec + (k * 3) * blockDim.x + threadIdx.x;
        q0 = valid ? r[0] : make_float4(0.f, 0.f, 0.f, 0.f);
        q1 = valid ? r[blockDim.x] : make_float4(0.f, 0.f, 0.f, 0.f);
        q2 = valid ? r[2 * blockDim.x] : make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
        // Records are 96 bytes from a cudaMalloc'd base, so each starts on a
        // 32-byte boundary: one 32-byte load (sm_100 ld.global.v8) for the
        // position and F00..F04, one 16-byte load for F05..F08.
        asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=f"(q0.x), "=f"(q0.y), "=f"(q0.z), "=f"(q0.w), "=f"(q1.x), "=f"(q1.y), "=f"(q1.z), "=f"(q1.w)
            : "l"(q));
        q2 = __ldg(q + 2);
    }
    float4 qv = make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (kMode != kG2PPlain) qv = __ldg(q + 3);  // old velocity
    const float pos[3] = {q0.x, q0.y, q0.z};
    const float F[9] = {q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};

    const int bx = stencil_base(pos[0]), by = stencil_base(pos[1]), bz = stencil_base(pos[2]);
    // f = pos - base is exact, so f - o equals pos - (base + o) bit for bit
    // and axis_weights gives bspline_weight's values.
    const float fx = pos[0] - (float)bx, fy = pos[1] - (float)by, fz = pos[2] - (float)bz;
    float wx[3], wy[3], wz[3];
    axis_weights(fx, 1.0f, wx);
    axis_weights(fy, 1.0f, wy);
    axis_weights(fz, 1.0f, wz);
    // Interpolation sums (g2PTransfer's loop, kernels.cu:214-235).  The plain,
    // large and collection modes take them separably per axis: with o =
    // (a, b, c) the node offset and x_node - x_p = (o - 1) - (f - 1),
    //   v' = sum w v,   C' = 4 (M - v' (f - 1)^T),   M[k][d] = sum w v_k (o_d - 1),
    // each row of three nodes along x reduced first (S0 = sum_a wx v, S1 =
    // sum_a wx (a - 1) v) before its weight wy wz is applied: a quarter fewer
    // instructions.  The learned modes sum node by node (the reference's
    // form), which holds fewer values live next to the MLP's registers: the
    // row form made the tcgen05 learned G2P spill three times as much and run
    // 7 % slower.
    float tv[3] = {0.f, 0.f, 0.f}, tc[9], tm = 0.f;
    // Set when a stencil node lies outside the grid or inside an obstacle:
    // only then can the SDF at the new position be negative (see below).
    uint32_t sdf_risk = 0u;
    const int plane = p.sx * p.sy;
    // Whole stencil inside the grid (almost every particle): no per-node
    // bounds tests.  Nodes outside the grid add nothing.
    const bool inside = p.sx >= 3 && p.sy >= 3 && p.sz >= 3 && (unsigned)bx <= (unsigned)(p.sx - 3) &&
                        (unsigned)by <= (unsigned)(p.sy - 3) && (unsigned)bz <= (unsigned)(p.sz - 3);
    constexpr bool kRowSums = kMode != kG2PLearned && kMode != kG2PLearnedTc;
    if constexpr (kRowSums) {
        float M[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) M[k] = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const int z = bz + c, y = by + b;
                float4 g[3];
                if (inside) {
                    const float4* row = vgrid + ((size_t)z * plane + (size_t)y * p.sx + bx);
#pragma unroll
                    for (int a = 0; a < 3; ++a) g[a] = __ldg(row + a);
                } else {
                    const bool zy = (unsigned)z < (unsigned)p.sz && (unsigned)y < (unsigned)p.sy;
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const bool ok = zy && (unsigned)(bx + a) < (unsigned)p.sx;
                        g[a] = ok ? __ldg(vgrid + ((size_t)z * plane + (size_t)y * p.sx + bx + a))
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
                        if (!ok) sdf_risk = 1u;
                    }
                }
                sdf_risk |= (__float_as_uint(g[0].x) | __float_as_uint(g[1].x) | __float_as_uint(g[2].x)) >> 31;
                const float s0[3] = {wx[0] * g[0].y + wx[1] * g[1].y + wx[2] * g[2].y,
                                     wx[0] * g[0].z + wx[1] * g[1].z + wx[2] * g[2].z,
                                     wx[0] * g[0].w + wx[1] * g[1].w + wx[2] * g[2].w};
                const float s1[3] = {wx[2] * g[2].y - wx[0] * g[0].y, wx[2] * g[2].z - wx[0] * g[0].z,
                                     wx[2] * g[2].w - wx[0] * g[0].w};
                const float wyz = wy[b] * wz[c];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    tv[k] += wyz * s0[k];
                    M[3 * k + 0] += wyz * s1[k];
                    if (b == 0) M[3 * k + 1] -= wyz * s0[k];
                    if (b == 2) M[3 * k + 1] += wyz * s0[k];
                    if (c == 0) M[3 * k + 2] -= wyz * s0[k];
                    if (c == 2) M[3 * k + 2] += wyz * s0[k];
                }
                if constexpr (kMode != kG2PPlain)
                    tm += wyz * (wx[0] * fabsf(g[0].x) + wx[1] * fabsf(g[1].x) + wx[2] * fabsf(g[2].x));
            }
        }
        const float gx = fx - 1.0f, gy = fy - 1.0f, gz = fz - 1.0f;  // exact
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            tc[3 * k + 0] = 4.0f * (M[3 * k + 0] - tv[k] * gx);
            tc[3 * k + 1] = 4.0f * (M[3 * k + 1] - tv[k] * gy);
            tc[3 * k + 2] = 4.0f * (M[3 * k + 2] - tv[k] * gz);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) tc[k] = 0.f;
        // One node of the stencil, offsets (a, b, c), `row` = node (base x, y, z).
        auto gather = [&](int a, int b, int c, const float4* row) {
            const float dxv = -(fx - (float)a), dyv = -(fy - (float)b), dzv = -(fz - (float)c);
            const float4 g = __ldg(row + a);
            sdf_risk |= __float_as_uint(g.x) >> 31;
            const float w = wx[a] * wy[b] * wz[c];
            tv[0] += w * g.y;
            tv[1] += w * g.z;
            tv[2] += w * g.w;
            tm += w * fabsf(g.x);
            const float term = 4.0f * w;
            tc[0] += term * g.y * dxv;
            tc[1] += term * g.y * dyv;
            tc[2] += term * g.y * dzv;
            tc[3] += term * g.z * dxv;
            tc[4] += term * g.z * dyv;
            tc[5] += term * g.z * dzv;
            tc[6] += term * g.w * dxv;
            tc[7] += term * g.w * dyv;
            tc[8] += term * g.w * dzv;
        };
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int z = bz + c;
            if (!inside && (unsigned)z >= (unsigned)p.sz) {
                sdf_risk = 1u;
                continue;
            }
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const int y = by + b;
                if (!inside && (unsigned)y >= (unsigned)p.sy) {
                    sdf_risk = 1u;
                    continue;
                }
                const float4* row = vgrid + ((size_t)z * plane + (size_t)y * p.sx + bx);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    if (!inside && (unsigned)(bx + a) >= (unsigned)p.sx) {
                        sdf_risk = 1u;
                        continue;
                    }
                    gather(a, b, c, row);
                }
            }
        }
    }
    if constexpr (kMode == kG2PLearned || kMode == kG2PCollect || kMode == kG2PLearnedTc) {
        float f[kMlpIn];
#pragma unroll
        for (int k = 0; k < 9; ++k) f[k] = tc[k];
        f[9] = tv[0], f[10] = tv[1], f[11] = tv[2];
        f[12] = tm * (p.pvol / p.pmass) - 1.0f;
        f[13] = f[14] = f[15] = 0.f;
        const float phi = sdf_trilinear(p, sdf, pos[0], pos[1], pos[2]);
        if (fabsf(phi) < 4.0f) {
            const float3 nrm = sdf_gradient_dir(p, sdf, pos[0], pos[1], pos[2]);
            const float s = phi * (1.0f - fabsf(phi) * 0.25f);
            f[13] = nrm.x * s, f[14] = nrm.y * s, f[15] = nrm.z * s;
        }
        if constexpr (kMode == kG2PLearned || kMode == kG2PLearnedTc) {
            float dv[3];
            if constexpr (kMode == kG2PLearned) {
                mlp_forward_warp(*reinterpret_cast<const MlpPacked*>(s_mlp_raw),
                                 s_stage + (threadIdx.x >> 5) * 32 * kMlpStageStride, f, dv);
            } else {
                MlpTcSmem& ts = *reinterpret_cast<MlpTcSmem*>(s_dyn);
                mlp_forward_tc(ts, f, dv);
                mlp_tc_end(ts);  // TMEM freed before the rest of the particle update
                if (ts.failed && threadIdx.x == 0) atomicOr(la.status, kStatusTimeout);
            }
            tv[0] += dv[0], tv[1] += dv[1], tv[2] += dv[2];
            // The fallback statistics, summed over particles into la.stat[0..2]:
            //  [0] the predicted relative density change of the step,
            //      |1 / det(I + dt C) - 1|;
            //  [1] the predicted density's deviation from rest density,
            //      |rho / rho0 / det(I + dt C) - 1|, with rho / rho0 the
            //      interpolated grid mass over the seeding density;
            //  [2] the current density's deviation from rest, |rho / rho0 - 1|.
            float T[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) T[k] = ((k % 4 == 0) ? 1.0f : 0.0f) + p.dt * tc[k];
            const float inv_det = 1.0f / det3(T), rho = tm * (p.pvol / p.pmass);
            float dev[3] = {fabsf(inv_det - 1.0f), fabsf(rho * inv_det - 1.0f), fabsf(rho - 1.0f)};
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (!valid) dev[q] = 0.f;
                if (!(dev[q] < 1e30f)) dev[q] = 1e30f;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) dev[q] += __shfl_xor_sync(0xffffffffu, dev[q], o);
            }
            if ((threadIdx.x & 31) == 0) {
                atomicAdd(la.stat, dev[0]);
                atomicAdd(la.stat + 1, dev[1]);
                atomicAdd(la.stat + 2, dev[2]);
            }
        } else if (valid) {  // collection probe: la.feat holds n rows
            float* fo = la.feat + (size_t)__ldg(sig_in + src) * kMlpIn;
#pragma unroll
            for (int k = 0; k < kMlpIn; k += 4) *reinterpret_cast<float4*>(fo + k) = make_float4(f[k], f[k + 1], f[k + 2], f[k + 3]);
        }
    }
    // F' = (I + DT C') F with the J < 0.3 volume rescue (calculateNewF,
    // common.cuh:255-261; kernels.cu:237-247).
    float T[9], NF[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) T[k] = ((k % 4 == 0) ? 1.0f : 0.0f) + p.dt * tc[k];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            NF[r * 3 + c] = T[r * 3 + 0] * F[0 * 3 + c] + T[r * 3 + 1] * F[1 * 3 + c] + T[r * 3 + 2] * F[2 * 3 + c];
    const float J = det3(NF);
    if (J < 0.3f) {
        const float scale = powf(0.3f / J, 1.0f / 3.0f);
#pragma unroll
        for (int k = 0; k < 9; ++k) NF[k] *= scale;
    }
    // Advect, then push out of obstacles (kernels.cu:249-270).
    float av[3] = {tv[0], tv[1], tv[2]};
    if constexpr (kMode != kG2PPlain) {
        av[0] = qv.x + la.blend * (tv[0] - qv.x);
        av[1] = qv.y + la.blend * (tv[1] - qv.y);
        av[2] = qv.z + la.blend * (tv[2] - qv.z);
    }
    const float sx = av[0] * p.dt, sy = av[1] * p.dt, sz = av[2] * p.dt;
    float nx = pos[0] + sx, ny = pos[1] + sy, nz = pos[2] + sz;
    // The stencil nodes are base..base+2 and pos - base lies in [0.5, 1.5):
    // a move of at most 0.25 per axis keeps every corner of the new
    // position's cell among them, so with no stencil node outside the grid or
    // with a negative SDF the trilinear SDF there is a convex combination of
    // non-negative values and the obstacle test below cannot fire.
    const bool far = !sdf_risk && fabsf(sx) <= 0.25f && fabsf(sy) <= 0.25f && fabsf(sz) <= 0.25f;
    const float dist = far ? 0.0f : sdf_trilinear(p, sdf, nx, ny, nz);
    if (dist < 0.0f) {
        const float3 nrm = sdf_gradient_dir(p, sdf, nx, ny, nz);
        nx -= nrm.x * dist;
        ny -= nrm.y * dist;
        nz -= nrm.z * dist;
        const float vdn = tv[0] * nrm.x + tv[1] * nrm.y + tv[2] * nrm.z;
        if (vdn < 0.0f) {
            tv[0] -= nrm.x * vdn;
            tv[1] -= nrm.y * vdn;
            tv[2] -= nrm.z * vdn;
        }
    }
    int bin = -1, gcell = -1, gbin = -1;
    if (valid) {
        gcell = (int)p.coff + cell_of(p, nx, ny, nz, &bin);
        gbin = (int)p.boff + bin;
    }
    file_particle(gcell, gbin, bin, scene, p.boff, next);
    if (!valid) continue;  // only the last passes of the last block have idle lanes
    float4* o = reinterpret_cast<float4*>(Pout + (size_t)j * kAFloats);
    {
        // Three 32-byte stores (st.global.v8) of the 96-byte record: half the
        // store instructions of 16-byte vectors.
        const float w[24] = {nx, ny, nz, NF[0], NF[1], NF[2], NF[3], NF[4], NF[5], NF[6], NF[7], NF[8],
                             tv[0], tv[1], tv[2], tc[0], tc[1], tc[2], tc[3], tc[4], tc[5], tc[6], tc[7], tc[8]};
#pragma unroll
        for (int h = 0; h < 3; ++h)
            asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(o + 2 * h),
                         "f"(w[8 * h + 0]), "f"(w[8 * h + 1]), "f"(w[8 * h + 2]), "f"(w[8 * h + 3]),
                         "f"(w[8 * h + 4]), "f"(w[8 * h + 5]), "f"(w[8 * h + 6]), "f"(w[8 * h + 7])
                         : "memory");
    }
    sig_out[j] = __ldg(sig_in + src);
    pcell[j] = gcell;
    if constexpr (kMode == kG2PCollect) {
        float* vo = la.vel + (size_t)__ldg(sig_in + src) * 3;
        vo[0] = tv[0], vo[1] = tv[1], vo[2] = tv[2];
    }

    uint32_t flags = 0;
    if (!(isfinite(nx) && isfinite(ny) && isfinite(nz) && isfinite(tv[0]) && isfinite(tv[1]) && isfinite(tv[2])))
        flags |= 1u;
    if (!(nx >= 0.f && nx < (float)p.sx && ny >= 0.f && ny < (float)p.sy && nz >= 0.f && nz < (float)p.sz))
        flags |= 2u;
    if (flags) atomicOr(health, flags);
    }
}

// ------------------------------------------------------- state transfer ----
// Field of the device state that holds host plane k (MPM_POS_X.., 0..23).
__device__ __forceinline__ int field_of_plane(int k) {
    if (k < 3) return kAPos + k;
    if (k < 6) return kAVel + (k - 3);
    if (k < 15) return kAC + (k - 6);
    return kAF + (k - 15);
}

__global__ void __launch_bounds__(256) state_import_kernel(SimParams p, const float* __restrict__ in,
                                                           float* __restrict__ P, int32_t* __restrict__ sigma,
                                                           bool init_rules) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const long long n = p.n;
    float v[kAFloats];
#pragma unroll
    for (int k = 0; k < kAFloats; ++k) v[field_of_plane(k)] = __ldg(in + k * n + i);
    if (init_rules) v[kAF + 0] = v[kAF + 4] = v[kAF + 8] = 1.0f;
    float4* o = reinterpret_cast<float4*>(P + (size_t)i * kAFloats);
#pragma unroll
    for (int k = 0; k < 6; ++k) o[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    sigma[i] = (int32_t)(p.poff + i);
}

// keys[sigma[j]] = setKeys' Morton key of the particle in slot j
// (kernels.cu:361-371): the keys in original particle order.
__global__ void __launch_bounds__(256) reference_keys_kernel(SimParams p, const float* __restrict__ P,
                                                             const int32_t* __restrict__ sigma,
                                                             int32_t* __restrict__ keys) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.n) return;
    const float4 q = __ldg(reinterpret_cast<const float4*>(P + (size_t)j * kAFloats));
    keys[__ldg(sigma + j) - p.poff] = morton_key(q.x, q.y, q.z);
}

__global__ void __launch_bounds__(256) state_export_kernel(SimParams p, const float* __restrict__ P,
                                                           const int32_t* __restrict__ sigma,
                                                           float* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.n) return;
    const long long n = p.n;
    const long long o = __ldg(sigma + j) - p.poff;
    const float4* q = reinterpret_cast<const float4*>(P + (size_t)j * kAFloats);
    float v[kAFloats];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float4 t = __ldg(q + k);
        v[4 * k] = t.x;
        v[4 * k + 1] = t.y;
        v[4 * k + 2] = t.z;
        v[4 * k + 3] = t.w;
    }
#pragma unroll
    for (int k = 0; k < kAFloats; ++k) out[k * n + o] = v[field_of_plane(k)];
    out[24 * n + o] = p.pvol;
    out[25 * n + o] = p.pmass;
}

__global__ void __launch_bounds__(256) positions_export_kernel(SimParams p, const float* __restrict__ P,
                                                               const int32_t* __restrict__ sigma,
                                                               float* __restrict__ xyz) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.n) return;
    const long long o = __ldg(sigma + j) - p.poff;
    const float4 q = __ldg(reinterpret_cast<const float4*>(P + (size_t)j * kAFloats));
    xyz[3 * o + 0] = q.x;
    xyz[3 * o + 1] = q.y;
    xyz[3 * o + 2] = q.z;
}

__global__ void __launch_bounds__(256) grid_export_kernel(SimParams p, const float4* __restrict__ grid,
                                                          float* __restrict__ planes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.g) return;
    const float4 v = __ldg(grid + i);
    const long long g = p.g;
    planes[i] = fabsf(v.x);  // the sign bit of a velocity node's mass marks a negative SDF
    planes[g + i] = v.y;
    planes[2 * g + i] = v.z;
    planes[3 * g + i] = v.w;
}

__global__ void __launch_bounds__(256) identity_kernel(int32_t* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = i;
}

__global__ void __launch_bounds__(256) fill_kernel(float* __restrict__ dst, long long count, float value) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = value;
}

// The learned step's accept / reject decision on the device: the mean of the
// statistic the rule names (la.stat sums, kernels above) against the
// threshold; reject (NaN included) sets the graph's conditional, which runs
// the fallback body.  counters[0] / [1] count accepted and rejected steps;
// last[0..2] receive the three means, last[3] the compared statistic.
__global__ void learned_decide_kernel(const float* __restrict__ stat, long long n, int rule, float threshold,
                                      cudaGraphConditionalHandle fallback, long long* __restrict__ counters,
                                      float* __restrict__ last) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const float inv = n > 0 ? 1.0f / (float)n : 0.0f;
    const float m0 = stat[0] * inv, m1 = stat[1] * inv, m2 = stat[2] * inv;
    const float st = rule == 1 ? m1 : (rule == 2 ? m1 - m2 : m0);
    const bool reject = !(st <= threshold);
    cudaGraphSetConditional(fallback, reject ? 1u : 0u);
    counters[reject ? 1 : 0] += 1;
    last[0] = m0;
    last[1] = m1;
    last[2] = m2;
    last[3] = st;
}

// dst[i] = src[i] for i < count 32-bit words (16-byte vectors when both
// pointers and the count allow).
__global__ void __launch_bounds__(256) copy_words_kernel(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                                                         long long count, bool vec) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (vec) {
        uint4* d = reinterpret_cast<uint4*>(dst);
        const uint4* q = reinterpret_cast<const uint4*>(src);
        for (long long i = i0; i < count / 4; i += stride) d[i] = __ldg(q + i);
    } else {
        for (long long i = i0; i < count; i += stride) dst[i] = __ldg(src + i);
    }
}

inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

// Launches a substep kernel (one that starts with pdl_wait) with programmatic
// stream serialisation.
template <typename... P, typename... A>
void launch_dep(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...);
}

}  // namespace

int launch_bin_count(const SceneTable& sc, long long n, const float* P, int32_t* pcell, const BinSet& set,
                     cudaStream_t st) {
    if (n <= 0) return 0;
    bin_count_kernel<<<blocks_for(n, 256), 256, 0, st>>>(sc, n, P, pcell, set);
    return 1;
}

int bin_scan_chunks(long long bins) { return (int)std::max(1LL, (bins + kScanChunk - 1) / kScanChunk); }

int launch_bin_order(const SceneTable& sc, long long n, long long bins_total, const BinSet& cur, const BinSet& other,
                     int32_t* bstart, int32_t* cstart, const int32_t* pcell, int32_t* ccur, int32_t* gidx,
                     uint8_t* corder, long long* itemoff, long long* clroff, uint32_t* work, int32_t* bpart,
                     int scan_chunks, const TileMarks& tiles, cudaStream_t st) {
    if (n <= 0) return 0;
    const dim3 scan_grid((unsigned)sc.count, (unsigned)scan_chunks);
    launch_dep(bin_sum_kernel, scan_grid, kScanThreads, 0, st, sc, cur.bcount, bpart);
    launch_dep(bin_scan_kernel, scan_grid, kScanThreads, 0, st, sc, cur.bcount, other.bcount, bpart, bstart, work, cur.nlist,
                                                       other.nlist, itemoff, clroff, tiles.stamp);
    const int ctas = (int)std::max(1LL, std::min((long long)blocks_for(bins_total * 32, 128), 148LL * 8));
    launch_dep(cell_scan_kernel, ctas, 128, 0, st, sc, cur, bstart, cstart, ccur, corder, other, itemoff, clroff,
               tiles.stamp, tiles.mark);
    launch_dep(bin_scatter_kernel, blocks_for(n, 256 * kScatterPer), 256, 0, st, n, sc.count, pcell, ccur, gidx, other.nlist);
    return 4;
}

int p2g_max_ctas_per_sm() {
    int k = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, p2g_kernel, 32, 0) != cudaSuccess) {
        cudaGetLastError();
        return kP2GWarpsPerSM;
    }
    return k;
}

int launch_p2g(const SceneTable& sc, long long n, long long bins_total, const float* P, const int32_t* gidx,
               const int32_t* cstart, const BinSet& cur, const uint8_t* corder, const long long* itemoff,
               uint32_t* work, float4* accum, int4* crowd, int crowd_cap, uint32_t* status, cudaStream_t st,
               int ctas_per_sm, int cell_cap) {
    if (n <= 0) return 0;
    const int per_sm = ctas_per_sm > 0 ? ctas_per_sm : kP2GWarpsPerSM;
    const int cap = cell_cap > 0 ? cell_cap : 0;
    const int warps = (int)std::min(bins_total * kBinZ, 148LL * per_sm);
    launch_dep(p2g_kernel, warps, 32, 0, st, sc, P, gidx, cstart, cur, corder, itemoff, work, accum, crowd, crowd_cap, status,
                                     cap);
    launch_dep(p2g_crowd_kernel, 148 * kP2GWarpsPerSM, 32, 0, st, sc, P, gidx, crowd, crowd_cap, work, accum, status);
    return 2;
}

int launch_grid_update(const SceneTable& sc, const SimParams& p0, long long g_total, float4* accum, float4* vgrid,
                       const float* sdf, const TileMarks& tiles, cudaStream_t st, int block) {
    if (g_total <= 0) return 0;
    const int b = (block == 128 || block == 256) ? block : 256;
    if (tiles.mark) {
        if (sc.count == 1)
            launch_dep(grid_tiles_kernel<false>, blocks_for(tiles.count, 8), 256, 0, st, sc, p0, tiles, accum, vgrid,
                       sdf);
        else
            launch_dep(grid_tiles_kernel<true>, blocks_for(tiles.count, 8), 256, 0, st, sc, p0, tiles, accum, vgrid,
                       sdf);
        return 1;
    }
    if (sc.count == 1)
        launch_dep(grid_update_kernel<false>, blocks_for(g_total, b), b, 0, st, sc, p0, g_total, accum, vgrid, sdf);
    else
        launch_dep(grid_update_kernel<true>, blocks_for(g_total, b), b, 0, st, sc, p0, g_total, accum, vgrid, sdf);
    return 1;
}

int launch_g2p(const SceneTable& sc, const SimParams& p0, long long n, const float* Pin, float* Pout,
               const int32_t* gidx, const int32_t* sig_in, int32_t* sig_out, const float4* vgrid, const float* sdf,
               int32_t* pcell, const BinSet& next, uint32_t* health, cudaStream_t st,
               const LearnArgs* learn, int block) {
    if (n <= 0) return 0;
    const LearnArgs la = learn ? *learn : LearnArgs{};
    const unsigned grid = blocks_for(n, 256);
    if (learn && sc.count == 1 && la.mlp_tc) {
        launch_dep(g2p_kernel<false, kG2PLearnedTc>, grid, 256, sizeof(MlpTcSmem), st,
            sc, p0, n, Pin, Pout, gidx, sig_in, sig_out, vgrid, sdf, pcell, next, health, la);
        return 1;
    }
    // Plain G2P: 128- or 256-thread CTAs, or 512 = the register-wide 256-thread
    // variant (the learned modes stage 8 warps of MLP inputs and always run 256).
    const bool wide = block == 512;
    const int pb = wide ? 256 : ((block == 128 || block == 256) ? block : 256);
    if (learn && sc.count == 1 && la.mlp)
        launch_dep(g2p_kernel<false, kG2PLearned>, grid, 256, 0, st, sc, p0, n, Pin, Pout, gidx, sig_in, sig_out, vgrid, sdf,
                                                             pcell, next, health, la);
    else if (learn && sc.count == 1 && la.feat)
        launch_dep(g2p_kernel<false, kG2PCollect>, grid, 256, 0, st, sc, p0, n, Pin, Pout, gidx, sig_in, sig_out, vgrid, sdf,
                                                             pcell, next, health, la);
    else if (learn && sc.count == 1)
        launch_dep(g2p_kernel<false, kG2PLarge>, grid, 256, 0, st, sc, p0, n, Pin, Pout, gidx, sig_in, sig_out, vgrid, sdf,
                                                           pcell, next, health, la);
    else if (sc.count == 1 && wide)
        launch_dep(g2p_kernel<false, kG2PPlain, true>, blocks_for(n, pb), pb, 0, st, sc, p0, n, Pin, Pout, gidx, sig_in,
                                                                             sig_out, vgrid, sdf, pcell, next,
                                                                             health, la);
    else if (sc.count == 1)
        launch_dep(g2p_kernel<false, kG2PPlain>, blocks_for(n, pb), pb, 0, st, sc, p0, n, Pin, Pout, gidx, sig_in, sig_out,
                                                                       vgrid, sdf, pcell, next, health, la);
    else if (wide)
        launch_dep(g2p_kernel<true, kG2PPlain, true>, blocks_for(n, pb), pb, 0, st, sc, p0, n, Pin, Pout, gidx, sig_in,
                                                                            sig_out, vgrid, sdf, pcell, next,
                                                                            health, la);
    else {
        constexpr int k = g2p_per_thread(true, kG2PPlain, false);
        launch_dep(g2p_kernel<true, kG2PPlain>, blocks_for(n, (long long)pb * k), pb, k * 3 * pb * sizeof(float4), st,
            sc, p0, n, Pin, Pout, gidx, sig_in, sig_out, vgrid, sdf, pcell, next, health, la);
    }
    return 1;
}

int launch_state_import(const SimParams& p, const float* soa26, float* P, int32_t* sigma, bool init_rules,
                        cudaStream_t st) {
    if (p.n <= 0) return 0;
    state_import_kernel<<<blocks_for(p.n, 256), 256, 0, st>>>(p, soa26, P, sigma, init_rules);
    return 1;
}

int launch_reference_keys(const SimParams& p, const float* P, const int32_t* sigma, int32_t* keys, cudaStream_t st) {
    if (p.n <= 0) return 0;
    reference_keys_kernel<<<blocks_for(p.n, 256), 256, 0, st>>>(p, P, sigma, keys);
    return 1;
}

int launch_state_export(const SimParams& p, const float* P, const int32_t* sigma, float* soa26, cudaStream_t st) {
    if (p.n <= 0) return 0;
    state_export_kernel<<<blocks_for(p.n, 256), 256, 0, st>>>(p, P, sigma, soa26);
    return 1;
}

int launch_positions_export(const SimParams& p, const float* P, const int32_t* sigma, float* xyz, cudaStream_t st) {
    if (p.n <= 0) return 0;
    positions_export_kernel<<<blocks_for(p.n, 256), 256, 0, st>>>(p, P, sigma, xyz);
    return 1;
}

int launch_grid_export(const SimParams& p, const float4* grid, float* planes4, cudaStream_t st) {
    grid_export_kernel<<<blocks_for(p.g, 256), 256, 0, st>>>(p, grid, planes4);
    return 1;
}

int launch_identity(int32_t* dst, int n, cudaStream_t st) {
    if (n <= 0) return 0;
    identity_kernel<<<blocks_for(n, 256), 256, 0, st>>>(dst, n);
    return 1;
}

int launch_learned_decide(const float* stat, long long n, int rule, float threshold,
                          cudaGraphConditionalHandle fallback, long long* counters, float* last, cudaStream_t st) {
    learned_decide_kernel<<<1, 32, 0, st>>>(stat, n, rule, threshold, fallback, counters, last);
    return 1;
}

int launch_copy_words(void* dst, const void* src, long long count, cudaStream_t st) {
    if (count <= 0) return 0;
    const bool vec = count % 4 == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(src) & 15) == 0;
    const long long units = vec ? count / 4 : count;
    const int blocks = (int)std::min<long long>((units + 255) / 256, 148LL * 16);
    copy_words_kernel<<<blocks, 256, 0, st>>>(static_cast<uint32_t*>(dst), static_cast<const uint32_t*>(src), count,
                                               vec);
    return 1;
}

int launch_fill(float* dst, long long count, float value, cudaStream_t st) {
    if (count <= 0) return 0;
    const int blocks = (int)std::min<long long>((count + 255) / 256, 148LL * 16);
    fill_kernel<<<blocks, 256, 0, st>>>(dst, count, value);
    return 1;
}

}  // namespace mpm
