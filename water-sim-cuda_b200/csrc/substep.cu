// One MLS-MPM substep on the device: P2G scatter, grid update, G2P gather,
// plus the kernels that move state across the boundary.
//
// Layout (HBM):
//  - particle state: 24 float planes (pos, vel, C, F) of stride ld, kept in
//    the Morton order of the last sort, so every particle kernel streams it;
//  - grid: one float4 per node, (mass, x, y, z).  `accum` receives the P2G
//    sums with 16-byte vector reductions (red.global.add.v4.f32); the grid
//    update turns it into `vgrid` (mass, velocity) and leaves `accum` zero
//    for the next substep, so no separate clear pass is needed;
//  - sdf: one float per node.
#include <algorithm>
#include <climits>

#include "kernels.h"

namespace mpm {
namespace {

constexpr int kP2GThreads = 256;
constexpr int kTileCap = 2048;  // nodes of the per-CTA shared tile (32 KB)

__device__ __forceinline__ void red_add_v4(float4* addr, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

// P2G (p2GTransferScatter, kernels.cu:6-142).  One thread per particle of the
// sorted order.  The CTA's particles are contiguous in Morton order, so the
// in-grid nodes of their 3x3x3 stencils fit a small box; the CTA accumulates
// into that box in shared memory and flushes each touched node once with a
// vector reduction.  A CTA whose box exceeds kTileCap nodes (its particles
// straddle a high-level Morton boundary) reduces straight to global memory.
// Unlike the reference, no tile partial sum is dropped (it drops tile cells
// whose partial mass is <= 1e-9, kernels.cu:132).
__global__ void __launch_bounds__(kP2GThreads) p2g_kernel(SimParams p, const float* __restrict__ P,
                                                          const int32_t* __restrict__ gidx,
                                                          float4* __restrict__ accum) {
    __shared__ float s_m[kTileCap], s_x[kTileCap], s_y[kTileCap], s_z[kTileCap];
    __shared__ int s_part[6][kP2GThreads / 32];
    __shared__ int s_box[6];

    const int i = blockIdx.x * kP2GThreads + threadIdx.x;
    const bool valid = i < p.n;
    float pos[3] = {0.f, 0.f, 0.f}, vel[3] = {0.f, 0.f, 0.f}, C[9], F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) C[k] = F[k] = 0.f;
    if (valid) {
        const float* q = P + __ldg(gidx + i);
#pragma unroll
        for (int k = 0; k < 3; ++k) pos[k] = __ldg(q + (kPX + k) * p.ld);
#pragma unroll
        for (int k = 0; k < 3; ++k) vel[k] = __ldg(q + (kVX + k) * p.ld);
#pragma unroll
        for (int k = 0; k < 9; ++k) C[k] = __ldg(q + (kC0 + k) * p.ld);
#pragma unroll
        for (int k = 0; k < 9; ++k) F[k] = __ldg(q + (kF0 + k) * p.ld);
    }
    const int bx = stencil_base(pos[0]), by = stencil_base(pos[1]), bz = stencil_base(pos[2]);
    // In-grid part of the stencil; 64-bit so saturated bases cannot overflow.
    const int lox = (int)max((long long)bx, 0LL), hix = (int)min((long long)bx + 2, (long long)p.sx - 1);
    const int loy = (int)max((long long)by, 0LL), hiy = (int)min((long long)by + 2, (long long)p.sy - 1);
    const int loz = (int)max((long long)bz, 0LL), hiz = (int)min((long long)bz + 2, (long long)p.sz - 1);
    const bool contributes = valid && lox <= hix && loy <= hiy && loz <= hiz;

    // CTA box of all contributing stencils.
    int box[6] = {contributes ? lox : INT_MAX, contributes ? loy : INT_MAX, contributes ? loz : INT_MAX,
                  contributes ? hix : INT_MIN, contributes ? hiy : INT_MIN, contributes ? hiz : INT_MIN};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 3; ++k) box[k] = __reduce_min_sync(0xffffffffu, box[k]);
#pragma unroll
    for (int k = 3; k < 6; ++k) box[k] = __reduce_max_sync(0xffffffffu, box[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) s_part[k][warp] = box[k];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        int v = s_part[k][0];
        for (int w = 1; w < kP2GThreads / 32; ++w) v = k < 3 ? min(v, s_part[k][w]) : max(v, s_part[k][w]);
        s_box[k] = v;
    }
    __syncthreads();
    const int ox = s_box[0], oy = s_box[1], oz = s_box[2];
    if (ox > s_box[3]) return;  // no particle of this CTA touches the grid (uniform)
    const int dx = s_box[3] - ox + 1, dy = s_box[4] - oy + 1, dz = s_box[5] - oz + 1;
    const long long vol = (long long)dx * dy * dz;
    const bool use_tile = vol <= kTileCap;
    if (use_tile) {
        for (int q = threadIdx.x; q < vol; q += kP2GThreads) s_m[q] = s_x[q] = s_y[q] = s_z[q] = 0.f;
    }
    __syncthreads();

    if (contributes) {
        // Tait pressure from the clamped det F and the APIC + stress affine
        // matrix C' = C + (4 DT V p / m) I (kernels.cu:26-35).
        float J = det3(F);
        J = fmaxf(0.9f, fminf(J, 1.1f));
        float pressure = p.compression * (powf(J, p.gamma) - 1.0f);
        if (pressure < 0.0f) pressure = 0.0f;
        const float volume = p.pvol * J;
        const float multi = 4.0f * p.dt * volume * pressure / p.pmass;
#pragma unroll
        for (int k = 0; k < 9; ++k) C[k] += multi * ((k % 4 == 0) ? 1.0f : 0.0f);

        float wx[3], wy[3], wz[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            wx[a] = bspline_weight(pos[0] - (float)(bx + a));
            wy[a] = bspline_weight(pos[1] - (float)(by + a));
            wz[a] = bspline_weight(pos[2] - (float)(bz + a));
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int z = bz + c;
            if ((unsigned)z >= (unsigned)p.sz) continue;
            const float dzv = -(pos[2] - (float)z);
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const int y = by + b;
                if ((unsigned)y >= (unsigned)p.sy) continue;
                const float dyv = -(pos[1] - (float)y);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const int x = bx + a;
                    if ((unsigned)x >= (unsigned)p.sx) continue;
                    const float dxv = -(pos[0] - (float)x);
                    const float w = wx[a] * wy[b] * wz[c];
                    const float wm = p.pmass * w;
                    const float mx = wm * (vel[0] + (C[0] * dxv + C[1] * dyv + C[2] * dzv));
                    const float my = wm * (vel[1] + (C[3] * dxv + C[4] * dyv + C[5] * dzv));
                    const float mz = wm * (vel[2] + (C[6] * dxv + C[7] * dyv + C[8] * dzv));
                    if (use_tile) {
                        const int l = ((z - oz) * dy + (y - oy)) * dx + (x - ox);
                        atomicAdd(&s_m[l], wm);
                        atomicAdd(&s_x[l], mx);
                        atomicAdd(&s_y[l], my);
                        atomicAdd(&s_z[l], mz);
                    } else {
                        red_add_v4(accum + node_index(p, x, y, z), wm, mx, my, mz);
                    }
                }
            }
        }
    }
    if (!use_tile) return;  // uniform
    __syncthreads();
    for (int q = threadIdx.x; q < vol; q += kP2GThreads) {
        const float m = s_m[q];
        if (m != 0.0f) {
            const int lx = q % dx, ly = (q / dx) % dy, lz = q / (dx * dy);
            red_add_v4(accum + node_index(p, ox + lx, oy + ly, oz + lz), m, s_x[q], s_y[q], s_z[q]);
        }
    }
}

// Grid update (gridUpdate, kernels.cu:144-196): v = p/m, gravity, SDF
// projection where sdf < 0, PADDING walls.  Writes (mass, v) to vgrid and
// zeroes accum for the next P2G.  The wall tests use the reference's
// unsigned arithmetic (SimConfig fields are uint32_t): x < PADDING and
// x > SIZE-1-PADDING with wrap-around.
__global__ void __launch_bounds__(256) grid_update_kernel(SimParams p, float4* __restrict__ accum,
                                                          float4* __restrict__ vgrid,
                                                          const float* __restrict__ sdf) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= p.g) return;
    const float4 a = accum[idx];
    float4 out = make_float4(a.x, 0.f, 0.f, 0.f);
    if (a.x > 1e-9f) {
        const int x = idx % p.sx, y = (idx / p.sx) % p.sy, z = idx / (p.sx * p.sy);
        float vx = a.y / a.x;
        float vy = a.z / a.x - p.gravity * p.dt;
        float vz = a.w / a.x;
        if (__ldg(sdf + idx) < 0.0f) {
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
    vgrid[idx] = out;
    if (a.x != 0.f || a.y != 0.f || a.z != 0.f || a.w != 0.f) accum[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// G2P (g2PTransfer, kernels.cu:199-280).  Thread j reads the particle at
// slot gidx[j] of the old order and writes slot j of the new order, so the
// state ends up in the order of this substep's sort.  The key of the new
// position is written at the particle's original index for the next sort.
__global__ void __launch_bounds__(256) g2p_kernel(SimParams p, const float* __restrict__ Pin,
                                                  float* __restrict__ Pout, const int32_t* __restrict__ gidx,
                                                  const int32_t* __restrict__ sigma,
                                                  const float4* __restrict__ vgrid, const float* __restrict__ sdf,
                                                  int32_t* __restrict__ keys_out, uint32_t* __restrict__ health) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.n) return;
    const float* q = Pin + __ldg(gidx + j);
    float pos[3], F[9];
#pragma unroll
    for (int k = 0; k < 3; ++k) pos[k] = __ldg(q + (kPX + k) * p.ld);
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = __ldg(q + (kF0 + k) * p.ld);

    const int bx = stencil_base(pos[0]), by = stencil_base(pos[1]), bz = stencil_base(pos[2]);
    float wx[3], wy[3], wz[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        wx[a] = bspline_weight(pos[0] - (float)(bx + a));
        wy[a] = bspline_weight(pos[1] - (float)(by + a));
        wz[a] = bspline_weight(pos[2] - (float)(bz + a));
    }
    float tv[3] = {0.f, 0.f, 0.f}, tc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) tc[k] = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int z = bz + c;
        if ((unsigned)z >= (unsigned)p.sz) continue;
        const float dzv = -(pos[2] - (float)z);
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int y = by + b;
            if ((unsigned)y >= (unsigned)p.sy) continue;
            const float dyv = -(pos[1] - (float)y);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int x = bx + a;
                if ((unsigned)x >= (unsigned)p.sx) continue;
                const float dxv = -(pos[0] - (float)x);
                const float4 g = __ldg(vgrid + node_index(p, x, y, z));
                const float w = wx[a] * wy[b] * wz[c];
                tv[0] += w * g.y;
                tv[1] += w * g.z;
                tv[2] += w * g.w;
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
            }
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
    float nx = pos[0] + tv[0] * p.dt, ny = pos[1] + tv[1] * p.dt, nz = pos[2] + tv[2] * p.dt;
    const float dist = sdf_trilinear(p, sdf, nx, ny, nz);
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
    float* o = Pout + j;
    o[kPX * p.ld] = nx;
    o[kPY * p.ld] = ny;
    o[kPZ * p.ld] = nz;
#pragma unroll
    for (int k = 0; k < 3; ++k) o[(kVX + k) * p.ld] = tv[k];
#pragma unroll
    for (int k = 0; k < 9; ++k) o[(kC0 + k) * p.ld] = tc[k];
#pragma unroll
    for (int k = 0; k < 9; ++k) o[(kF0 + k) * p.ld] = NF[k];
    keys_out[__ldg(sigma + j)] = morton_key(nx, ny, nz);

    uint32_t flags = 0;
    if (!(isfinite(nx) && isfinite(ny) && isfinite(nz) && isfinite(tv[0]) && isfinite(tv[1]) && isfinite(tv[2])))
        flags |= 1u;
    if (!(nx >= 0.f && nx < (float)p.sx && ny >= 0.f && ny < (float)p.sy && nz >= 0.f && nz < (float)p.sz))
        flags |= 2u;
    if (flags) atomicOr(health, flags);
}

__global__ void __launch_bounds__(256) state_import_kernel(SimParams p, const float* __restrict__ in,
                                                           float* __restrict__ P, int32_t* __restrict__ sigma,
                                                           int32_t* __restrict__ rank, int32_t* __restrict__ keys,
                                                           bool init_rules) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const long long n = p.n;
#pragma unroll
    for (int k = 0; k < kStatePlanes; ++k) {
        float v = __ldg(in + k * n + i);
        if (init_rules && (k == kF0 || k == kF0 + 4 || k == kF0 + 8)) v = 1.0f;
        P[k * p.ld + i] = v;
    }
    sigma[i] = i;
    rank[i] = i;
    keys[i] = morton_key(__ldg(in + kPX * n + i), __ldg(in + kPY * n + i), __ldg(in + kPZ * n + i));
}

__global__ void __launch_bounds__(256) state_export_kernel(SimParams p, const float* __restrict__ P,
                                                           const int32_t* __restrict__ sigma,
                                                           float* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.n) return;
    const long long n = p.n;
    const int o = __ldg(sigma + j);
#pragma unroll
    for (int k = 0; k < kStatePlanes; ++k) out[k * n + o] = __ldg(P + k * p.ld + j);
    out[24 * n + o] = p.pvol;
    out[25 * n + o] = p.pmass;
}

__global__ void __launch_bounds__(256) positions_export_kernel(SimParams p, const float* __restrict__ P,
                                                               const int32_t* __restrict__ sigma,
                                                               float* __restrict__ xyz) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.n) return;
    const long long o = __ldg(sigma + j);
    xyz[3 * o + 0] = __ldg(P + kPX * p.ld + j);
    xyz[3 * o + 1] = __ldg(P + kPY * p.ld + j);
    xyz[3 * o + 2] = __ldg(P + kPZ * p.ld + j);
}

__global__ void __launch_bounds__(256) grid_export_kernel(SimParams p, const float4* __restrict__ grid,
                                                          float* __restrict__ planes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.g) return;
    const float4 v = __ldg(grid + i);
    const long long g = p.g;
    planes[i] = v.x;
    planes[g + i] = v.y;
    planes[2 * g + i] = v.z;
    planes[3 * g + i] = v.w;
}

__global__ void __launch_bounds__(256) fill_kernel(float* __restrict__ dst, long long count, float value) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = value;
}

inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

int launch_p2g(const SimParams& p, const float* P, const int32_t* gidx, float4* accum, cudaStream_t st) {
    if (p.n <= 0) return 0;
    p2g_kernel<<<blocks_for(p.n, kP2GThreads), kP2GThreads, 0, st>>>(p, P, gidx, accum);
    return 1;
}

int launch_grid_update(const SimParams& p, float4* accum, float4* vgrid, const float* sdf, cudaStream_t st) {
    grid_update_kernel<<<blocks_for(p.g, 256), 256, 0, st>>>(p, accum, vgrid, sdf);
    return 1;
}

int launch_g2p(const SimParams& p, const float* Pin, float* Pout, const int32_t* gidx, const int32_t* sigma,
               const float4* vgrid, const float* sdf, int32_t* keys_out, uint32_t* health, cudaStream_t st) {
    if (p.n <= 0) return 0;
    g2p_kernel<<<blocks_for(p.n, 256), 256, 0, st>>>(p, Pin, Pout, gidx, sigma, vgrid, sdf, keys_out, health);
    return 1;
}

int launch_state_import(const SimParams& p, const float* soa26, float* P, int32_t* sigma, int32_t* rank,
                        int32_t* keys, bool init_rules, cudaStream_t st) {
    if (p.n <= 0) return 0;
    state_import_kernel<<<blocks_for(p.n, 256), 256, 0, st>>>(p, soa26, P, sigma, rank, keys, init_rules);
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

int launch_fill(float* dst, long long count, float value, cudaStream_t st) {
    if (count <= 0) return 0;
    const int blocks = (int)std::min<long long>((count + 255) / 256, 148LL * 16);
    fill_kernel<<<blocks, 256, 0, st>>>(dst, count, value);
    return 1;
}

}  // namespace mpm
