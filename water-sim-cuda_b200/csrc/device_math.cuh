// Device math shared by the substep and SDF kernels.
//
// Each helper states the reference function it restates.  Parameters come
// from a per-engine SimParams passed by value to every kernel instead of the
// reference's process-global `__constant__ SimConfig d_config`
// (common.cuh:65-83, config.cu:3), so several engines can share a device.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mpm {

// Particle state on the device, particle-major: 24 floats (96 bytes, six
// 16-byte vectors) per particle, position and F first so that G2P reads its
// inputs as three vectors.  VOL and MASS are not stored per particle:
// Engine::init's initFMatrices sets every particle to VOL = RESOLUTION^3 and
// MASS = 1 (kernels.cu:349-358) and no kernel writes them again, so they are
// two scalars in SimParams.
enum ParticleField : int {
    kAPos = 0,   // x, y, z
    kAF = 3,     // F00..F22 row-major
    kAVel = 12,  // vx, vy, vz
    kAC = 15,    // C00..C22 row-major
    kAFloats = 24
};

// Particles are binned by their stencil base cell b = stencil_base(pos)
// (the cell whose 3x3x3 node stencil they scatter to).  A particle reaches
// the grid only if b lies in [-2, SIZE-1] on every axis; bins are blocks of
// kBinX x kBinY x kBinZ base cells over that shifted range (u = b + 2).  Bin
// `nb` collects the particles that reach no node.
constexpr int kBinX = 8, kBinY = 4, kBinZ = 4;
constexpr int kBinCells = kBinX * kBinY * kBinZ;  // 128

// One scene.  An engine holds one or more independent scenes whose arrays are
// concatenated: particle slots, grid nodes, cells and bins are numbered
// globally, and poff/goff/coff/boff give where this scene's part begins.
struct SimParams {
    int sx, sy, sz;       // SIZE_X/Y/Z
    int padding;          // PADDING
    float gravity, dt, gamma, compression;
    float pvol, pmass;    // per-particle volume and mass
    int n;                // particles
    int g;                // grid nodes sx*sy*sz
    int nbx, nby, nbz;    // bin blocks per axis: ceil((SIZE+2) / kBin*)
    int nb;               // bin blocks; bin nb holds the particles that reach no node
    long long poff;       // first particle slot
    long long goff;       // first grid node
    long long coff;       // first cell: (nb + 1) * kBinCells cells per scene
    long long boff;       // first bin entry: nb + 2 entries per scene
};

// The scenes of an engine on the device: prm[s], and the prefix arrays
// poff[s] / goff[s] (S + 1 entries each) that map a global particle slot or
// grid node to its scene.
struct SceneTable {
    const SimParams* prm;
    const long long* poff;
    const long long* goff;
    int count;
};

// Largest s with first[s] <= i (first[0] = 0, first is non-decreasing).
__device__ __forceinline__ int scene_of(const long long* __restrict__ first, int count, long long i) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(first + mid) <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Node index z*SX*SY + y*SX + x (getGridIdx, common.cuh:131-134).
__device__ __forceinline__ int node_index(const SimParams& p, int x, int y, int z) {
    return (z * p.sy + y) * p.sx + x;
}

// isInBounds (common.cuh:212-218).
__device__ __forceinline__ bool node_in_grid(const SimParams& p, int x, int y, int z) {
    return (unsigned)x < (unsigned)p.sx && (unsigned)y < (unsigned)p.sy && (unsigned)z < (unsigned)p.sz;
}

// Quadratic B-spline weight (spline, common.cuh:205-210).  The reference
// evaluates `0.75 - x*x` and `(1.5-|x|)^2 * 0.5` with double literals: x*x is
// rounded to float, the rest is exact in double and rounded once on return.
// The same single roundings in float, written with _rn intrinsics so that
// no FMA contraction changes them, give the bit-identical result.  NaN -> 0.
__device__ __forceinline__ float bspline_weight(float x) {
    const float ax = fabsf(x);
    if (ax < 0.5f) return __fsub_rn(0.75f, __fmul_rn(x, x));
    if (ax < 1.5f) {
        const float t = __fsub_rn(1.5f, ax);  // exact for ax in [0.5, 1.5)
        return __fmul_rn(__fmul_rn(t, t), 0.5f);
    }
    return 0.0f;
}

// Stencil base cell: the reference truncates toward zero, not floor
// ((int)(pos - 0.5f), kernels.cu:14, 204).  cvt.rzi saturates; NaN -> 0.
__device__ __forceinline__ int stencil_base(float pos) { return __float2int_rz(__fsub_rn(pos, 0.5f)); }

// Spreads the low bits of v to every third bit with the published
// multiply-and-mask sequence (T. Karras, "Thinking Parallel, Part III",
// 2012), the sequence expandBits uses (common.cuh:277-284).  Inputs >= 1024
// alias exactly as there, which keeps keys bit-exact for particles outside
// a 1024^3 box.
__device__ __forceinline__ uint32_t spread_bits3(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// Morton key of a position (setKeys + calculateMorton, kernels.cu:361-371,
// common.cuh:304-307): coordinates are max(0, p) truncated to unsigned
// (saturating, NaN -> 0), interleaved z:y:x from the high end, and stored
// as a signed int, which is what the reference sorts.
__device__ __forceinline__ int32_t morton_key(float px, float py, float pz) {
    const uint32_t x = __float2uint_rz(fmaxf(0.0f, px));
    const uint32_t y = __float2uint_rz(fmaxf(0.0f, py));
    const uint32_t z = __float2uint_rz(fmaxf(0.0f, pz));
    return (int32_t)((spread_bits3(z) << 2) | (spread_bits3(y) << 1) | spread_bits3(x));
}

// Cell of a particle at (x, y, z): bin * kBinCells + the index of its stencil
// base cell inside the bin (x fastest), and its bin.  A particle none of
// whose 27 stencil nodes is in the grid (isInBounds, common.cuh:212-218)
// goes to the single cell of the overflow bin nb.
__device__ __forceinline__ int cell_of(const SimParams& p, float x, float y, float z, int* bin) {
    const int bx = stencil_base(x), by = stencil_base(y), bz = stencil_base(z);
    if (bx < -2 || by < -2 || bz < -2 || bx > p.sx - 1 || by > p.sy - 1 || bz > p.sz - 1) {
        *bin = p.nb;
        return p.nb * kBinCells;
    }
    const int ux = bx + 2, uy = by + 2, uz = bz + 2;
    const int b = ((uz / kBinZ) * p.nby + uy / kBinY) * p.nbx + ux / kBinX;
    *bin = b;
    return b * kBinCells + ((uz % kBinZ) * kBinY + uy % kBinY) * kBinX + ux % kBinX;
}

__device__ __forceinline__ float det3(const float* A) {
    // det3x3 (common.cuh:250-253), same expansion order.
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
}

// Trilinear SDF sample with clamped node indices (getSDF, common.cuh:136-167).
__device__ __forceinline__ float sdf_trilinear(const SimParams& p, const float* __restrict__ sdf, float qx, float qy,
                                               float qz) {
    const int i = __float2int_rz(floorf(qx)), j = __float2int_rz(floorf(qy)), k = __float2int_rz(floorf(qz));
    const float tx = qx - (float)i, ty = qy - (float)j, tz = qz - (float)k;
    const int x0 = max(0, min(i, p.sx - 1)), x1 = max(0, min(i + 1, p.sx - 1));
    const int y0 = max(0, min(j, p.sy - 1)), y1 = max(0, min(j + 1, p.sy - 1));
    const int z0 = max(0, min(k, p.sz - 1)), z1 = max(0, min(k + 1, p.sz - 1));
    const float n000 = __ldg(sdf + node_index(p, x0, y0, z0)), n100 = __ldg(sdf + node_index(p, x1, y0, z0));
    const float n010 = __ldg(sdf + node_index(p, x0, y1, z0)), n110 = __ldg(sdf + node_index(p, x1, y1, z0));
    const float n001 = __ldg(sdf + node_index(p, x0, y0, z1)), n101 = __ldg(sdf + node_index(p, x1, y0, z1));
    const float n011 = __ldg(sdf + node_index(p, x0, y1, z1)), n111 = __ldg(sdf + node_index(p, x1, y1, z1));
    const float a0 = n000 * (1.0f - tx) + n100 * tx;
    const float a1 = n010 * (1.0f - tx) + n110 * tx;
    const float a2 = n001 * (1.0f - tx) + n101 * tx;
    const float a3 = n011 * (1.0f - tx) + n111 * tx;
    const float b0 = a0 * (1.0f - ty) + a1 * ty;
    const float b1 = a2 * (1.0f - ty) + a3 * ty;
    return b0 * (1.0f - tz) + b1 * tz;
}

// Normalised central difference of the trilinear SDF, eps = 0.1
// (calculateNormal, common.cuh:169-182).
__device__ __forceinline__ float3 sdf_gradient_dir(const SimParams& p, const float* __restrict__ sdf, float qx,
                                                   float qy, float qz) {
    const float eps = 0.1f;
    float nx = sdf_trilinear(p, sdf, qx + eps, qy, qz) - sdf_trilinear(p, sdf, qx - eps, qy, qz);
    float ny = sdf_trilinear(p, sdf, qx, qy + eps, qz) - sdf_trilinear(p, sdf, qx, qy - eps, qz);
    float nz = sdf_trilinear(p, sdf, qx, qy, qz + eps) - sdf_trilinear(p, sdf, qx, qy, qz - eps);
    const float len = sqrtf(nx * nx + ny * ny + nz * nz) + 1e-6f;
    return make_float3(nx / len, ny / len, nz / len);
}

// Normalised central difference of the SDF at a node with clamped
// neighbours (getNormalAtNode, common.cuh:195-203).
__device__ __forceinline__ float3 sdf_node_normal(const SimParams& p, const float* __restrict__ sdf, int x, int y,
                                                  int z) {
    const float nx = __ldg(sdf + node_index(p, min(x + 1, p.sx - 1), y, z)) - __ldg(sdf + node_index(p, max(x - 1, 0), y, z));
    const float ny = __ldg(sdf + node_index(p, x, min(y + 1, p.sy - 1), z)) - __ldg(sdf + node_index(p, x, max(y - 1, 0), z));
    const float nz = __ldg(sdf + node_index(p, x, y, min(z + 1, p.sz - 1))) - __ldg(sdf + node_index(p, x, y, max(z - 1, 0)));
    const float len = sqrtf(nx * nx + ny * ny + nz * nz) + 1e-9f;
    return make_float3(nx / len, ny / len, nz / len);
}

}  // namespace mpm
