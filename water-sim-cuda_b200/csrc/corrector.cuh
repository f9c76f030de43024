// Learned large-step corrector: a per-particle MLP 16 -> 64 -> 64 -> 3 (GELU)
// that predicts the velocity correction which lets one substep of RATIO x DT
// match RATIO plain substeps.  Inference runs inside the large step's G2P on
// the tensor cores (bf16 operands, fp32 accumulation, mma.m16n8k16); the
// plain substep stays the drop-in path and the fallback.
//
// Inputs (features of a particle, gathered from the large step's grid at the
// particle's start-of-step position x):
//   f[0..8]   C, the APIC affine matrix (row-major)
//   f[9..11]  v, the grid velocity at x
//   f[12]     rho / rho0 - 1: the B-spline-interpolated node mass at x over
//             the seeding density pmass / pvol
//   f[13..15] n(x) * phi(x) * max(0, 1 - |phi(x)| / 4): the obstacle's SDF
//             distance and unit normal folded into one vector, which fades to
//             zero four cells away from the surface
// Outputs: the velocity correction dv (3), added to v before advection.
#pragma once

#include <cuda_bf16.h>

#include "device_math.cuh"

namespace mpm {

constexpr int kMlpIn = 16, kMlpHidden = 64, kMlpOut = 3;

// FP32 parameter vector (host and device master copy).  W* are row-major
// [out][in].  The first 35 floats normalise the inputs and scale the outputs;
// training keeps them fixed.
enum MlpParam : int {
    kPInMean = 0,                              // [16]
    kPInInvStd = kPInMean + kMlpIn,            // [16]
    kPOutStd = kPInInvStd + kMlpIn,            // [3]
    kPW1 = kPOutStd + kMlpOut,                 // [64][16]
    kPB1 = kPW1 + kMlpHidden * kMlpIn,         // [64]
    kPW2 = kPB1 + kMlpHidden,                  // [64][64]
    kPB2 = kPW2 + kMlpHidden * kMlpHidden,     // [64]
    kPW3 = kPB2 + kMlpHidden,                  // [3][64]
    kPB3 = kPW3 + kMlpOut * kMlpHidden,        // [3]
    kPCount = kPB3 + kMlpOut,                  // 5478
    kPTrainFirst = kPW1                        // parameters trained: [kPW1, kPCount)
};

// Inference copy: weights as bf16 mma.m16n8k16 B fragments in lane order (one
// 8-byte load per lane and fragment, conflict-free from shared memory), fp32
// biases and normalisation.  Fragment (n-tile j, k-chunk c) of a layer holds,
// for lane (g = lane / 4, t = lane % 4), W[8j + g][16c + 2t, +1] and
// W[8j + g][16c + 2t + 8, +9].
struct MlpPacked {
    uint2 f1[8 * 1][32];  // layer 1: 8 n-tiles x 1 k-chunk
    uint2 f2[8 * 4][32];  // layer 2: 8 n-tiles x 4 k-chunks, index j * 4 + c
    uint2 f3[1 * 4][32];  // layer 3: outputs padded to one n-tile of 8
    float b1[kMlpHidden];
    float b2[kMlpHidden];
    float b3[8];
    float in_mean[kMlpIn];
    float in_inv_std[kMlpIn];
    float out_std[4];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "MlpPacked is copied in 16-byte vectors");

// Shared-memory row stride (32-bit words) of the per-warp feature stage: 12
// words keep the 8 rows read by one fragment load in distinct banks.
constexpr int kMlpStageStride = 12;

#if defined(__CUDACC__)

__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
__device__ __forceinline__ float gelu_tanh(float x) {
    const float u = 0.7978845608f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.0f + tanh_fast(u));
}
// d/dx of gelu_tanh.
__device__ __forceinline__ float gelu_tanh_grad(float x) {
    const float u = 0.7978845608f * (x + 0.044715f * x * x * x);
    const float t = tanh_fast(u);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608f * (1.0f + 3.0f * 0.044715f * x * x);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// D = A (16x16 bf16, row) * B (16x8 bf16, col) + D, fp32 accumulate.
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// Accumulators of one 16x64 hidden layer (8 n-tiles) -> GELU -> the bf16 A
// fragments of the next layer's 4 k-chunks: the C fragment of n-tiles 2c and
// 2c+1 is, lane for lane, the A fragment of k-chunk c.
__device__ __forceinline__ void gelu_to_afrag(const float (&acc)[8][4], uint32_t (&a)[4][4]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        a[c][0] = pack_bf16x2(gelu_tanh(acc[2 * c][0]), gelu_tanh(acc[2 * c][1]));
        a[c][1] = pack_bf16x2(gelu_tanh(acc[2 * c][2]), gelu_tanh(acc[2 * c][3]));
        a[c][2] = pack_bf16x2(gelu_tanh(acc[2 * c + 1][0]), gelu_tanh(acc[2 * c + 1][1]));
        a[c][3] = pack_bf16x2(gelu_tanh(acc[2 * c + 1][2]), gelu_tanh(acc[2 * c + 1][3]));
    }
}

// The MLP for the 32 particles of a warp: lane l passes its particle's raw
// features x[16] and receives its correction out[3].  `m` is the packed MLP
// (shared memory), `stage` this warp's 32 x kMlpStageStride words of shared
// memory.  Every lane of the warp must call it.
__device__ __forceinline__ void mlp_forward_warp(const MlpPacked& m, uint32_t* stage, const float (&x)[kMlpIn],
                                                 float (&out)[3]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int i = 0; i < kMlpIn / 2; ++i)
        stage[lane * kMlpStageStride + i] =
            pack_bf16x2((x[2 * i] - m.in_mean[2 * i]) * m.in_inv_std[2 * i],
                        (x[2 * i + 1] - m.in_mean[2 * i + 1]) * m.in_inv_std[2 * i + 1]);
    __syncwarp();
    out[0] = out[1] = out[2] = 0.f;
#pragma unroll 1
    for (int mt = 0; mt < 2; ++mt) {
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        const uint32_t a0[4] = {stage[r0 * kMlpStageStride + t], stage[r1 * kMlpStageStride + t],
                                stage[r0 * kMlpStageStride + t + 4], stage[r1 * kMlpStageStride + t + 4]};
        float acc[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float bl = m.b1[8 * j + 2 * t], bh = m.b1[8 * j + 2 * t + 1];
            acc[j][0] = bl, acc[j][1] = bh, acc[j][2] = bl, acc[j][3] = bh;
            mma_bf16_16816(acc[j], a0, m.f1[j][lane]);
        }
        uint32_t a1[4][4];
        gelu_to_afrag(acc, a1);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float bl = m.b2[8 * j + 2 * t], bh = m.b2[8 * j + 2 * t + 1];
            acc[j][0] = bl, acc[j][1] = bh, acc[j][2] = bl, acc[j][3] = bh;
#pragma unroll
            for (int c = 0; c < 4; ++c) mma_bf16_16816(acc[j], a1[c], m.f2[j * 4 + c][lane]);
        }
        uint32_t a2[4][4];
        gelu_to_afrag(acc, a2);
        float y[4];
        {
            const float bl = m.b3[2 * t], bh = m.b3[2 * t + 1];
            y[0] = bl, y[1] = bh, y[2] = bl, y[3] = bh;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) mma_bf16_16816(y, a2[c], m.f3[c][lane]);
        // Row r of this m-tile, output o: lane 4 (r % 8) + o / 2, register
        // (r < 8 ? 0 : 2) + o % 2.
        const int r = lane - mt * 16;
        const int src = 4 * (r & 7);
        const float x0 = __shfl_sync(0xffffffffu, y[0], src), x1 = __shfl_sync(0xffffffffu, y[1], src);
        const float x2 = __shfl_sync(0xffffffffu, y[2], src), x3 = __shfl_sync(0xffffffffu, y[3], src);
        const float z0 = __shfl_sync(0xffffffffu, y[0], src + 1), z2 = __shfl_sync(0xffffffffu, y[2], src + 1);
        if (r >= 0 && r < 16) {
            out[0] = (r < 8 ? x0 : x2) * m.out_std[0];
            out[1] = (r < 8 ? x1 : x3) * m.out_std[1];
            out[2] = (r < 8 ? z0 : z2) * m.out_std[2];
        }
    }
    __syncwarp();
}

#endif  // __CUDACC__

}  // namespace mpm
