// Training step of the corrector MLP on the 5th-generation tensor cores.
//
// A persistent CTA of 256 threads takes tiles of 128 samples.  Per tile,
// every GEMM is a tcgen05.mma with bf16 operands in shared memory in the
// canonical K-major layout of corrector_tc.cuh and fp32 accumulators in TMEM:
//
//   forward   Z1 = X W1^T,  Z2 = H1 W2^T,  Y = H2 W3^T   (M = 128 samples)
//   backward  dH2 = dY W3,  dH1 = dZ2 W2                (M = 128 samples)
//   weights   dW2 += dZ2^T H1,  dW1 += dZ1^T X          (M = 64 units padded to
//                                                      128, K = 128 samples)
//
// The weight-gradient GEMMs read transposed copies of dZ, H1 and X written
// beside the row-major ones, so that every operand is K-major.  dW2 and dW1
// accumulate in TMEM across the CTA's tiles and reach the global gradient
// once.  The output layer's gradients (3 x 64 + 3) and the hidden biases'
// gradients are summed on the CUDA cores; the latter with a warp butterfly
// reduce-scatter of the fp32 dZ rows.  Inputs, weights and activations are
// rounded to bf16 where the inference rounds them; dY and dZ are rounded to
// bf16 as MMA operands; every sum is fp32.
//
// Epilogue ownership: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its 32
// samples, or units for the weight gradients) and the column half w / 4 of a
// 64-column accumulator.
#pragma once

#include "corrector_tc.cuh"

namespace mpm {

// Weights of a training step in the canonical layout, staged by each CTA
// from the fp32 master parameters.
struct MlpTrainW {
    __nv_bfloat16 w1[64 * 16];   // [u][i]   Z1 = X W1^T
    __nv_bfloat16 w2[64 * 64];   // [u][k]   Z2 = H1 W2^T
    __nv_bfloat16 w3[16 * 64];   // [o][k]   Y = H2 W3^T (rows 3..15 zero)
    __nv_bfloat16 w2t[64 * 64];  // [k][u]   dH1 = dZ2 W2
    __nv_bfloat16 w3t[64 * 16];  // [k][o]   dH2 = dY W3 (columns 3..15 zero)
    float b1[64];
    float b2[64];
    float b3[4];
};

constexpr int kTrTile = 128;
constexpr int kTrThreads = 256;
// TMEM columns: Z1, then dH2 [0, 64); Z2, then dH1 [64, 128); Y [128, 144);
// dW2 [256, 320); dW1 [320, 336).
constexpr int kTrTmemCols = 512;
constexpr uint32_t kTrColZ1 = 0, kTrColZ2 = 64, kTrColY = 128, kTrColDW2 = 256, kTrColDW1 = 320;

struct MlpTrainSmem {
    MlpTrainW w;
    __nv_bfloat16 x[kTrTile * 16];     // [s][i]
    __nv_bfloat16 xt[16 * kTrTile];    // [i][s]
    __nv_bfloat16 h1[kTrTile * 64];    // [s][k]
    __nv_bfloat16 h1t[64 * kTrTile];   // [k][s]
    __nv_bfloat16 h2[kTrTile * 64];    // [s][k]
    __nv_bfloat16 dy[kTrTile * 16];    // [s][o], columns 3..15 zero
    __nv_bfloat16 dz[kTrTile * 64];    // dZ2 [s][u]
    __nv_bfloat16 dzt[128 * kTrTile];  // dZ2^T, then dZ1^T: [u][s], rows 64..127 zero
    float dyf[kTrTile * 4];            // targets, then dY (fp32)
    long long sidx[kTrTile];
    unsigned long long mbar;
    uint32_t tmem;
    uint32_t failed;
};

#if defined(__CUDACC__)

// Thread 0 issues D (+)= A B^T over K in steps of 16 (A: 128 x K, B: N x K,
// both canonical K-major).
__device__ __forceinline__ void mlp_tr_mma(uint32_t d, const __nv_bfloat16* a, const __nv_bfloat16* b, int n, int k,
                                           bool accumulate) {
    const uint32_t idesc = umma_idesc(n);
    const uint32_t sbo = (uint32_t)(k / 8) * 128u;
    for (int kk = 0; kk < k; kk += 16) {
        const uint64_t ad = umma_desc(a + (kk / 8) * 64, 128u, sbo);
        const uint64_t bd = umma_desc(b + (kk / 8) * 64, 128u, sbo);
        umma_f16(d, ad, bd, idesc, (kk > 0 || accumulate) ? 1u : 0u);
    }
}

// Makes this thread's shared-memory writes visible to the tensor cores and
// orders its earlier tcgen05.ld before the MMAs issued after the barrier.
__device__ __forceinline__ void mlp_tr_publish() {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// Waits for the commit of phase `phase` (bounded; a wait that gives up
// drains the committed MMAs first).  A give-up is recorded and turned into a
// CTA-wide outcome.
__device__ __forceinline__ bool mlp_tr_wait(MlpTrainSmem& s, uint32_t& phase) {
    if (!mma_wait_checked(&s.mbar, phase, 0u)) atomicOr(&s.failed, 1u);
    phase ^= 1u;
    __syncthreads();
    tc_fence_after();
    return s.failed == 0u;
}

// Butterfly reduce-scatter over the warp: lane l returns the sum of v[l] over
// the 32 lanes (five exchange steps, each halving the values kept).
__device__ __forceinline__ float warp_column_sums(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
        const bool up = (lane & m) != 0;
#pragma unroll
        for (int i = 0; i < m; ++i) {
            const float keep = up ? v[i + m] : v[i];
            const float send = up ? v[i] : v[i + m];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
    }
    return v[0];
}

// 32 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    float a[16], b[16];
    tmem_ld16(taddr, a);
    tmem_ld16(taddr + 16u, b);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = a[i], v[16 + i] = b[i];
}

#endif  // __CUDACC__

}  // namespace mpm
