// The corrector MLP on the 5th-generation tensor cores: tcgen05.mma with
// bf16 operands in shared memory and fp32 accumulators in tensor memory.
//
// A CTA of 256 threads evaluates the MLP for its 256 particles (thread t =
// row t): rows 0..127 form M-tile 0 and rows 128..255 M-tile 1.  Per layer:
// every thread writes its row of the layer input (bf16) into shared memory in
// the canonical no-swizzle K-major layout, one thread issues the MMAs of both
// tiles (D[128 x N] in TMEM columns tile * 64 ..) and commits them to an
// mbarrier, and after the barrier every warp reads its 32 rows back with
// tcgen05.ld (warp w owns TMEM lanes 32 (w % 4) .. + 31, columns of tile w / 4),
// adds the bias and applies GELU.  The output layer has N = 16 (3 used).
//
// Canonical K-major layout without swizzle: 8 x 16-byte core matrices; the
// element (r, k) of an R x K bf16 matrix sits at byte
// ((r / 8) * (K / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2, so core
// matrices adjacent in K are 128 bytes apart (leading byte offset) and 8-row
// groups K / 8 * 128 bytes apart (stride byte offset).
#pragma once

#include <cuda_bf16.h>

#include "corrector.cuh"

namespace mpm {

// Weights in the canonical layout, fp32 biases and normalisation.
struct MlpTc {
    __nv_bfloat16 w1[64 * 16];  // N = 64 rows x K = 16
    __nv_bfloat16 w2[64 * 64];  // 64 x 64
    __nv_bfloat16 w3[16 * 64];  // 16 x 64, rows 3..15 zero
    float b1[64];
    float b2[64];
    float b3[4];
    float in_mean[16];
    float in_inv_std[16];
    float out_std[4];
};
static_assert(sizeof(MlpTc) % 16 == 0, "MlpTc is copied in 16-byte vectors");

// Shared memory of one CTA: weights, the layer input of 256 rows (K up to
// 64), the mbarrier and the TMEM base address.
struct MlpTcSmem {
    MlpTc w;
    __nv_bfloat16 a[256 * 64];  // layer input, two M-tiles of 128 x K
    unsigned long long mbar;
    uint32_t tmem;
    uint32_t failed;
    uint32_t wait_test;  // test hooks for the first layer's wait (kWaitTest*)
};
constexpr int kTcThreads = 256;
constexpr int kTcTmemCols = 128;  // two tiles x 64 fp32 columns

__host__ __device__ __forceinline__ int canon_index(int r, int k, int K) {
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

#if defined(__CUDACC__)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm_100): start, leading and stride byte
// offsets in 16-byte units, version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(const void* base, uint32_t lbo, uint32_t sbo) {
    const uint64_t a = (smem_u32(base) & 0x3FFFFu) >> 4;
    return a | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           (1ull << 46);
}

// Instruction descriptor, kind::f16: fp32 accumulate, bf16 A and B, both
// K-major, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(void* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(void* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ unsigned long long tc_globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Limits of the bounded MMA waits: a commit normally lands within
// microseconds; the test hook's expiring wait (below) gives up after 20 ms.
constexpr unsigned long long kMmaWaitNs = 1000000000ull;
constexpr unsigned long long kTestWaitNs = 20000000ull;

// Test hooks of the bounded waits (mpm_set_wait_test), acted on only after
// the real completion has been observed, so that no MMA or copy is in flight
// when the caller gives up: kWaitTestGiveUp reports a give-up at once;
// kWaitTestExpire waits for the barrier's next phase, which nothing
// completes, until the short limit really runs out.
enum : uint32_t { kWaitTestGiveUp = 1u, kWaitTestExpire = 2u };

// Waits for phase `parity` of the mbarrier for at most limit_ns; false if
// it gave up.
__device__ __forceinline__ bool mbar_wait(void* mbar, uint32_t parity, unsigned long long limit_ns = kMmaWaitNs) {
    const uint32_t addr = smem_u32(mbar);
    unsigned long long t0 = 0;
    for (int i = 0;; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (i == 0) t0 = tc_globaltimer_ns();
        else if (tc_globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// Waits for the commit of phase `parity`.  If the wait gives up, waits once
// more (bounded) so that the committed MMAs have finished before the caller
// frees its TMEM columns, and returns false.  wait_test: the test hooks above.
__device__ __forceinline__ bool mma_wait_checked(void* mbar, uint32_t parity, uint32_t wait_test) {
    if (!mbar_wait(mbar, parity)) {
        mbar_wait(mbar, parity);  // drain
        return false;
    }
    if (wait_test & kWaitTestGiveUp) return false;
    if (wait_test & kWaitTestExpire) return mbar_wait(mbar, parity ^ 1u, kTestWaitNs);
    return true;
}

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Allocates kTcTmemCols TMEM columns (warp 0) and initialises the mbarrier;
// every thread of the CTA calls it.  wait_test: test hooks (kWaitTest*) for
// the first layer's wait.
__device__ __forceinline__ void mlp_tc_begin(MlpTcSmem& s, uint32_t wait_test = 0u) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(&s.mbar, 1);
        s.failed = 0u;
        s.wait_test = wait_test;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// Frees the TMEM columns (warp 0) once every thread is past its last
// tcgen05.ld; every thread of the CTA calls it.
__device__ __forceinline__ void mlp_tc_end(MlpTcSmem& s) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(kTcTmemCols)
                     : "memory");
}

// One layer: thread 0 issues D[tile] = A[tile] * B^T for both tiles (K / 16
// MMAs each) and commits; everyone waits for `parity`.  Returns false if the
// wait gave up (the caller stops using TMEM; the MMAs have been drained).
// `first`: the layer to which the test hooks apply.
__device__ __forceinline__ bool mlp_tc_layer(MlpTcSmem& s, const __nv_bfloat16* b, int n, int k, uint32_t parity,
                                             bool first = false) {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc_fence_after();
        const uint32_t idesc = umma_idesc(n);
        const uint32_t sbo_a = (uint32_t)(k / 8) * 128u, sbo_b = (uint32_t)(k / 8) * 128u;
#pragma unroll 1
        for (int tile = 0; tile < 2; ++tile) {
            const __nv_bfloat16* a = s.a + tile * 128 * k;
            for (int kk = 0; kk < k; kk += 16) {
                // Each K-step of 16 covers two core matrices along K.
                const uint64_t ad = umma_desc(a + (kk / 8) * 64, 128u, sbo_a);
                const uint64_t bd = umma_desc(b + (kk / 8) * 64, 128u, sbo_b);
                umma_f16(s.tmem + (uint32_t)(tile * 64), ad, bd, idesc, kk > 0 ? 1u : 0u);
            }
        }
        umma_commit(&s.mbar);
    }
    // A wait that gives up is recorded and turned into a CTA-wide decision,
    // so every thread takes the same path through the barriers that follow.
    if (!mma_wait_checked(&s.mbar, parity, first ? s.wait_test : 0u)) atomicOr(&s.failed, 1u);
    __syncthreads();
    tc_fence_after();
    return s.failed == 0u;
}

// This thread's TMEM lane and the column base of its tile.
__device__ __forceinline__ uint32_t mlp_tc_taddr(const MlpTcSmem& s) {
    const int w = threadIdx.x >> 5;
    return s.tmem + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)((w >> 2) * 64);
}

// Row `row` (= threadIdx.x) of the hidden activations: bias, GELU, bf16, into
// the next layer's input (K = 64).
__device__ __forceinline__ void mlp_tc_hidden(MlpTcSmem& s, const float* bias) {
    const int row = threadIdx.x, tile = row >> 7, r = row & 127;
    __nv_bfloat16* a = s.a + tile * 128 * 64;
    const uint32_t taddr = mlp_tc_taddr(s);
#pragma unroll
    for (int c0 = 0; c0 < 64; c0 += 16) {
        float v[16];
        tmem_ld16(taddr + (uint32_t)c0, v);
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
            const float g0 = gelu_tanh(v[i] + bias[c0 + i]), g1 = gelu_tanh(v[i + 1] + bias[c0 + i + 1]);
            *reinterpret_cast<__nv_bfloat162*>(a + canon_index(r, c0 + i, 64)) = __floats2bfloat162_rn(g0, g1);
        }
    }
}

// The MLP for the CTA's 256 rows: thread t passes row t's raw features and
// receives its 3 outputs (zero if a wait gave up; s.failed is then set).
// Every thread of the CTA must call it, between mlp_tc_begin and mlp_tc_end.
__device__ __forceinline__ void mlp_forward_tc(MlpTcSmem& s, const float (&x)[kMlpIn], float (&out)[3]) {
    const int row = threadIdx.x, tile = row >> 7, r = row & 127;
    out[0] = out[1] = out[2] = 0.f;
    {
        __nv_bfloat16* a = s.a + tile * 128 * 16;
#pragma unroll
        for (int i = 0; i < kMlpIn; i += 2) {
            const float u0 = (x[i] - s.w.in_mean[i]) * s.w.in_inv_std[i];
            const float u1 = (x[i + 1] - s.w.in_mean[i + 1]) * s.w.in_inv_std[i + 1];
            *reinterpret_cast<__nv_bfloat162*>(a + canon_index(r, i, 16)) = __floats2bfloat162_rn(u0, u1);
        }
    }
    if (!mlp_tc_layer(s, s.w.w1, 64, 16, 0, true)) return;
    mlp_tc_hidden(s, s.w.b1);
    if (!mlp_tc_layer(s, s.w.w2, 64, 64, 1)) return;
    mlp_tc_hidden(s, s.w.b2);
    if (!mlp_tc_layer(s, s.w.w3, 16, 64, 0)) return;
    float v[16];
    tmem_ld16(mlp_tc_taddr(s), v);
#pragma unroll
    for (int o = 0; o < 3; ++o) out[o] = (v[o] + s.w.b3[o]) * s.w.out_std[o];
}

#endif  // __CUDACC__

}  // namespace mpm
