// Learned large-step corrector: dataset, training and stand-alone inference.
//
// The dataset holds (features, target) pairs: the 16 features of a particle
// at the start of a large step (corrector.cuh) and the velocity difference
// between RATIO plain substeps and one uncorrected substep of RATIO x DT from
// the same state.  Training minimises the mean squared error of the
// normalised targets with Adam.  The forward pass of training rounds weights
// and activations to bf16 exactly where the tensor-core inference does; the
// backward pass and the master weights are fp32.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "corrector_tc_train.cuh"
#include "kernels.h"

namespace mpm {
namespace {

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ long long sample_index(unsigned long long seed, unsigned long long stream, long long i,
                                                  long long size) {
    const unsigned long long h = splitmix64(splitmix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) + (unsigned long long)i);
    return (long long)(h % (unsigned long long)size);
}

// One thread per fragment word: params (fp32, MlpParam layout) -> MlpPacked.
__global__ void mlp_pack_kernel(const float* __restrict__ w, MlpPacked* __restrict__ m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    auto frag = [&](const float* W, int nout, int nin, int j, int c, int lane) {
        const int g = lane >> 2, t = lane & 3, row = 8 * j + g, k = 16 * c + 2 * t;
        auto at = [&](int kk) { return row < nout ? W[row * nin + kk] : 0.f; };
        uint2 r;
        const __nv_bfloat162 lo = __floats2bfloat162_rn(at(k), at(k + 1));
        const __nv_bfloat162 hi = __floats2bfloat162_rn(at(k + 8), at(k + 9));
        r.x = *reinterpret_cast<const uint32_t*>(&lo);
        r.y = *reinterpret_cast<const uint32_t*>(&hi);
        return r;
    };
    if (i < 8 * 32) {
        m->f1[i >> 5][i & 31] = frag(w + kPW1, kMlpHidden, kMlpIn, i >> 5, 0, i & 31);
    } else if (i < 8 * 32 + 32 * 32) {
        const int q = i - 8 * 32, jc = q >> 5;
        m->f2[jc][q & 31] = frag(w + kPW2, kMlpHidden, kMlpHidden, jc >> 2, jc & 3, q & 31);
    } else if (i < 8 * 32 + 32 * 32 + 4 * 32) {
        const int q = i - 8 * 32 - 32 * 32, c = q >> 5;
        m->f3[c][q & 31] = frag(w + kPW3, kMlpOut, kMlpHidden, 0, c, q & 31);
    } else if (i == 8 * 32 + 32 * 32 + 4 * 32) {
        for (int k = 0; k < kMlpHidden; ++k) m->b1[k] = w[kPB1 + k], m->b2[k] = w[kPB2 + k];
        for (int k = 0; k < 8; ++k) m->b3[k] = k < kMlpOut ? w[kPB3 + k] : 0.f;
        for (int k = 0; k < kMlpIn; ++k) m->in_mean[k] = w[kPInMean + k], m->in_inv_std[k] = w[kPInInvStd + k];
        for (int k = 0; k < 4; ++k) m->out_std[k] = k < kMlpOut ? w[kPOutStd + k] : 0.f;
    }
}

// params (fp32) -> the tcgen05 operand layout: one thread per weight entry.
__global__ void mlp_pack_tc_kernel(const float* __restrict__ w, MlpTc* __restrict__ m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 64 * 16) {
        const int r = i / 16, k = i % 16;
        m->w1[canon_index(r, k, 16)] = __float2bfloat16_rn(w[kPW1 + i]);
    } else if (i < 64 * 16 + 64 * 64) {
        const int q = i - 64 * 16, r = q / 64, k = q % 64;
        m->w2[canon_index(r, k, 64)] = __float2bfloat16_rn(w[kPW2 + q]);
    } else if (i < 64 * 16 + 64 * 64 + 16 * 64) {
        const int q = i - 64 * 16 - 64 * 64, r = q / 64, k = q % 64;
        m->w3[canon_index(r, k, 64)] = __float2bfloat16_rn(r < kMlpOut ? w[kPW3 + r * 64 + k] : 0.f);
    } else if (i == 64 * 16 + 64 * 64 + 16 * 64) {
        for (int k = 0; k < 64; ++k) m->b1[k] = w[kPB1 + k], m->b2[k] = w[kPB2 + k];
        for (int k = 0; k < 4; ++k) m->b3[k] = k < kMlpOut ? w[kPB3 + k] : 0.f;
        for (int k = 0; k < kMlpIn; ++k) m->in_mean[k] = w[kPInMean + k], m->in_inv_std[k] = w[kPInInvStd + k];
        for (int k = 0; k < 4; ++k) m->out_std[k] = k < kMlpOut ? w[kPOutStd + k] : 0.f;
    }
}

// Stand-alone tcgen05 inference: 256 rows per CTA (the routine of the
// learned G2P's tcgen05 mode).
__global__ void __launch_bounds__(kTcThreads) mlp_infer_tc_kernel(const MlpTc* __restrict__ mlp,
                                                                  const float* __restrict__ feat, long long n,
                                                                  float* __restrict__ out, uint32_t* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    MlpTcSmem& s = *reinterpret_cast<MlpTcSmem*>(smem_raw);
    const uint4* src = reinterpret_cast<const uint4*>(mlp);
    uint4* dst = reinterpret_cast<uint4*>(&s.w);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpTc) / 16); i += blockDim.x) dst[i] = __ldg(src + i);
    mlp_tc_begin(s);
    const long long jj = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long j = jj < n ? jj : n - 1;
    float x[kMlpIn], y[3];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) x[k] = __ldg(feat + j * kMlpIn + k);
    mlp_forward_tc(s, x, y);
    mlp_tc_end(s);
    if (s.failed) {
        if (threadIdx.x == 0) atomicOr(status, kStatusTimeout);
        return;
    }
    if (jj < n)
        for (int o = 0; o < 3; ++o) out[j * 3 + o] = y[o];
}

// Stand-alone tensor-core inference (the same warp routine as the learned G2P).
__global__ void __launch_bounds__(256) mlp_infer_kernel(const MlpPacked* __restrict__ mlp,
                                                        const float* __restrict__ feat, long long n,
                                                        float* __restrict__ out) {
    __shared__ __align__(16) unsigned char s_mlp_raw[sizeof(MlpPacked)];
    __shared__ uint32_t s_stage[8 * 32 * kMlpStageStride];
    const uint4* src = reinterpret_cast<const uint4*>(mlp);
    uint4* dst = reinterpret_cast<uint4*>(s_mlp_raw);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
    const long long jj = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long j = jj < n ? jj : n - 1;
    float x[kMlpIn], y[3];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) x[k] = __ldg(feat + j * kMlpIn + k);
    mlp_forward_warp(*reinterpret_cast<const MlpPacked*>(s_mlp_raw), s_stage + (threadIdx.x >> 5) * 32 * kMlpStageStride,
                     x, y);
    if (jj < n)
        for (int o = 0; o < 3; ++o) out[j * 3 + o] = y[o];
}

// out[orig * 3 + c] = velocity of slot j (sigma[j] = orig).
__global__ void velocity_export_kernel(const float* __restrict__ P, const int32_t* __restrict__ sigma, long long n,
                                       float* __restrict__ out) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const long long o = sigma[j];
    const float* q = P + j * kAFloats + kAVel;
    out[o * 3 + 0] = q[0], out[o * 3 + 1] = q[1], out[o * 3 + 2] = q[2];
}

// Appends `samples` particles drawn with replacement: features and the
// target vplain - vlarge.
__global__ void dataset_append_kernel(const float* __restrict__ feat_all, const float* __restrict__ vplain,
                                      const float* __restrict__ vlarge, long long n, long long samples,
                                      unsigned long long seed, float* __restrict__ feat, float* __restrict__ targ) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= samples) return;
    const long long r = sample_index(seed, 0x5A17ull, i, n);
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) feat[i * kMlpIn + k] = feat_all[r * kMlpIn + k];
#pragma unroll
    for (int c = 0; c < 3; ++c) targ[i * 3 + c] = vplain[r * 3 + c] - vlarge[r * 3 + c];
}

// Sums and sums of squares of the 16 features and 3 targets (fp64).
__global__ void moments_kernel(const float* __restrict__ feat, const float* __restrict__ targ, long long size,
                               double* __restrict__ acc /* [2][19] */) {
    double s[kMlpIn + kMlpOut], q[kMlpIn + kMlpOut];
    for (int k = 0; k < kMlpIn + kMlpOut; ++k) s[k] = q[k] = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < size;
         i += (long long)gridDim.x * blockDim.x) {
        for (int k = 0; k < kMlpIn; ++k) {
            const double v = feat[i * kMlpIn + k];
            s[k] += v, q[k] += v * v;
        }
        for (int k = 0; k < kMlpOut; ++k) {
            const double v = targ[i * kMlpOut + k];
            s[kMlpIn + k] += v, q[kMlpIn + k] += v * v;
        }
    }
    for (int k = 0; k < kMlpIn + kMlpOut; ++k) {
        double a = s[k], b = q[k];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(acc + k, a);
            atomicAdd(acc + kMlpIn + kMlpOut + k, b);
        }
    }
}

// ------------------------------------------------------------- training ----
// One CTA of 256 threads takes tiles of kTile samples.  Shared memory: the
// bf16-rounded weights, the tile's normalised inputs and targets, and the
// pre-activations / activations of both hidden layers (rows of kRow floats,
// an odd stride so that 32 samples of one column fall in 32 banks).  Thread
// (s = tid % 64, ug = tid / 64) computes units 16 ug .. 16 ug + 15 of sample
// s; the weight gradients stay in registers across the CTA's tiles (thread
// (u = tid / 4, q = tid % 4) owns dW2[u][q + 4m], dW1[u][q + 4m]) and are
// added to the global gradient once per CTA.
constexpr int kTile = 64;
constexpr int kRow = kMlpHidden + 1;
constexpr int kXRow = kMlpIn + 1;
constexpr int kTrainThreads = 256;
constexpr int kSmW1 = 0;
constexpr int kSmB1 = kSmW1 + kMlpHidden * kMlpIn;
constexpr int kSmW2 = kSmB1 + kMlpHidden;
constexpr int kSmB2 = kSmW2 + kMlpHidden * kMlpHidden;
constexpr int kSmW3 = kSmB2 + kMlpHidden;
constexpr int kSmB3 = kSmW3 + kMlpOut * kMlpHidden;
constexpr int kSmX = kSmB3 + 4;
constexpr int kSmT = kSmX + kTile * kXRow;
constexpr int kSmDY = kSmT + kTile * kMlpOut;
constexpr int kSmZ1 = kSmDY + kTile * kMlpOut;
constexpr int kSmH1 = kSmZ1 + kTile * kRow;
constexpr int kSmZ2 = kSmH1 + kTile * kRow;
constexpr int kSmH2 = kSmZ2 + kTile * kRow;
constexpr int kSmIdx = kSmH2 + kTile * kRow;
constexpr int kSmFloats = kSmIdx + 2 * kTile;  // sample indices as long long
constexpr size_t kTrainSmem = (size_t)kSmFloats * sizeof(float);

__global__ void __launch_bounds__(kTrainThreads) mlp_train_kernel(
    const float* __restrict__ w, const float* __restrict__ feat, const float* __restrict__ targ, long long size,
    const long long* __restrict__ idx_list, int batch, unsigned long long seed, int step, float* __restrict__ grad,
    float* __restrict__ loss) {
    extern __shared__ __align__(16) float sm[];
    float* W1 = sm + kSmW1;
    float* B1 = sm + kSmB1;
    float* W2 = sm + kSmW2;
    float* B2 = sm + kSmB2;
    float* W3 = sm + kSmW3;
    float* B3 = sm + kSmB3;
    float* X = sm + kSmX;
    float* T = sm + kSmT;
    float* DY = sm + kSmDY;
    float* Z1 = sm + kSmZ1;
    float* H1 = sm + kSmH1;
    float* Z2 = sm + kSmZ2;
    float* H2 = sm + kSmH2;
    long long* sidx = reinterpret_cast<long long*>(sm + kSmIdx);
    const int tid = threadIdx.x;
    for (int i = tid; i < kMlpHidden * kMlpIn; i += kTrainThreads) W1[i] = bf16_round(w[kPW1 + i]);
    for (int i = tid; i < kMlpHidden * kMlpHidden; i += kTrainThreads) W2[i] = bf16_round(w[kPW2 + i]);
    for (int i = tid; i < kMlpOut * kMlpHidden; i += kTrainThreads) W3[i] = bf16_round(w[kPW3 + i]);
    if (tid < kMlpHidden) B1[tid] = w[kPB1 + tid], B2[tid] = w[kPB2 + tid];
    if (tid < kMlpOut) B3[tid] = w[kPB3 + tid];

    const float inv_count = 1.0f / ((float)batch * kMlpOut);
    float gW2[16], gW1[4], gW3 = 0.f, gB3 = 0.f, gB2 = 0.f, gB1 = 0.f, lsum = 0.f;
#pragma unroll
    for (int m = 0; m < 16; ++m) gW2[m] = 0.f;
#pragma unroll
    for (int m = 0; m < 4; ++m) gW1[m] = 0.f;
    const int s = tid & (kTile - 1), ug = tid >> 6;  // sample, unit group
    const int u4 = tid >> 2, q4 = tid & 3;            // gradient ownership
    const int ntiles = batch / kTile;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();  // weights staged / previous tile done
        if (tid < kTile) {
            const long long i = (long long)tile * kTile + tid;
            sidx[tid] = idx_list ? idx_list[i] : sample_index(seed, 0x7A11ull + (unsigned long long)step, i, size);
        }
        __syncthreads();
        for (int e = tid; e < kTile * kMlpIn; e += kTrainThreads) {
            const int r = e >> 4, k = e & 15;
            X[r * kXRow + k] = bf16_round((feat[sidx[r] * kMlpIn + k] - w[kPInMean + k]) * w[kPInInvStd + k]);
        }
        for (int e = tid; e < kTile * kMlpOut; e += kTrainThreads) {
            const int r = e / kMlpOut, o = e % kMlpOut;
            T[r * kMlpOut + o] = targ[sidx[r] * kMlpOut + o] / w[kPOutStd + o];
        }
        __syncthreads();
        // Layer 1.
        {
            float xr[kMlpIn];
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) xr[k] = X[s * kXRow + k];
#pragma unroll 4
            for (int uu = 0; uu < 16; ++uu) {
                const int u = ug * 16 + uu;
                float z = B1[u];
#pragma unroll
                for (int k = 0; k < kMlpIn; ++k) z += W1[u * kMlpIn + k] * xr[k];
                Z1[s * kRow + u] = z;
                H1[s * kRow + u] = bf16_round(gelu_tanh(z));
            }
        }
        __syncthreads();
        // Layer 2.
        {
            float acc[16];
#pragma unroll
            for (int uu = 0; uu < 16; ++uu) acc[uu] = B2[ug * 16 + uu];
            for (int k0 = 0; k0 < kMlpHidden; k0 += 16) {
                float hr[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) hr[k] = H1[s * kRow + k0 + k];
#pragma unroll
                for (int uu = 0; uu < 16; ++uu) {
                    const float4* wr = reinterpret_cast<const float4*>(W2 + (ug * 16 + uu) * kMlpHidden + k0);
#pragma unroll
                    for (int k4 = 0; k4 < 4; ++k4) {
                        const float4 wv = wr[k4];
                        acc[uu] += wv.x * hr[4 * k4] + wv.y * hr[4 * k4 + 1] + wv.z * hr[4 * k4 + 2] + wv.w * hr[4 * k4 + 3];
                    }
                }
            }
#pragma unroll
            for (int uu = 0; uu < 16; ++uu) {
                Z2[s * kRow + ug * 16 + uu] = acc[uu];
                H2[s * kRow + ug * 16 + uu] = bf16_round(gelu_tanh(acc[uu]));
            }
        }
        __syncthreads();
        // Output layer and loss gradient.
        if (tid < kTile * kMlpOut) {
            const int o = tid >> 6, r = tid & (kTile - 1);
            float y = B3[o];
            for (int k = 0; k < kMlpHidden; ++k) y += W3[o * kMlpHidden + k] * H2[r * kRow + k];
            const float d = y - T[r * kMlpOut + o];
            lsum += d * d;
            DY[r * kMlpOut + o] = 2.0f * d * inv_count;
        }
        __syncthreads();
        // dW3, db3; dZ2 = (W3^T dY) * gelu'(Z2), in place of Z2.
        if (tid < kTile * kMlpOut) {
            const int o = tid >> 6, k = tid & (kTile - 1);
            for (int r = 0; r < kTile; ++r) gW3 += DY[r * kMlpOut + o] * H2[r * kRow + k];
        } else if (tid < kTile * kMlpOut + kMlpOut) {
            const int o = tid - kTile * kMlpOut;
            for (int r = 0; r < kTile; ++r) gB3 += DY[r * kMlpOut + o];
        }
        {
            const float d0 = DY[s * kMlpOut], d1 = DY[s * kMlpOut + 1], d2 = DY[s * kMlpOut + 2];
#pragma unroll 4
            for (int uu = 0; uu < 16; ++uu) {
                const int u = ug * 16 + uu;
                const float dh = d0 * W3[u] + d1 * W3[kMlpHidden + u] + d2 * W3[2 * kMlpHidden + u];
                Z2[s * kRow + u] = dh * gelu_tanh_grad(Z2[s * kRow + u]);
            }
        }
        __syncthreads();
        // dW2, db2; dZ1 = (W2^T dZ2) * gelu'(Z1), in place of Z1.
        for (int r = 0; r < kTile; ++r) {
            const float d = Z2[r * kRow + u4];
#pragma unroll
            for (int m = 0; m < 16; ++m) gW2[m] += d * H1[r * kRow + q4 + 4 * m];
            if (q4 == 0) gB2 += d;
        }
        {
            float acc[16];
#pragma unroll
            for (int kk = 0; kk < 16; ++kk) acc[kk] = 0.f;
            for (int u = 0; u < kMlpHidden; ++u) {
                const float d = Z2[s * kRow + u];
                const float4* wr = reinterpret_cast<const float4*>(W2 + u * kMlpHidden + ug * 16);
#pragma unroll
                for (int k4 = 0; k4 < 4; ++k4) {
                    const float4 wv = wr[k4];
                    acc[4 * k4] += d * wv.x, acc[4 * k4 + 1] += d * wv.y;
                    acc[4 * k4 + 2] += d * wv.z, acc[4 * k4 + 3] += d * wv.w;
                }
            }
#pragma unroll
            for (int kk = 0; kk < 16; ++kk) {
                const int k = ug * 16 + kk;
                Z1[s * kRow + k] = acc[kk] * gelu_tanh_grad(Z1[s * kRow + k]);
            }
        }
        __syncthreads();
        // dW1, db1.
        for (int r = 0; r < kTile; ++r) {
            const float d = Z1[r * kRow + u4];
#pragma unroll
            for (int m = 0; m < 4; ++m) gW1[m] += d * X[r * kXRow + q4 + 4 * m];
            if (q4 == 0) gB1 += d;
        }
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) atomicAdd(grad + kPW2 + u4 * kMlpHidden + q4 + 4 * m, gW2[m]);
#pragma unroll
    for (int m = 0; m < 4; ++m) atomicAdd(grad + kPW1 + u4 * kMlpIn + q4 + 4 * m, gW1[m]);
    if (q4 == 0) {
        atomicAdd(grad + kPB2 + u4, gB2);
        atomicAdd(grad + kPB1 + u4, gB1);
    }
    if (tid < kTile * kMlpOut) atomicAdd(grad + kPW3 + (tid >> 6) * kMlpHidden + (tid & (kTile - 1)), gW3);
    else if (tid < kTile * kMlpOut + kMlpOut) atomicAdd(grad + kPB3 + tid - kTile * kMlpOut, gB3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((tid & 31) == 0) atomicAdd(loss, lsum * inv_count);
}

// Adam on the trained parameters; zeroes the gradient.
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ grad, float* __restrict__ m1,
                            float* __restrict__ m2, float lr, float beta1, float beta2, float eps, float bc1,
                            float bc2) {
    const int i = kPTrainFirst + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kPCount) return;
    const float g = grad[i];
    grad[i] = 0.f;
    const float a = beta1 * m1[i] + (1.0f - beta1) * g;
    const float b = beta2 * m2[i] + (1.0f - beta2) * g * g;
    m1[i] = a;
    m2[i] = b;
    w[i] -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
}

// The training gradient on tcgen05 (corrector_tc_train.cuh): the loss and
// batch of mlp_train_kernel, tiles of 128 samples, rows at or beyond `batch`
// masked by dY = 0.  A bounded wait that gives up sets kStatusTimeout in
// *status and the CTA adds nothing to the gradient.
__global__ void __launch_bounds__(kTrThreads, 1) mlp_train_tc_kernel(
    const float* __restrict__ w, const float* __restrict__ feat, const float* __restrict__ targ, long long size,
    const long long* __restrict__ idx_list, int batch, unsigned long long seed, int step, float* __restrict__ grad,
    float* __restrict__ loss, uint32_t* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    MlpTrainSmem& s = *reinterpret_cast<MlpTrainSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, wq = (tid >> 5) & 3, ch = 32 * (tid >> 7);
    const int srow = 32 * wq + lane;  // this thread's sample row in the epilogues
    // Weights, their transposed copies, and the zero padding of dY and dZ^T.
    for (int i = tid; i < 64 * 16; i += kTrThreads)
        s.w.w1[canon_index(i / 16, i % 16, 16)] = __float2bfloat16_rn(w[kPW1 + i]);
    for (int i = tid; i < 64 * 64; i += kTrThreads) {
        const int u = i / 64, k = i % 64;
        const __nv_bfloat16 v = __float2bfloat16_rn(w[kPW2 + i]);
        s.w.w2[canon_index(u, k, 64)] = v;
        s.w.w2t[canon_index(k, u, 64)] = v;
    }
    for (int i = tid; i < 16 * 64; i += kTrThreads) {
        const int o = i / 64, k = i % 64;
        const __nv_bfloat16 v = __float2bfloat16_rn(o < kMlpOut ? w[kPW3 + o * 64 + k] : 0.f);
        s.w.w3[canon_index(o, k, 64)] = v;
        s.w.w3t[canon_index(k, o, 16)] = v;
    }
    if (tid < 64) s.w.b1[tid] = w[kPB1 + tid], s.w.b2[tid] = w[kPB2 + tid];
    if (tid < 4) s.w.b3[tid] = tid < kMlpOut ? w[kPB3 + tid] : 0.f;
    for (int i = tid; i < (int)(sizeof(s.dy) / 16); i += kTrThreads) reinterpret_cast<uint4*>(s.dy)[i] = uint4{0, 0, 0, 0};
    for (int i = tid; i < (int)(sizeof(s.dzt) / 16); i += kTrThreads)
        reinterpret_cast<uint4*>(s.dzt)[i] = uint4{0, 0, 0, 0};
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"(kTrTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&s.mbar, 1);
        s.failed = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = s.tmem;
    const uint32_t trow = tm + ((uint32_t)(32 * wq) << 16);  // this warp's TMEM lanes
    const float inv_count = 1.0f / ((float)batch * kMlpOut);
    float gW3 = 0.f, gB3 = 0.f, gB2 = 0.f, gB1 = 0.f, lsum = 0.f;
    uint32_t phase = 0;
    bool any = false;
    const int ntiles = (batch + kTrTile - 1) / kTrTile;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        if (tid < kTrTile) {
            const long long i = (long long)tile * kTrTile + tid;
            long long j = 0;
            if (i < batch) j = idx_list ? idx_list[i] : sample_index(seed, 0x7A11ull + (unsigned long long)step, i, size);
            s.sidx[tid] = j;
        }
        __syncthreads();
        for (int e = tid; e < kTrTile * kMlpIn; e += kTrThreads) {
            const int r = e >> 4, k = e & 15;
            const __nv_bfloat16 v =
                __float2bfloat16_rn((feat[s.sidx[r] * kMlpIn + k] - w[kPInMean + k]) * w[kPInInvStd + k]);
            s.x[canon_index(r, k, 16)] = v;
            s.xt[canon_index(k, r, kTrTile)] = v;
        }
        for (int e = tid; e < kTrTile * kMlpOut; e += kTrThreads) {
            const int r = e / kMlpOut, o = e % kMlpOut;
            s.dyf[r * 4 + o] = targ[s.sidx[r] * kMlpOut + o] / w[kPOutStd + o];
        }
        // Z1 = X W1^T.
        mlp_tr_publish();
        if (tid == 0) {
            mlp_tr_mma(tm + kTrColZ1, s.x, s.w.w1, 64, 16, false);
            umma_commit(&s.mbar);
        }
        if (!mlp_tr_wait(s, phase)) break;
        float g1[32], g2[32];
        {
            float v[32];
            tmem_ld32(trow + kTrColZ1 + (uint32_t)ch, v);
#pragma unroll
            for (int j = 0; j < 32; j += 2) {
                const int u = ch + j;
                const float z0 = v[j] + s.w.b1[u], z1 = v[j + 1] + s.w.b1[u + 1];
                g1[j] = gelu_tanh_grad(z0);
                g1[j + 1] = gelu_tanh_grad(z1);
                const __nv_bfloat162 h = __floats2bfloat162_rn(gelu_tanh(z0), gelu_tanh(z1));
                *reinterpret_cast<__nv_bfloat162*>(s.h1 + canon_index(srow, u, 64)) = h;
                s.h1t[canon_index(u, srow, kTrTile)] = h.x;
                s.h1t[canon_index(u + 1, srow, kTrTile)] = h.y;
            }
        }
        // Z2 = H1 W2^T.
        mlp_tr_publish();
        if (tid == 0) {
            mlp_tr_mma(tm + kTrColZ2, s.h1, s.w.w2, 64, 64, false);
            umma_commit(&s.mbar);
        }
        if (!mlp_tr_wait(s, phase)) break;
        {
            float v[32];
            tmem_ld32(trow + kTrColZ2 + (uint32_t)ch, v);
#pragma unroll
            for (int j = 0; j < 32; j += 2) {
                const int u = ch + j;
                const float z0 = v[j] + s.w.b2[u], z1 = v[j + 1] + s.w.b2[u + 1];
                g2[j] = gelu_tanh_grad(z0);
                g2[j + 1] = gelu_tanh_grad(z1);
                *reinterpret_cast<__nv_bfloat162*>(s.h2 + canon_index(srow, u, 64)) =
                    __floats2bfloat162_rn(gelu_tanh(z0), gelu_tanh(z1));
            }
        }
        // Y = H2 W3^T; the loss and dY.
        mlp_tr_publish();
        if (tid == 0) {
            mlp_tr_mma(tm + kTrColY, s.h2, s.w.w3, 16, 64, false);
            umma_commit(&s.mbar);
        }
        if (!mlp_tr_wait(s, phase)) break;
        if (ch == 0) {
            float v[16];
            tmem_ld16(trow + kTrColY, v);
            const bool valid = (long long)tile * kTrTile + srow < batch;
#pragma unroll
            for (int o = 0; o < kMlpOut; ++o) {
                const float d = v[o] + s.w.b3[o] - s.dyf[srow * 4 + o];
                const float dy = valid ? 2.0f * d * inv_count : 0.f;
                if (valid) lsum += d * d;
                s.dyf[srow * 4 + o] = dy;
                s.dy[canon_index(srow, o, 16)] = __float2bfloat16_rn(dy);
            }
        }
        // dH2 = dY W3 on the tensor cores while the CUDA cores sum the
        // output layer's gradients.
        mlp_tr_publish();
        if (tid == 0) {
            mlp_tr_mma(tm + kTrColZ1, s.dy, s.w.w3t, 64, 16, false);
            umma_commit(&s.mbar);
        }
        if (tid < kMlpOut * 64) {
            const int o = tid >> 6, k = tid & 63;
            float acc = 0.f;
            for (int r = 0; r < kTrTile; ++r) acc += s.dyf[r * 4 + o] * __bfloat162float(s.h2[canon_index(r, k, 64)]);
            gW3 += acc;
        } else if (tid < kMlpOut * 64 + kMlpOut) {
            const int o = tid - kMlpOut * 64;
            float acc = 0.f;
            for (int r = 0; r < kTrTile; ++r) acc += s.dyf[r * 4 + o];
            gB3 += acc;
        }
        if (!mlp_tr_wait(s, phase)) break;
        {
            float v[32];
            tmem_ld32(trow + kTrColZ1 + (uint32_t)ch, v);
#pragma unroll
            for (int j = 0; j < 32; j += 2) {
                const int u = ch + j;
                v[j] *= g2[j];
                v[j + 1] *= g2[j + 1];
                const __nv_bfloat162 d = __floats2bfloat162_rn(v[j], v[j + 1]);
                *reinterpret_cast<__nv_bfloat162*>(s.dz + canon_index(srow, u, 64)) = d;
                s.dzt[canon_index(u, srow, kTrTile)] = d.x;
                s.dzt[canon_index(u + 1, srow, kTrTile)] = d.y;
            }
            gB2 += warp_column_sums(v);
        }
        // dH1 = dZ2 W2 and dW2 += dZ2^T H1.
        mlp_tr_publish();
        if (tid == 0) {
            mlp_tr_mma(tm + kTrColZ2, s.dz, s.w.w2t, 64, 64, false);
            mlp_tr_mma(tm + kTrColDW2, s.dzt, s.h1t, 64, kTrTile, any);
            umma_commit(&s.mbar);
        }
        if (!mlp_tr_wait(s, phase)) break;
        {
            float v[32];
            tmem_ld32(trow + kTrColZ2 + (uint32_t)ch, v);
#pragma unroll
            for (int j = 0; j < 32; j += 2) {
                const int u = ch + j;
                v[j] *= g1[j];
                v[j + 1] *= g1[j + 1];
                const __nv_bfloat162 d = __floats2bfloat162_rn(v[j], v[j + 1]);
                s.dzt[canon_index(u, srow, kTrTile)] = d.x;
                s.dzt[canon_index(u + 1, srow, kTrTile)] = d.y;
            }
            gB1 += warp_column_sums(v);
        }
        // dW1 += dZ1^T X.
        mlp_tr_publish();
        if (tid == 0) {
            mlp_tr_mma(tm + kTrColDW1, s.dzt, s.xt, 16, kTrTile, any);
            umma_commit(&s.mbar);
        }
        if (!mlp_tr_wait(s, phase)) break;
        any = true;
    }
    if (s.failed) {
        if (tid == 0) atomicOr(status, kStatusTimeout);
    } else if (any) {
        if (wq < 2) {  // TMEM lanes 0..63: the hidden units
            const int u = srow;
            float v[32];
            tmem_ld32(trow + kTrColDW2 + (uint32_t)ch, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) atomicAdd(grad + kPW2 + u * 64 + ch + j, v[j]);
            if (ch == 0) {
                float v16[16];
                tmem_ld16(trow + kTrColDW1, v16);
#pragma unroll
                for (int i = 0; i < kMlpIn; ++i) atomicAdd(grad + kPW1 + u * kMlpIn + i, v16[i]);
            }
        }
        atomicAdd(grad + kPB2 + ch + lane, gB2);
        atomicAdd(grad + kPB1 + ch + lane, gB1);
        if (tid < kMlpOut * 64) atomicAdd(grad + kPW3 + tid, gW3);
        else if (tid < kMlpOut * 64 + kMlpOut) atomicAdd(grad + kPB3 + tid - kMlpOut * 64, gB3);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0 && ch == 0) atomicAdd(loss, lsum * inv_count);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(kTrTmemCols) : "memory");
}

inline int blocks_of(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

int launch_mlp_pack(const float* params, MlpPacked* out, cudaStream_t st) {
    mlp_pack_kernel<<<blocks_of(8 * 32 + 32 * 32 + 4 * 32 + 1, 256), 256, 0, st>>>(params, out);
    return 1;
}

int launch_mlp_pack_tc(const float* params, MlpTc* out, cudaStream_t st) {
    mlp_pack_tc_kernel<<<blocks_of(64 * 16 + 64 * 64 + 16 * 64 + 1, 256), 256, 0, st>>>(params, out);
    return 1;
}

int launch_mlp_infer_tc(const MlpTc* mlp, const float* feat, long long n, float* out, uint32_t* status,
                        cudaStream_t st) {
    if (n <= 0) return 0;
    mlp_infer_tc_kernel<<<blocks_of(n, kTcThreads), kTcThreads, sizeof(MlpTcSmem), st>>>(mlp, feat, n, out, status);
    return 1;
}

int launch_mlp_infer(const MlpPacked* mlp, const float* feat, long long n, float* out, cudaStream_t st) {
    if (n <= 0) return 0;
    mlp_infer_kernel<<<blocks_of(n, 256), 256, 0, st>>>(mlp, feat, n, out);
    return 1;
}

int launch_velocity_export(const float* P, const int32_t* sigma, long long n, float* out, cudaStream_t st) {
    if (n <= 0) return 0;
    velocity_export_kernel<<<blocks_of(n, 256), 256, 0, st>>>(P, sigma, n, out);
    return 1;
}

}  // namespace mpm

// ------------------------------------------------------------- C ABI ----
struct mpm_corrector {
    int device = 0;
    cudaStream_t stream = nullptr;
    long long capacity = 0;
    long long size = 0;
    float* feat = nullptr;   // [capacity][16]
    float* targ = nullptr;   // [capacity][3]
    float* w = nullptr;      // [kPCount] master parameters
    float* grad = nullptr;   // [kPCount]
    float* m1 = nullptr;     // Adam moments
    float* m2 = nullptr;
    float* loss = nullptr;   // [1]
    double* mom = nullptr;   // [2][19]
    long long* idx = nullptr;  // explicit batch indices (gradient checks)
    long long idx_cap = 0;
    mpm::MlpPacked* packed = nullptr;
    mpm::MlpTc* packed_tc = nullptr;
    uint32_t* status = nullptr;
    float* io = nullptr;     // stand-alone inference staging
    long long io_cap = 0;
    int adam_t = 0;
    int train_kind = MPM_TRAIN_TCGEN05;
    std::string last_error;
};

namespace {

mpm_status cfail(mpm_corrector* c, cudaError_t err, const char* what) {
    cudaGetLastError();
    const std::string msg = std::string("CUDA error in ") + what + ": " + cudaGetErrorName(err) + " (" +
                            cudaGetErrorString(err) + ")";
    if (c) c->last_error = msg;
    else mpm::set_global_error(msg);
    return err == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA;
}

#define CC(c, call)                                                 \
    do {                                                            \
        cudaError_t err_ = (call);                                  \
        if (err_ != cudaSuccess) return cfail((c), err_, #call);    \
    } while (0)

mpm_status cbad(mpm_corrector* c, const char* msg) {
    if (c) c->last_error = msg;
    else mpm::set_global_error(msg);
    return MPM_ERR_INVALID_ARGUMENT;
}

mpm_status center(mpm_corrector* c) {
    if (!c) return cbad(nullptr, "corrector is NULL");
    c->last_error.clear();
    CC(c, cudaSetDevice(c->device));
    return MPM_OK;
}

mpm_status ensure_io(mpm_corrector* c, long long floats) {
    if (c->io_cap >= floats) return MPM_OK;
    if (c->io) cudaFree(c->io);
    c->io = nullptr;
    c->io_cap = 0;
    CC(c, cudaMalloc(&c->io, (size_t)floats * sizeof(float)));
    c->io_cap = floats;
    return MPM_OK;
}

}  // namespace

namespace mpm {

// Appends `samples` pairs drawn from the engine-side buffers (features and
// velocities by original index of an n-particle scene).  Stream-ordered on st.
mpm_status corrector_append(mpm_corrector* c, const float* feat_all, const float* vplain, const float* vlarge,
                            long long n, long long samples, unsigned long long seed, cudaStream_t st) {
    if (samples <= 0 || n <= 0) return MPM_OK;
    if (c->size + samples > c->capacity) return cbad(c, "dataset capacity exceeded");
    dataset_append_kernel<<<blocks_of(samples, 256), 256, 0, st>>>(feat_all, vplain, vlarge, n, samples, seed,
                                                                     c->feat + c->size * kMlpIn,
                                                                     c->targ + c->size * kMlpOut);
    CC(c, cudaGetLastError());
    c->size += samples;
    return MPM_OK;
}

}  // namespace mpm

extern "C" {

mpm_status mpm_corrector_create(int32_t device, int64_t capacity, mpm_corrector** out) {
    if (!out) return cbad(nullptr, "out is NULL");
    *out = nullptr;
    if (capacity < 0) return cbad(nullptr, "capacity < 0");
    auto* c = new mpm_corrector();
    c->device = device;
    c->capacity = capacity;
    auto fail = [&](mpm_status s) {
        mpm::set_global_error(c->last_error);
        mpm_corrector_destroy(c);
        return s;
    };
    cudaError_t err = cudaSetDevice(device);
    if (err != cudaSuccess) return fail(cfail(c, err, "cudaSetDevice"));
#define CA(call)                                           \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return fail(cfail(c, e_, #call)); \
    } while (0)
    CA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const size_t cap = (size_t)std::max<long long>(capacity, 1);
    CA(cudaMalloc(&c->feat, cap * mpm::kMlpIn * sizeof(float)));
    CA(cudaMalloc(&c->targ, cap * mpm::kMlpOut * sizeof(float)));
    CA(cudaMalloc(&c->w, mpm::kPCount * sizeof(float)));
    CA(cudaMalloc(&c->grad, mpm::kPCount * sizeof(float)));
    CA(cudaMalloc(&c->m1, mpm::kPCount * sizeof(float)));
    CA(cudaMalloc(&c->m2, mpm::kPCount * sizeof(float)));
    CA(cudaMalloc(&c->loss, sizeof(float)));
    CA(cudaMalloc(&c->mom, 2 * (mpm::kMlpIn + mpm::kMlpOut) * sizeof(double)));
    CA(cudaMalloc(&c->packed, sizeof(mpm::MlpPacked)));
    CA(cudaMalloc(&c->packed_tc, sizeof(mpm::MlpTc)));
    CA(cudaMalloc(&c->status, sizeof(uint32_t)));
    CA(cudaMemsetAsync(c->status, 0, sizeof(uint32_t), c->stream));
    CA(cudaMemsetAsync(c->w, 0, mpm::kPCount * sizeof(float), c->stream));
    CA(cudaMemsetAsync(c->grad, 0, mpm::kPCount * sizeof(float), c->stream));
    CA(cudaMemsetAsync(c->m1, 0, mpm::kPCount * sizeof(float), c->stream));
    CA(cudaMemsetAsync(c->m2, 0, mpm::kPCount * sizeof(float), c->stream));
    CA(cudaFuncSetAttribute(mpm::mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)mpm::kTrainSmem));
    CA(cudaFuncSetAttribute(mpm::mlp_train_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sizeof(mpm::MlpTrainSmem)));
    CA(cudaStreamSynchronize(c->stream));
#undef CA
    *out = c;
    return MPM_OK;
}

void mpm_corrector_destroy(mpm_corrector* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void* p : {(void*)c->feat, (void*)c->targ, (void*)c->w, (void*)c->grad, (void*)c->m1, (void*)c->m2,
                    (void*)c->loss, (void*)c->mom, (void*)c->idx, (void*)c->packed, (void*)c->io,
                    (void*)c->packed_tc, (void*)c->status})
        if (p) cudaFree(p);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* mpm_corrector_last_error(const mpm_corrector* c) { return c ? c->last_error.c_str() : ""; }

int64_t mpm_corrector_size(const mpm_corrector* c) { return c ? c->size : -1; }

mpm_status mpm_corrector_clear(mpm_corrector* c) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    c->size = 0;
    return MPM_OK;
}

mpm_status mpm_corrector_add_data(mpm_corrector* c, int64_t count, const float* features_host,
                                  const float* targets_host) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (count < 0 || (count > 0 && (!features_host || !targets_host))) return cbad(c, "bad data arguments");
    if (c->size + count > c->capacity) return cbad(c, "dataset capacity exceeded");
    CC(c, cudaMemcpyAsync(c->feat + c->size * mpm::kMlpIn, features_host, (size_t)count * mpm::kMlpIn * sizeof(float),
                          cudaMemcpyHostToDevice, c->stream));
    CC(c, cudaMemcpyAsync(c->targ + c->size * mpm::kMlpOut, targets_host,
                          (size_t)count * mpm::kMlpOut * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    c->size += count;
    return MPM_OK;
}

mpm_status mpm_corrector_get_data(mpm_corrector* c, int64_t first, int64_t count, float* features_host,
                                  float* targets_host) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (first < 0 || count < 0 || first + count > c->size) return cbad(c, "range outside the dataset");
    if (features_host)
        CC(c, cudaMemcpyAsync(features_host, c->feat + first * mpm::kMlpIn, (size_t)count * mpm::kMlpIn * sizeof(float),
                              cudaMemcpyDeviceToHost, c->stream));
    if (targets_host)
        CC(c, cudaMemcpyAsync(targets_host, c->targ + first * mpm::kMlpOut,
                              (size_t)count * mpm::kMlpOut * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    return MPM_OK;
}

mpm_status mpm_corrector_init(mpm_corrector* c, uint64_t seed) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (c->size < 2) return cbad(c, "the dataset needs at least two samples");
    const int nm = mpm::kMlpIn + mpm::kMlpOut;
    CC(c, cudaMemsetAsync(c->mom, 0, 2 * nm * sizeof(double), c->stream));
    const int grid = (int)std::min<long long>(mpm::blocks_of(c->size, 256), 148 * 4);
    mpm::moments_kernel<<<grid, 256, 0, c->stream>>>(c->feat, c->targ, c->size, c->mom);
    CC(c, cudaGetLastError());
    std::vector<double> mom(2 * nm);
    CC(c, cudaMemcpyAsync(mom.data(), c->mom, mom.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    std::vector<float> w(mpm::kPCount, 0.f);
    for (int k = 0; k < nm; ++k) {
        const double mean = mom[k] / c->size;
        const double var = std::max(0.0, mom[nm + k] / c->size - mean * mean);
        const double sd = std::max(std::sqrt(var), 1e-6);
        if (k < mpm::kMlpIn) {
            w[mpm::kPInMean + k] = (float)mean;
            w[mpm::kPInInvStd + k] = (float)(1.0 / sd);
        } else {
            w[mpm::kPOutStd + k - mpm::kMlpIn] = (float)std::sqrt(var + mean * mean + 1e-12);
        }
    }
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    auto init = [&](int off, int nout, int nin, float gain) {
        const float sd = gain / std::sqrt((float)nin);
        for (int i = 0; i < nout * nin; ++i) w[off + i] = sd * nd(rng);
    };
    init(mpm::kPW1, mpm::kMlpHidden, mpm::kMlpIn, 1.0f);
    init(mpm::kPW2, mpm::kMlpHidden, mpm::kMlpHidden, 1.0f);
    init(mpm::kPW3, mpm::kMlpOut, mpm::kMlpHidden, 0.1f);
    CC(c, cudaMemcpyAsync(c->w, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CC(c, cudaMemsetAsync(c->grad, 0, mpm::kPCount * sizeof(float), c->stream));
    CC(c, cudaMemsetAsync(c->m1, 0, mpm::kPCount * sizeof(float), c->stream));
    CC(c, cudaMemsetAsync(c->m2, 0, mpm::kPCount * sizeof(float), c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    c->adam_t = 0;
    return MPM_OK;
}

mpm_status mpm_corrector_get_params(mpm_corrector* c, float* params_host) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (!params_host) return cbad(c, "params_host is NULL");
    CC(c, cudaMemcpyAsync(params_host, c->w, mpm::kPCount * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    return MPM_OK;
}

mpm_status mpm_corrector_set_params(mpm_corrector* c, const float* params_host) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (!params_host) return cbad(c, "params_host is NULL");
    CC(c, cudaMemcpyAsync(c->w, params_host, mpm::kPCount * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CC(c, cudaMemsetAsync(c->m1, 0, mpm::kPCount * sizeof(float), c->stream));
    CC(c, cudaMemsetAsync(c->m2, 0, mpm::kPCount * sizeof(float), c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    c->adam_t = 0;
    return MPM_OK;
}

namespace {
mpm_status launch_train(mpm_corrector* c, int batch, const long long* idx, unsigned long long seed, int step) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    if (c->train_kind == MPM_TRAIN_TCGEN05) {
        const int tiles = (batch + mpm::kTrTile - 1) / mpm::kTrTile;
        const int grid = std::max(1, std::min(tiles, sms));
        mpm::mlp_train_tc_kernel<<<grid, mpm::kTrThreads, sizeof(mpm::MlpTrainSmem), c->stream>>>(
            c->w, c->feat, c->targ, c->size, idx, batch, seed, step, c->grad, c->loss, c->status);
        CC(c, cudaGetLastError());
        return MPM_OK;
    }
    const int tiles = batch / mpm::kTile;
    int per_sm = 0;
    CC(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mpm::mlp_train_kernel, mpm::kTrainThreads,
                                                         mpm::kTrainSmem));
    const int grid = std::max(1, std::min(tiles, sms * std::max(per_sm, 1)));
    mpm::mlp_train_kernel<<<grid, mpm::kTrainThreads, mpm::kTrainSmem, c->stream>>>(
        c->w, c->feat, c->targ, c->size, idx, batch, seed, step, c->grad, c->loss);
    CC(c, cudaGetLastError());
    return MPM_OK;
}

// The status word the tcgen05 kernels set when a bounded wait gave up (read
// back by the caller together with its results).
mpm_status check_status(mpm_corrector* c, uint32_t flag) {
    if (!flag) return MPM_OK;
    c->last_error = "a bounded wait of a tcgen05 kernel gave up";
    return MPM_ERR_TIMEOUT;
}
}  // namespace

mpm_status mpm_corrector_train(mpm_corrector* c, int32_t steps, int32_t batch, float lr, uint64_t seed,
                               float* mean_loss) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (steps < 0 || batch <= 0 || batch % mpm::kTile != 0) return cbad(c, "batch must be a positive multiple of 64");
    if (c->size < 1) return cbad(c, "the dataset is empty");
    if (!(lr > 0.f)) return cbad(c, "lr must be positive");
    CC(c, cudaMemsetAsync(c->loss, 0, sizeof(float), c->stream));
    CC(c, cudaMemsetAsync(c->status, 0, sizeof(uint32_t), c->stream));
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    const int ntrain = mpm::kPCount - mpm::kPTrainFirst;
    for (int i = 0; i < steps; ++i) {
        st = launch_train(c, batch, nullptr, seed, c->adam_t);
        if (st != MPM_OK) return st;
        ++c->adam_t;
        const float bc1 = 1.0f - (float)std::pow((double)beta1, c->adam_t);
        const float bc2 = 1.0f - (float)std::pow((double)beta2, c->adam_t);
        mpm::adam_kernel<<<mpm::blocks_of(ntrain, 256), 256, 0, c->stream>>>(c->w, c->grad, c->m1, c->m2, lr, beta1,
                                                                         beta2, eps, bc1, bc2);
        CC(c, cudaGetLastError());
    }
    float loss = 0.f;
    uint32_t flag = 0;
    CC(c, cudaMemcpyAsync(&loss, c->loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CC(c, cudaMemcpyAsync(&flag, c->status, sizeof(flag), cudaMemcpyDeviceToHost, c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    if (mean_loss) *mean_loss = steps > 0 ? loss / (float)steps : 0.f;
    return check_status(c, flag);
}

mpm_status mpm_corrector_gradient(mpm_corrector* c, int64_t count, const int64_t* idx_host, float* grad_host,
                                  float* loss_host) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (count <= 0 || count % mpm::kTile != 0 || !idx_host) return cbad(c, "count must be a positive multiple of 64");
    for (int64_t i = 0; i < count; ++i)
        if (idx_host[i] < 0 || idx_host[i] >= c->size) return cbad(c, "sample index outside the dataset");
    if (c->idx_cap < count) {
        if (c->idx) cudaFree(c->idx);
        c->idx = nullptr;
        c->idx_cap = 0;
        CC(c, cudaMalloc(&c->idx, (size_t)count * sizeof(long long)));
        c->idx_cap = count;
    }
    CC(c, cudaMemcpyAsync(c->idx, idx_host, (size_t)count * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    CC(c, cudaMemsetAsync(c->grad, 0, mpm::kPCount * sizeof(float), c->stream));
    CC(c, cudaMemsetAsync(c->loss, 0, sizeof(float), c->stream));
    CC(c, cudaMemsetAsync(c->status, 0, sizeof(uint32_t), c->stream));
    st = launch_train(c, (int)count, c->idx, 0, 0);
    if (st != MPM_OK) return st;
    if (grad_host)
        CC(c, cudaMemcpyAsync(grad_host, c->grad, mpm::kPCount * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    if (loss_host) CC(c, cudaMemcpyAsync(loss_host, c->loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    uint32_t flag = 0;
    CC(c, cudaMemcpyAsync(&flag, c->status, sizeof(flag), cudaMemcpyDeviceToHost, c->stream));
    CC(c, cudaMemsetAsync(c->grad, 0, mpm::kPCount * sizeof(float), c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    return check_status(c, flag);
}

mpm_status mpm_corrector_set_train_kernel(mpm_corrector* c, int32_t kind) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (kind != MPM_TRAIN_TCGEN05 && kind != MPM_TRAIN_FP32) return cbad(c, "unknown training kernel");
    c->train_kind = kind;
    return MPM_OK;
}

mpm_status mpm_corrector_forward_tc(mpm_corrector* c, int64_t n, const float* features_host, float* out_host) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (n < 0 || (n > 0 && (!features_host || !out_host))) return cbad(c, "bad forward arguments");
    if (n == 0) return MPM_OK;
    st = ensure_io(c, n * (mpm::kMlpIn + mpm::kMlpOut));
    if (st != MPM_OK) return st;
    float* d_in = c->io;
    float* d_out = c->io + n * mpm::kMlpIn;
    mpm::launch_mlp_pack_tc(c->w, c->packed_tc, c->stream);
    CC(c, cudaGetLastError());
    CC(c, cudaMemcpyAsync(d_in, features_host, (size_t)n * mpm::kMlpIn * sizeof(float), cudaMemcpyHostToDevice,
                          c->stream));
    CC(c, cudaMemsetAsync(c->status, 0, sizeof(uint32_t), c->stream));
    mpm::launch_mlp_infer_tc(c->packed_tc, d_in, n, d_out, c->status, c->stream);
    CC(c, cudaGetLastError());
    CC(c, cudaMemcpyAsync(out_host, d_out, (size_t)n * mpm::kMlpOut * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
    uint32_t flag = 0;
    CC(c, cudaMemcpyAsync(&flag, c->status, sizeof(flag), cudaMemcpyDeviceToHost, c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    if (flag) {
        c->last_error = "a bounded wait of the tcgen05 MLP gave up";
        return MPM_ERR_TIMEOUT;
    }
    return MPM_OK;
}

mpm_status mpm_corrector_forward(mpm_corrector* c, int64_t n, const float* features_host, float* out_host) {
    mpm_status st = center(c);
    if (st != MPM_OK) return st;
    if (n < 0 || (n > 0 && (!features_host || !out_host))) return cbad(c, "bad forward arguments");
    if (n == 0) return MPM_OK;
    st = ensure_io(c, n * (mpm::kMlpIn + mpm::kMlpOut));
    if (st != MPM_OK) return st;
    float* d_in = c->io;
    float* d_out = c->io + n * mpm::kMlpIn;
    mpm::launch_mlp_pack(c->w, c->packed, c->stream);
    CC(c, cudaGetLastError());
    CC(c, cudaMemcpyAsync(d_in, features_host, (size_t)n * mpm::kMlpIn * sizeof(float), cudaMemcpyHostToDevice,
                          c->stream));
    mpm::launch_mlp_infer(c->packed, d_in, n, d_out, c->stream);
    CC(c, cudaGetLastError());
    CC(c, cudaMemcpyAsync(out_host, d_out, (size_t)n * mpm::kMlpOut * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
    CC(c, cudaStreamSynchronize(c->stream));
    return MPM_OK;
}

}  // extern "C"
