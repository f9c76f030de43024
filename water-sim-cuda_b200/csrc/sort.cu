// Morton keys and the stable radix sort of the substep.
//
// The reference builds int keys with setKeys (kernels.cu:361-371) and sorts
// (key, 0..n-1) pairs with thrust::sort_by_key (engine.cu:98-99), a stable
// ascending sort on signed keys.  This file restates that contract with a
// least-significant-digit radix sort written for this engine: 8-bit digits,
// four passes, each pass a per-CTA histogram, a per-digit scan of the CTA
// counts, and a scatter that ranks each 2048-key tile in shared memory with
// warp match/ballot and writes runs of equal digits contiguously.  The first
// pass generates the values (input position) instead of reading them; the
// last pass writes only the permutation (and, for the engine, the inverse
// permutation and the gather index of the reordered state).
#include <algorithm>

#include "kernels.h"

namespace mpm {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 8;                   // keys per thread per tile
constexpr int kTile = kThreads * kItems;    // 2048 keys
constexpr int kRadix = 256;
constexpr int kPasses = 4;
constexpr int kMaxCtas = 4 * 148;           // four CTAs per SM of a B200

__device__ __forceinline__ uint32_t digit_of(int32_t key, int shift) {
    // Flipping the sign bit orders signed keys as unsigned.
    return ((static_cast<uint32_t>(key) ^ 0x80000000u) >> shift) & 0xFFu;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Inclusive block scan over 256 threads; *total gets the block sum.
__device__ __forceinline__ uint32_t block_scan_incl(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWarps) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t prefix = warp > 0 ? s_warp[warp - 1] : 0u;
    *total = s_warp[kWarps - 1];
    __syncthreads();
    return x + prefix;
}

__global__ void __launch_bounds__(256) morton_keys_kernel(const float* __restrict__ px, const float* __restrict__ py,
                                                          const float* __restrict__ pz, int n,
                                                          int32_t* __restrict__ keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = morton_key(__ldg(px + i), __ldg(py + i), __ldg(pz + i));
}

// Per-CTA digit histogram: hist[d * nb + cta].
__global__ void __launch_bounds__(kThreads) radix_hist_kernel(const int32_t* __restrict__ keys, int n, int per_cta,
                                                              int nb, int shift, uint32_t* __restrict__ hist) {
    __shared__ uint32_t s_hist[kWarps][kRadix];
    for (int t = threadIdx.x; t < kWarps * kRadix; t += kThreads) (&s_hist[0][0])[t] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int begin = blockIdx.x * per_cta;
    const int end = min(begin + per_cta, n);
    for (int base = begin + warp * 32; base < end; base += kThreads) {
        const int idx = base + lane;
        const bool valid = idx < end;
        const uint32_t d = valid ? digit_of(__ldg(keys + idx), shift) : 0u;
        const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
        const uint32_t peers = __match_any_sync(0xffffffffu, d) & vmask;
        if (valid && lane == __ffs(peers) - 1) s_hist[warp][d] += __popc(peers);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kThreads) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += s_hist[w][d];
        hist[(size_t)d * nb + blockIdx.x] = s;
    }
}

// One CTA per digit: exclusive scan of the digit's CTA counts in place.
__global__ void __launch_bounds__(kThreads) radix_spine_kernel(uint32_t* __restrict__ hist, int nb,
                                                               uint32_t* __restrict__ totals) {
    __shared__ uint32_t s_warp[kWarps];
    uint32_t* row = hist + (size_t)blockIdx.x * nb;
    uint32_t carry = 0;
    for (int base = 0; base < nb; base += kThreads) {
        const int idx = base + threadIdx.x;
        const uint32_t v = idx < nb ? row[idx] : 0u;
        uint32_t tot;
        const uint32_t incl = block_scan_incl(v, s_warp, &tot);
        if (idx < nb) row[idx] = carry + incl - v;
        carry += tot;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// Stable scatter of one pass.  FIRST: values are the input positions.
// FINAL: write the permutation (and rank/gidx) instead of keys and values.
template <bool FIRST, bool FINAL>
__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(
    const int32_t* __restrict__ keys_in, const int32_t* __restrict__ vals_in, int32_t* __restrict__ keys_out,
    int32_t* __restrict__ vals_out, const uint32_t* __restrict__ hist, const uint32_t* __restrict__ totals, int n,
    int per_cta, int nb, int shift, int32_t* __restrict__ rank_out, const int32_t* __restrict__ rank_in,
    int32_t* __restrict__ gidx) {
    __shared__ uint32_t s_base[kRadix];    // global position of this CTA's next key of each digit
    __shared__ uint32_t s_tstart[kRadix];  // tile-local start of each digit
    __shared__ uint32_t s_tcount[kRadix];
    __shared__ uint32_t s_whist[kWarps][kRadix];
    __shared__ int32_t s_keys[kTile];
    __shared__ int32_t s_vals[kTile];
    __shared__ uint32_t s_warp[kWarps];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint32_t tot = totals[tid];
        uint32_t all;
        const uint32_t incl = block_scan_incl(tot, s_warp, &all);
        s_base[tid] = incl - tot + hist[(size_t)tid * nb + blockIdx.x];
    }
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s_whist[w][tid] = 0u;
    __syncthreads();

    const int begin = blockIdx.x * per_cta;
    const int end = min(begin + per_cta, n);
    const uint32_t lt = lanemask_lt();
    for (int tile = begin; tile < end; tile += kTile) {
        const int tile_n = min(kTile, end - tile);
        int32_t k[kItems], v[kItems];
        uint32_t r[kItems];
#pragma unroll
        for (int it = 0; it < kItems; ++it) {
            const int local = warp * (32 * kItems) + it * 32 + lane;
            const bool valid = local < tile_n;
            const int idx = tile + local;
            const int32_t key = valid ? __ldg(keys_in + idx) : 0;
            int32_t val = 0;
            if (valid) val = FIRST ? idx : __ldg(vals_in + idx);
            const uint32_t d = digit_of(key, shift);
            const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
            const uint32_t peers = __match_any_sync(0xffffffffu, d) & vmask;
            const uint32_t before = s_whist[warp][d];
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1) s_whist[warp][d] = before + __popc(peers);
            __syncwarp();
            k[it] = key;
            v[it] = val;
            r[it] = before + __popc(peers & lt);
        }
        __syncthreads();
        {
            uint32_t run = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                const uint32_t c = s_whist[w][tid];
                s_whist[w][tid] = run;
                run += c;
            }
            s_tcount[tid] = run;
            uint32_t all;
            const uint32_t incl = block_scan_incl(run, s_warp, &all);
            s_tstart[tid] = incl - run;
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < kItems; ++it) {
            const int local = warp * (32 * kItems) + it * 32 + lane;
            if (local < tile_n) {
                const uint32_t d = digit_of(k[it], shift);
                const uint32_t pos = s_tstart[d] + s_whist[warp][d] + r[it];
                s_keys[pos] = k[it];
                s_vals[pos] = v[it];
            }
        }
        __syncthreads();
        for (int q = tid; q < tile_n; q += kThreads) {
            const int32_t key = s_keys[q];
            const int32_t val = s_vals[q];
            const uint32_t d = digit_of(key, shift);
            const uint32_t g = s_base[d] + (uint32_t)q - s_tstart[d];
            if (FINAL) {
                vals_out[g] = val;
                if (rank_out) rank_out[val] = (int32_t)g;
                if (gidx) gidx[g] = rank_in ? __ldg(rank_in + val) : val;
            } else {
                keys_out[g] = key;
                vals_out[g] = val;
            }
        }
        __syncthreads();
        s_base[tid] += s_tcount[tid];
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s_whist[w][tid] = 0u;
        __syncthreads();
    }
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

void plan(int n, int* nb, int* per_cta) {
    const int tiles = std::max(1, (n + kTile - 1) / kTile);
    const int tiles_per_cta = std::max(1, (tiles + kMaxCtas - 1) / kMaxCtas);
    *per_cta = tiles_per_cta * kTile;
    *nb = std::max(1, (n + *per_cta - 1) / *per_cta);
}

}  // namespace

size_t sort_scratch_bytes(int n) {
    int nb, per;
    plan(n, &nb, &per);
    const size_t kv = align256((size_t)std::max(n, 1) * sizeof(int32_t));
    return 4 * kv + align256((size_t)kRadix * nb * sizeof(uint32_t)) + align256(kRadix * sizeof(uint32_t));
}

void sort_scratch_carve(void* base, int n, SortScratch* s) {
    int nb, per;
    plan(n, &nb, &per);
    const size_t kv = align256((size_t)std::max(n, 1) * sizeof(int32_t));
    char* p = static_cast<char*>(base);
    s->key_a = reinterpret_cast<int32_t*>(p);
    s->val_a = reinterpret_cast<int32_t*>(p + kv);
    s->key_b = reinterpret_cast<int32_t*>(p + 2 * kv);
    s->val_b = reinterpret_cast<int32_t*>(p + 3 * kv);
    s->hist = reinterpret_cast<uint32_t*>(p + 4 * kv);
    s->totals = reinterpret_cast<uint32_t*>(p + 4 * kv + align256((size_t)kRadix * nb * sizeof(uint32_t)));
    s->n = n;
    s->nb = nb;
    s->per_cta = per;
}

int launch_morton_keys(const float* px, const float* py, const float* pz, int n, int32_t* keys, cudaStream_t st) {
    if (n <= 0) return 0;
    morton_keys_kernel<<<(n + 255) / 256, 256, 0, st>>>(px, py, pz, n, keys);
    return 1;
}

int launch_radix_sort(const int32_t* keys, int n, const SortScratch& s, int32_t* sigma, int32_t* rank_out,
                      const int32_t* rank_in, int32_t* gidx, cudaStream_t st) {
    if (n <= 0) return 0;
    int launches = 0;
    const int32_t* kin = keys;
    const int32_t* vin = nullptr;
    for (int pass = 0; pass < kPasses; ++pass) {
        const int shift = 8 * pass;
        int32_t* kout = (pass & 1) ? s.key_b : s.key_a;
        int32_t* vout = (pass & 1) ? s.val_b : s.val_a;
        radix_hist_kernel<<<s.nb, kThreads, 0, st>>>(kin, n, s.per_cta, s.nb, shift, s.hist);
        radix_spine_kernel<<<kRadix, kThreads, 0, st>>>(s.hist, s.nb, s.totals);
        const bool first = pass == 0, final = pass == kPasses - 1;
        if (first) {
            radix_scatter_kernel<true, false><<<s.nb, kThreads, 0, st>>>(kin, vin, kout, vout, s.hist, s.totals, n,
                                                                       s.per_cta, s.nb, shift, nullptr, nullptr,
                                                                       nullptr);
        } else if (final) {
            radix_scatter_kernel<false, true><<<s.nb, kThreads, 0, st>>>(kin, vin, nullptr, sigma, s.hist, s.totals,
                                                                       n, s.per_cta, s.nb, shift, rank_out, rank_in,
                                                                       gidx);
        } else {
            radix_scatter_kernel<false, false><<<s.nb, kThreads, 0, st>>>(kin, vin, kout, vout, s.hist, s.totals, n,
                                                                        s.per_cta, s.nb, shift, nullptr, nullptr,
                                                                        nullptr);
        }
        launches += 3;
        kin = kout;
        vin = vout;
    }
    return launches;
}

}  // namespace mpm
