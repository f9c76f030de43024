// Morton keys + stable sort for callers that cannot allocate device memory.
//
// mpm_sort_particles_device takes its radix-sort scratch (ping-pong key and
// value buffers, per-CTA digit histograms) with cudaMallocAsync on every
// call.  Some hosts cannot do that: a process whose device memory is owned
// by another allocator (a game engine's or a framework's pool that has
// reserved the memory up front), a real-time frame loop that must not take
// an allocator's locks or block on a cudaFree's device synchronisation, or a
// driver stack where stream-ordered allocation is not available.  This file
// gives them the same operator with the scratch in one file-scope device
// array, sized for at most MPM_SORT_STATIC_MAX_PARTICLES particles.
//
// The array exists once per device that loads this library and stays
// resident until the process exits.  Host code cannot pass the array's name
// to a kernel (on the host it names a stand-in object, not device memory),
// so the first call on each device looks up its device address with
// cudaGetSymbolAddress, with that device current, and caches it.  The cache
// assumes the device's primary context lives as long as the process: after a
// cudaDeviceReset the module is loaded again at another address, and a
// process that resets a device must not call this entry point afterwards.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "kernels.h"
#include "mpm_b200.h"

namespace {

// 4 key/value buffers of 4 bytes per particle, plus the [256][CTAs] digit
// histogram (at most 4 CTAs per SM x 148 SMs) and the 256 digit totals, each
// rounded to 256 bytes: 1 MiB covers the last two with room to spare.
constexpr size_t kStaticSortScratchBytes = 16ull * MPM_SORT_STATIC_MAX_PARTICLES + (1ull << 20);

static __device__ __align__(256) unsigned char g_sort_scratch[kStaticSortScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

mpm_status fail(mpm_status s, const std::string& msg) {
    mpm::set_global_error(msg);
    return s;
}

mpm_status cuda_fail(cudaError_t err, const char* what) {
    cudaGetLastError();  // clear a non-sticky error
    return fail(MPM_ERR_CUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorName(err) + " (" +
                                  cudaGetErrorString(err) + ")");
}

// Device address of g_sort_scratch on the current device, looked up once per
// device.
mpm_status scratch_on_current_device(void** out) {
    int dev = -1;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return cuda_fail(err, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(MPM_ERR_UNSUPPORTED, "device index beyond 63");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        err = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (err != cudaSuccess) return cuda_fail(err, "cudaGetSymbolAddress(sort scratch)");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return MPM_OK;
}

}  // namespace

extern "C" mpm_status mpm_sort_particles_device_static(const float* px, const float* py, const float* pz,
                                                       int64_t n, int32_t* d_keys, int32_t* d_perm, void* stream) {
    mpm::set_global_error("");
    if (n < 0) return fail(MPM_ERR_INVALID_ARGUMENT, "n out of range");
    if (n > MPM_SORT_STATIC_MAX_PARTICLES)
        return fail(MPM_ERR_INVALID_ARGUMENT,
                    "n = " + std::to_string(n) + " exceeds the static sort scratch maximum of " +
                        std::to_string(MPM_SORT_STATIC_MAX_PARTICLES) +
                        " particles; use mpm_sort_particles_device for larger inputs");
    if (n == 0) return MPM_OK;
    if (!px || !py || !pz || !d_keys || !d_perm) return fail(MPM_ERR_INVALID_ARGUMENT, "device pointers must be non-NULL");
    const int ni = (int)n;
    if (mpm::sort_scratch_bytes(ni) > kStaticSortScratchBytes)
        return fail(MPM_ERR_UNSUPPORTED, "static sort scratch is smaller than the sort plan needs");
    void* scratch = nullptr;
    mpm_status s = scratch_on_current_device(&scratch);
    if (s != MPM_OK) return s;
    // Every histogram entry and digit total is written by its pass before it
    // is read, and the key/value buffers are written before they are read, so
    // nothing left in the array by an earlier call needs clearing.
    mpm::SortScratch plan;
    mpm::sort_scratch_carve(scratch, ni, &plan);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    mpm::launch_morton_keys(px, py, pz, ni, d_keys, st);
    mpm::launch_radix_sort(d_keys, ni, plan, d_perm, nullptr, nullptr, nullptr, st);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_fail(err, "static sort launch");
    return MPM_OK;
}
