// Allocation-free ray sort: ray_sort_rays_noalloc.
//
// Some callers cannot call cudaMalloc: a renderer embedded in a host
// application whose GPU memory is owned by that application's own allocator
// and budget, or a latency-bound frame loop that must not stall on
// cudaMalloc's implicit device-wide synchronisation. This entry point does
// the same work as ray_sort_rays without allocating anything: its scratch
// memory is a fixed array in this file, so it exists on every GPU that loads
// the library from the moment the module is loaded until the process exits.
#include <mutex>

#include "../../include/raygpu.h"
#include "common.cuh"
#include "radix_sort.cuh"
#include "scene.hpp"
#include "sort.cuh"

namespace rg {
namespace {

// Scratch for RAY_SORT_NOALLOC_MAX_RAYS rays, laid out as sort_rays expects:
// the keys being sorted, then the radix sort's ping-pong keys and values, its
// digit counts and tile counters, and its look-back status words
// (13,640,192 bytes = 13.01 MiB for 1,048,576 rays).
constexpr uint64_t kMaxRays = RAY_SORT_NOALLOC_MAX_RAYS;
constexpr uint64_t kScratchBytes = rs_align256(kMaxRays * 4) + radix_sort_scratch_bytes_c(kMaxRays, 4);
static_assert(kScratchBytes == 13640192ull, "the documented size of the static scratch");

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

// Device address of g_sort_scratch per device, looked up once per device.
// Host code cannot use the symbol g_sort_scratch itself as a device pointer.
constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;

} // namespace
} // namespace rg

using namespace rg;

extern "C" int ray_sort_rays_noalloc(const float *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                                     uint32_t *perm_out, float *rays_out, void *stream) {
    RG_API_LOCK; // host side serialised with every other entry point, like ray_sort_rays
    if (!root_min || !cell_size || (n && (!rays || !perm_out))) {
        set_error("ray_sort_rays_noalloc: null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (n > kMaxRays) {
        set_error("ray_sort_rays_noalloc: too many rays; the static scratch holds at most RAY_SORT_NOALLOC_MAX_RAYS (1048576)");
        return RAY_ERR_INVALID_ARG;
    }
    if (n == 0) return RAY_OK;
    int dev = 0;
    RG_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("ray_sort_rays_noalloc: device index out of range");
        return RAY_ERR_INVALID_ARG;
    }
    void *scratch = nullptr;
    {
        // First call on this device (with the device current): look up the
        // array's device address. This may load the library's module on the
        // device, so make this first call before any stream capture begins.
        // The address is kept for the life of the process: a device reset
        // (cudaDeviceReset) while the library is in use invalidates it.
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
            if (e != cudaSuccess) {
                set_error(std::string("ray_sort_rays_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
                return RAY_ERR_CUDA;
            }
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    if (sort_rays_scratch_bytes(n) > kScratchBytes) {
        set_error("ray_sort_rays_noalloc: scratch layout larger than the static array");
        return RAY_ERR_INVALID_ARG;
    }
    // Nothing in the scratch has to start at zero: the hash pass writes every
    // key it sorts, and each radix pass writes all of its histograms before
    // reading them. The array keeps the last call's contents, and calls that
    // overlap on the GPU (different streams, or host threads) share it and race.
    RG_CUDA_TRY(sort_rays(reinterpret_cast<const float4 *>(rays), n, root_min, cell_size, keys_out, perm_out,
                          reinterpret_cast<float4 *>(rays_out), scratch, static_cast<cudaStream_t>(stream)));
    return RAY_OK;
}
