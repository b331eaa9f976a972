// Ray hashing and sorting (compiled with --fmad=false). The hash is the
// reference's get_ray_hash (CoreRef.cpp:316-333) bit for bit; the order is the
// one SortRays_CPU (CoreRef.cpp:615-657) produces, which equals a stable sort
// of the rays by that 32-bit key: the reference compresses runs of equal
// adjacent keys into chunks, radix-sorts the chunks stably and expands them
// again, so equal keys keep their input order.
#include <algorithm>

#include "radix_sort.cuh"
#include "render.cuh"
#include "sort.cuh"

namespace rg {
namespace {

// Direction tables of the hash (Core.cpp:126-150): sector numbers of the
// polar angle (indexed by (1 + d.z) / 0.0625) and of the azimuth (indexed by
// (1 + d.y) / 0.125 and (1 + d.x) / 0.125). They are data; the reference's
// values are reproduced as they are.
__constant__ uint8_t c_omega[33] = {15, 14, 13, 12, 12, 11, 11, 11, 10, 10, 9, 9, 9, 8, 8, 8, 8,
                                    7,  7,  7,  6,  6,  6,  5,  5,  4,  4, 4, 3, 3, 2, 1, 0};
__constant__ uint8_t c_phi[17][17] = {
    {2, 2, 2, 2, 2, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 6},
    {1, 2, 2, 2, 2, 2, 3, 3, 4, 4, 4, 5, 5, 5, 5, 6, 6},
    {1, 1, 2, 2, 2, 2, 3, 3, 4, 4, 4, 5, 5, 5, 6, 6, 6},
    {1, 1, 1, 2, 2, 2, 3, 3, 4, 4, 4, 5, 5, 6, 6, 6, 6},
    {1, 1, 1, 1, 2, 2, 2, 3, 4, 4, 5, 5, 6, 6, 6, 6, 6},
    {0, 1, 1, 1, 1, 2, 2, 3, 4, 4, 5, 6, 6, 6, 6, 6, 7},
    {0, 0, 0, 0, 1, 1, 2, 2, 4, 5, 6, 6, 6, 7, 7, 7, 7},
    {0, 0, 0, 0, 0, 0, 1, 2, 4, 6, 6, 7, 7, 7, 7, 7, 7},
    {15, 15, 15, 15, 15, 15, 15, 15, 8, 8, 8, 8, 8, 8, 8, 8, 8},
    {15, 15, 15, 15, 15, 15, 14, 14, 12, 10, 9, 8, 8, 8, 8, 8, 8},
    {15, 15, 15, 15, 14, 14, 14, 13, 12, 10, 10, 9, 9, 8, 8, 8, 8},
    {15, 14, 14, 14, 14, 14, 13, 12, 12, 11, 10, 10, 9, 9, 9, 9, 8},
    {14, 14, 14, 14, 14, 13, 13, 12, 12, 11, 10, 10, 10, 9, 9, 9, 9},
    {14, 14, 14, 14, 13, 13, 12, 12, 12, 11, 11, 10, 10, 10, 9, 9, 9},
    {14, 14, 14, 13, 13, 13, 12, 12, 12, 11, 11, 10, 10, 10, 10, 9, 9},
    {14, 14, 13, 13, 13, 13, 12, 12, 12, 11, 11, 10, 10, 10, 10, 10, 9},
    {14, 13, 13, 13, 13, 12, 12, 12, 12, 11, 11, 11, 10, 10, 10, 10, 10}};

// (int)f as the reference's x86 build computes it (cvttss2si): NaN and
// values outside the int range give INT_MIN, where CUDA's conversion would
// saturate.
__device__ __forceinline__ int f2i_x86(float f) {
    if (f != f || f >= 2147483648.0f || f < -2147483648.0f) return (int)0x80000000u;
    return __float2int_rz(f);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Bit k of v to bit 3k (morton_table_256, Core.cpp:109-126) or 2k (morton_table_16, Core.cpp:106).
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0xFFu;
    v = (v | (v << 8)) & 0x0000F00Fu;
    v = (v | (v << 4)) & 0x000C30C3u;
    v = (v | (v << 2)) & 0x00249249u;
    return v;
}
__device__ __forceinline__ uint32_t spread2(uint32_t v) {
    v &= 0xFu;
    v = (v | (v << 2)) & 0x33u;
    v = (v | (v << 1)) & 0x55u;
    return v;
}

// get_ray_hash, CoreRef.cpp:316-333: the origin's cell as a 24-bit Morton
// code under 8 bits of direction sector.
__device__ __forceinline__ uint32_t ray_hash(float4 o, float4 d, float3 root_min, float3 cell) {
    const int x = clampi(f2i_x86(__fdiv_rn(__fsub_rn(o.x, root_min.x), cell.x)), 0, 255);
    const int y = clampi(f2i_x86(__fdiv_rn(__fsub_rn(o.y, root_min.y), cell.y)), 0, 255);
    const int z = clampi(f2i_x86(__fdiv_rn(__fsub_rn(o.z, root_min.z), cell.z)), 0, 255);
    const int oi = clampi(f2i_x86(__fdiv_rn(__fadd_rn(1.0f, d.z), 0.0625f)), 0, 32);
    const int py = clampi(f2i_x86(__fdiv_rn(__fadd_rn(1.0f, d.y), 0.125f)), 0, 16);
    const int px = clampi(f2i_x86(__fdiv_rn(__fadd_rn(1.0f, d.x), 0.125f)), 0, 16);
    const uint32_t om = spread2(c_omega[oi]);
    const uint32_t pm = spread2(c_phi[py][px]);
    return (om << 25) | (pm << 24) | (spread3((uint32_t)y) << 2) | (spread3((uint32_t)z) << 1) | spread3((uint32_t)x);
}

// Hash of every ray, also counted into the radix sort's digit histograms
// (all four 8-bit digits); a grid-stride loop.
__global__ void k_ray_hash(const float4 *__restrict__ rays, uint32_t n, float3 root_min, float3 cell, uint32_t *__restrict__ keys_out,
                           uint32_t *__restrict__ sort_keys, uint32_t *__restrict__ counts) {
    __shared__ uint32_t s_counts[4 * 256];
    for (int k = threadIdx.x; k < 4 * 256; k += blockDim.x) s_counts[k] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t key = ray_hash(rays[2ull * i], rays[2ull * i + 1], root_min, cell);
        if (keys_out) keys_out[i] = key;
        sort_keys[i] = key;
        rs_count_key(s_counts, key, 0, 4);
    }
    __syncthreads();
    rs_flush_counts(s_counts, counts, 4);
}

// Blocks of the key kernels: a grid that strides over the rays, few enough
// that the blocks' flushes of their digit counts stay cheap.
constexpr uint32_t KEY_BLOCKS = 148 * 4;

// Keys of a trace order: the ray hash (mode 1) or the hash with its 8-bit
// direction sector moved below the origin cell (mode 2).
__global__ void k_order_keys(const float4 *__restrict__ rays, uint32_t n, float3 root_min, float3 cell, int mode,
                             uint32_t *__restrict__ keys) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t h = ray_hash(rays[2ull * i], rays[2ull * i + 1], root_min, cell);
    keys[i] = mode == 2 ? ((h << 8) | (h >> 24)) : h;
}

__global__ void k_gather_rays(const float4 *__restrict__ rays, const uint32_t *__restrict__ perm, uint32_t n, float4 *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s = perm[i];
    out[2ull * i] = rays[2ull * s];
    out[2ull * i + 1] = rays[2ull * s + 1];
}

// Keys of the render loop's sort for the live rays (i < *count): the ray's
// hash in its job's grid, with the job above it when there are several.
template <typename Key>
__global__ void k_loop_keys(const FrameJob *__restrict__ jobs, const float4 *__restrict__ rays, const uint32_t *__restrict__ ray_job,
                            const uint32_t *__restrict__ count, uint32_t capacity, Key *__restrict__ keys, int begin_bit, int passes,
                            uint32_t *__restrict__ counts) {
    __shared__ uint32_t s_counts[RS_MAX_PASSES * 256];
    const uint32_t n = min(*count, capacity);
    if (blockIdx.x * blockDim.x >= n) return; // the whole block is past the live rays
    for (int k = threadIdx.x; k < passes * 256; k += blockDim.x) s_counts[k] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t j = ray_job[i];
        const FrameJob &J = jobs[j];
        const uint32_t h = ray_hash(rays[2ull * i], rays[2ull * i + 1], make_float3(J.root_min[0], J.root_min[1], J.root_min[2]),
                                    make_float3(J.cell[0], J.cell[1], J.cell[2]));
        const Key key = sizeof(Key) == 8 ? (Key)(((uint64_t)j << 32) | h) : (Key)h;
        keys[i] = key;
        rs_count_key(s_counts, key, begin_bit, passes);
    }
    __syncthreads();
    rs_flush_counts(s_counts, counts, passes);
}

__global__ void k_loop_gather(const float4 *__restrict__ rays, const RayPayload *__restrict__ pay, const uint32_t *__restrict__ ray_job,
                              const uint32_t *__restrict__ perm, const uint32_t *__restrict__ count, uint32_t capacity,
                              float4 *__restrict__ rays_out, RayPayload *__restrict__ pay_out, uint32_t *__restrict__ job_out,
                              uint32_t *__restrict__ count_out) {
    const uint32_t n = min(*count, capacity);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *count_out = n;
    if (i >= n) return;
    const uint32_t s = perm[i];
    if (s >= n) return; // cannot happen: the first n positions hold the n valid rays
    rays_out[2ull * i] = rays[2ull * s];
    rays_out[2ull * i + 1] = rays[2ull * s + 1];
    static_assert(sizeof(RayPayload) % 16 == 0, "payload copied as uint4");
    const uint4 *src = reinterpret_cast<const uint4 *>(pay + s);
    uint4 *dst = reinterpret_cast<uint4 *>(pay_out + i);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(RayPayload) / 16); k++) dst[k] = src[k];
    job_out[i] = ray_job[s];
}

// The render loop's sort keys: the ray hash from this bit up (the job above).
constexpr int LOOP_SORT_BEGIN_BIT = 16;

int job_bits(int n_jobs) {
    int b = 0;
    while ((1 << b) < n_jobs) b++;
    return b;
}

} // namespace

size_t loop_sort_scratch_bytes(uint64_t capacity, int n_jobs) {
    const int kb = n_jobs > 1 ? 8 : 4;
    return ((capacity * kb + 255) / 256) * 256 + ((capacity * 4 + 255) / 256) * 256 + radix_sort_scratch_bytes(capacity, kb);
}

cudaError_t launch_loop_sort(const FrameJob *jobs, int n_jobs, const float4 *rays, const RayPayload *pay, const uint32_t *ray_job,
                             const uint32_t *count, uint32_t capacity, float4 *rays_out, RayPayload *pay_out, uint32_t *job_out,
                             uint32_t *count_out, void *scratch, cudaStream_t st, uint32_t *err) {
    if (capacity == 0) return cudaSuccess;
    const int kb = n_jobs > 1 ? 8 : 4;
    char *p = static_cast<char *>(scratch);
    void *keys = p;
    uint32_t *perm = reinterpret_cast<uint32_t *>(p + ((uint64_t(capacity) * kb + 255) / 256) * 256);
    void *rs_scratch = reinterpret_cast<char *>(perm) + ((uint64_t(capacity) * 4 + 255) / 256) * 256;
    const uint32_t blocks = (capacity + 255) / 256;
    const uint32_t key_blocks = std::min(blocks, KEY_BLOCKS);
    // Only the live rays (their count is on the device): keys, sort and
    // gather all read min(*count, capacity) there; blocks past it return at
    // once. The sort uses the hash's top 16 bits (the direction sector and
    // the origin's cell at 1/32 of the scene box per axis) under the job:
    // the images do not depend on the order, and two digit passes group the
    // rays as well for the trace as four.
    const int begin = LOOP_SORT_BEGIN_BIT, end = kb == 8 ? 32 + job_bits(n_jobs) : 32, passes = (end - begin + 7) / 8;
    cudaError_t e = radix_sort_begin(rs_scratch, capacity, kb, begin, end, st);
    if (e != cudaSuccess) return e;
    uint32_t *counts = radix_sort_counts(rs_scratch, capacity, kb);
    if (kb == 8)
        k_loop_keys<uint64_t><<<key_blocks, 256, 0, st>>>(jobs, rays, ray_job, count, capacity, static_cast<uint64_t *>(keys), begin, passes,
                                                         counts);
    else
        k_loop_keys<uint32_t><<<key_blocks, 256, 0, st>>>(jobs, rays, ray_job, count, capacity, static_cast<uint32_t *>(keys), begin, passes,
                                                         counts);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = radix_sort_pairs(keys, perm, capacity, kb, begin, end, rs_scratch, st, count, true, err, true);
    if (e != cudaSuccess) return e;
    k_loop_gather<<<blocks, 256, 0, st>>>(rays, pay, ray_job, perm, count, capacity, rays_out, pay_out, job_out, count_out);
    return cudaGetLastError();
}

size_t sort_rays_scratch_bytes(uint64_t n) { return ((n * 4 + 255) / 256) * 256 + radix_sort_scratch_bytes(n, 4); }

cudaError_t sort_rays(const float4 *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                      uint32_t *perm_out, float4 *rays_out, void *scratch, cudaStream_t st, uint32_t *err) {
    if (n == 0) return cudaSuccess;
    if (n > RS_MAX_ITEMS) return cudaErrorInvalidValue;
    char *p = static_cast<char *>(scratch);
    uint32_t *sort_keys = reinterpret_cast<uint32_t *>(p);
    void *rs_scratch = p + ((n * 4 + 255) / 256) * 256;
    const uint32_t blocks = (uint32_t)((n + 255) / 256);
    cudaError_t e = radix_sort_begin(rs_scratch, n, 4, 0, 32, st);
    if (e != cudaSuccess) return e;
    k_ray_hash<<<std::min(blocks, KEY_BLOCKS), 256, 0, st>>>(rays, (uint32_t)n, make_float3(root_min[0], root_min[1], root_min[2]),
                                       make_float3(cell_size[0], cell_size[1], cell_size[2]), keys_out, sort_keys,
                                       radix_sort_counts(rs_scratch, n, 4));
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = radix_sort_pairs(sort_keys, perm_out, n, 4, 0, 32, rs_scratch, st, nullptr, true, err, true);
    if (e != cudaSuccess) return e;
    if (rays_out) {
        k_gather_rays<<<blocks, 256, 0, st>>>(rays, perm_out, (uint32_t)n, rays_out);
        e = cudaGetLastError();
    }
    return e;
}

} // namespace rg

namespace rg {

size_t order_scratch_bytes(uint64_t n) { return ((n * 4 + 255) / 256) * 256 * 2 + radix_sort_scratch_bytes(n, 4); }

cudaError_t order_rays(const float4 *rays, uint32_t n, const float root_min[3], const float cell_size[3], int mode, int bits, void *scratch,
                       uint32_t **order_out, cudaStream_t st) {
    if (bits <= 0 || bits > 32) bits = 32;
    if (bits < 8) bits = 8;
    char *p = static_cast<char *>(scratch);
    uint32_t *keys = reinterpret_cast<uint32_t *>(p);
    uint32_t *order = reinterpret_cast<uint32_t *>(p + ((uint64_t(n) * 4 + 255) / 256) * 256);
    void *rs_scratch = p + ((uint64_t(n) * 4 + 255) / 256) * 256 * 2;
    *order_out = order;
    if (n == 0) return cudaSuccess;
    k_order_keys<<<(n + 255) / 256, 256, 0, st>>>(rays, n, make_float3(root_min[0], root_min[1], root_min[2]),
                                                 make_float3(cell_size[0], cell_size[1], cell_size[2]), mode, keys);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return radix_sort_pairs(keys, order, n, 4, 32 - bits, 32, rs_scratch, st, nullptr, true);
}

} // namespace rg
