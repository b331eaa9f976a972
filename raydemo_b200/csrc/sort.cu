// Ray hashing and sorting (compiled with --fmad=false). The hash is the
// reference's get_ray_hash (CoreRef.cpp:316-333) bit for bit; the order is the
// one SortRays_CPU (CoreRef.cpp:615-657) produces, which equals a stable sort
// of the rays by that 32-bit key: the reference compresses runs of equal
// adjacent keys into chunks, radix-sorts the chunks stably and expands them
// again, so equal keys keep their input order.
#include "radix_sort.cuh"
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

__global__ void k_ray_hash(const float4 *__restrict__ rays, uint32_t n, float3 root_min, float3 cell, uint32_t *__restrict__ keys_out,
                           uint32_t *__restrict__ sort_keys, uint32_t *__restrict__ perm) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = rays[2ull * i], d = rays[2ull * i + 1];
    // get_ray_hash, CoreRef.cpp:316-333
    const int x = clampi(f2i_x86(__fdiv_rn(__fsub_rn(o.x, root_min.x), cell.x)), 0, 255);
    const int y = clampi(f2i_x86(__fdiv_rn(__fsub_rn(o.y, root_min.y), cell.y)), 0, 255);
    const int z = clampi(f2i_x86(__fdiv_rn(__fsub_rn(o.z, root_min.z), cell.z)), 0, 255);
    const int oi = clampi(f2i_x86(__fdiv_rn(__fadd_rn(1.0f, d.z), 0.0625f)), 0, 32);
    const int py = clampi(f2i_x86(__fdiv_rn(__fadd_rn(1.0f, d.y), 0.125f)), 0, 16);
    const int px = clampi(f2i_x86(__fdiv_rn(__fadd_rn(1.0f, d.x), 0.125f)), 0, 16);
    const uint32_t om = spread2(c_omega[oi]);
    const uint32_t pm = spread2(c_phi[py][px]);
    const uint32_t key = (om << 25) | (pm << 24) | (spread3((uint32_t)y) << 2) | (spread3((uint32_t)z) << 1) | spread3((uint32_t)x);
    if (keys_out) keys_out[i] = key;
    sort_keys[i] = key;
    perm[i] = i;
}

__global__ void k_gather_rays(const float4 *__restrict__ rays, const uint32_t *__restrict__ perm, uint32_t n, float4 *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s = perm[i];
    out[2ull * i] = rays[2ull * s];
    out[2ull * i + 1] = rays[2ull * s + 1];
}

} // namespace

size_t sort_rays_scratch_bytes(uint64_t n) { return ((n * 4 + 255) / 256) * 256 + radix_sort_scratch_bytes(n, 4); }

cudaError_t sort_rays(const float4 *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                      uint32_t *perm_out, float4 *rays_out, void *scratch, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    if (n > 0xffffffffull) return cudaErrorInvalidValue;
    char *p = static_cast<char *>(scratch);
    uint32_t *sort_keys = reinterpret_cast<uint32_t *>(p);
    void *rs_scratch = p + ((n * 4 + 255) / 256) * 256;
    const uint32_t blocks = (uint32_t)((n + 255) / 256);
    k_ray_hash<<<blocks, 256, 0, st>>>(rays, (uint32_t)n, make_float3(root_min[0], root_min[1], root_min[2]),
                                       make_float3(cell_size[0], cell_size[1], cell_size[2]), keys_out, sort_keys, perm_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = radix_sort_pairs(sort_keys, perm_out, n, 4, 0, 32, rs_scratch, st);
    if (e != cudaSuccess) return e;
    if (rays_out) {
        k_gather_rays<<<blocks, 256, 0, st>>>(rays, perm_out, (uint32_t)n, rays_out);
        e = cudaGetLastError();
    }
    return e;
}

} // namespace rg
