// Ray hashing and sorting (the reference's SortRays_CPU, CoreRef.cpp:615-657).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rg {

// Scratch bytes sort_rays needs for n rays.
size_t sort_rays_scratch_bytes(uint64_t n);

// keys_out[i] = get_ray_hash(ray i) (CoreRef.cpp:316-333); perm_out = the
// order SortRays_CPU puts the rays in (a stable sort on the key: perm_out[k]
// is the input index of the ray at position k); rays_out (may be null) = the
// rays in that order. rays / rays_out: n records of 8 floats
// (ox, oy, oz, tmax, dx, dy, dz, unused). All pointers are device memory.
// err (may be null): device word that gets SORT_ERR_LOOKBACK if the radix
// sort's bounded wait ran out. At most RS_MAX_ITEMS rays.
cudaError_t sort_rays(const float4 *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                      uint32_t *perm_out, float4 *rays_out, void *scratch, cudaStream_t st, uint32_t *err = nullptr);

} // namespace rg

namespace rg {

// Trace order of n rays (n <= RS_MAX_ITEMS): a stable sort of the ray indices
// by get_ray_hash over the grid (root_min, cell) -- mode 1 -- or by that hash
// rotated so that the origin's 24-bit Morton cell lies above the 8-bit
// direction sector -- mode 2 --, on the key's top `bits` bits. *order_out
// points into scratch (order_scratch_bytes(n)) when the call returns.
size_t order_scratch_bytes(uint64_t n);
cudaError_t order_rays(const float4 *rays, uint32_t n, const float root_min[3], const float cell_size[3], int mode, int bits, void *scratch,
                       uint32_t **order_out, cudaStream_t st);

} // namespace rg
