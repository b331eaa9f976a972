// Stable LSD radix sort of (key, value) pairs on the GPU, 8-bit digits.
// One pass = per-tile digit histograms, one exclusive scan over the
// digit-major histogram matrix, and a stable scatter that ranks equal digits
// inside a tile with warp match masks. Used by the BVH build (64-bit Morton
// keys) and by the ray sort (32-bit ray hashes).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rg {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;                       // items per thread per tile
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;     // 4096 keys per tile
constexpr int RS_WARPS = RS_THREADS / 32;

// Scratch needed by radix_sort_pairs for n items (bytes).
size_t radix_sort_scratch_bytes(uint64_t n, int key_bytes);

// Sorts keys/vals (n items) in place, using `scratch` (radix_sort_scratch_bytes)
// for the ping-pong buffers and histograms. key_bytes: 4 or 8. Only the digits
// in [begin_bit, end_bit) are sorted on. Returns a CUDA error code.
cudaError_t radix_sort_pairs(void *keys, uint32_t *vals, uint64_t n, int key_bytes, int begin_bit, int end_bit, void *scratch,
                             cudaStream_t stream);

} // namespace rg
