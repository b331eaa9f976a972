// Stable LSD radix sort of (key, value) pairs on the GPU, 8-bit digits, in
// the one-sweep form (Adinets and Merrill, "Onesweep: a faster least
// significant digit radix sort for GPUs", 2022): one histogram launch counts
// the digits of every pass at once, then each digit pass is ONE launch in
// which every tile ranks its keys, publishes its per-digit counts and finds
// its global offsets by a decoupled look-back over the tiles before it, then
// scatters through shared memory so that each digit's run is written
// contiguously. Used by the BVH build (64-bit Morton keys), the ray sort
// (32-bit ray hashes) and the render loop's sort (keys of the live rays only,
// their count read on the device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rg {

constexpr int RS_THREADS = 256;                // one digit per thread
constexpr int RS_ITEMS = 16;                   // keys per thread per tile
constexpr int RS_TILE = RS_THREADS * RS_ITEMS; // 4096 keys per tile
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_MAX_PASSES = 8;
constexpr uint64_t RS_MAX_ITEMS = (1ull << 30) - 1; // look-back counts are 30 bits

// Error bit OR-ed into the caller's error word when a tile's look-back waited
// longer than its bound for a tile before it (a wait that cannot end on a
// correct launch; the sort's output is then not valid).
constexpr uint32_t SORT_ERR_LOOKBACK = 8u;

// Scratch needed by radix_sort_pairs for up to n items (bytes): the
// ping-pong keys and values, the digit counts and tile counters of every
// pass, and one status word per (pass, tile, digit).
constexpr uint64_t RS_COUNTER_WORDS = RS_MAX_PASSES * 256 + 64;
constexpr uint64_t rs_align256(uint64_t b) { return (b + 255) / 256 * 256; }
constexpr uint64_t radix_sort_scratch_bytes_c(uint64_t n, int key_bytes) {
    return rs_align256(n * key_bytes) + rs_align256(n * 4) +
           (RS_COUNTER_WORDS + (uint64_t)key_bytes * ((n + RS_TILE - 1) / RS_TILE) * 256) * 4 + 256;
}
size_t radix_sort_scratch_bytes(uint64_t n, int key_bytes);

// Digit counts accumulated by the caller's key kernel instead of the sort's
// own histogram launch (one read of the keys saved): radix_sort_begin zeroes
// the sort's counters on the stream; the key kernel counts each key's digits
// into a block-shared array (rs_count_key; RS_MAX_PASSES x 256 words, zeroed
// by the block) and adds the block's counts to radix_sort_counts(scratch)
// (rs_flush_counts); radix_sort_pairs then runs with counted = true and the
// same n, key_bytes and bit range.
cudaError_t radix_sort_begin(void *scratch, uint64_t n, int key_bytes, int begin_bit, int end_bit, cudaStream_t st);
uint32_t *radix_sort_counts(void *scratch, uint64_t n, int key_bytes);

#ifdef __CUDACC__
template <typename K>
__device__ __forceinline__ void rs_count_key(uint32_t *s_counts, K key, int begin_bit, int passes) {
    for (int p = 0; p < passes; p++) atomicAdd(&s_counts[p * 256 + ((uint32_t)(key >> (begin_bit + 8 * p)) & 0xFFu)], 1u);
}
__device__ __forceinline__ void rs_flush_counts(const uint32_t *s_counts, uint32_t *g_counts, int passes) {
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        if (s_counts[i]) atomicAdd(&g_counts[i], s_counts[i]);
}
#endif

// Sorts keys/vals in place, stably, on the digits in [begin_bit, end_bit).
// n: the number of items, or, when n_dev is not null, the capacity of the
// arrays, with the item count read on the device as min(n, *n_dev) (nothing
// past it is read or written). vals may hold anything; with vals_identity the
// input values are taken as 0, 1, 2, ... and vals is only written. key_bytes:
// 4 or 8. err (may be null): device word that gets SORT_ERR_LOOKBACK.
// Returns a CUDA error code; n above RS_MAX_ITEMS is cudaErrorInvalidValue.
cudaError_t radix_sort_pairs(void *keys, uint32_t *vals, uint64_t n, int key_bytes, int begin_bit, int end_bit, void *scratch,
                             cudaStream_t stream, const uint32_t *n_dev = nullptr, bool vals_identity = false,
                             uint32_t *err = nullptr, bool counted = false);

} // namespace rg
