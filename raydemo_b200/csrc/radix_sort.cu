// Stable LSD radix sort, 8-bit digits (see radix_sort.cuh).
#include "radix_sort.cuh"

namespace rg {
namespace {

template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const K *__restrict__ keys, uint64_t n, int shift, uint32_t num_tiles,
                                                        uint32_t *__restrict__ hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int j = 0; j < RS_ITEMS; j++) {
        const uint64_t i = base + (uint64_t)j * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * num_tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of `count` entries with one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_rs_scan(uint32_t *__restrict__ data, uint32_t count) {
    __shared__ uint32_t sums[1024];
    const uint32_t per = (count + 1023) / 1024;
    const uint32_t b = threadIdx.x * per, e = min(count, b + per);
    uint32_t s = 0;
    for (uint32_t i = b; i < e; i++) s += data[i];
    sums[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const uint32_t v = threadIdx.x >= (uint32_t)off ? sums[threadIdx.x - off] : 0u;
        __syncthreads();
        sums[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = sums[threadIdx.x] - s; // exclusive prefix of this thread's chunk
    for (uint32_t i = b; i < e; i++) {
        const uint32_t v = data[i];
        data[i] = run;
        run += v;
    }
}

template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const K *__restrict__ keys, const uint32_t *__restrict__ vals, K *__restrict__ keys_out,
                                                           uint32_t *__restrict__ vals_out, uint64_t n, int shift, uint32_t num_tiles,
                                                           const uint32_t *__restrict__ offsets) {
    __shared__ uint32_t run[256];
    __shared__ uint32_t wc[RS_WARPS][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    run[tid] = offsets[(uint64_t)tid * num_tiles + blockIdx.x];
    for (int w = 0; w < RS_WARPS; w++) wc[w][tid] = 0;
    __syncthreads();
    const uint32_t lanemask_lt = (1u << lane) - 1u;
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
    for (int j = 0; j < RS_ITEMS; j++) {
        const uint64_t i = base + (uint64_t)j * RS_THREADS + tid;
        const bool valid = i < n;
        K key = 0;
        uint32_t val = 0;
        if (valid) {
            key = keys[i];
            val = vals[i];
        }
        const uint32_t d = valid ? ((uint32_t)(key >> shift) & 0xFFu) : 0x100u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & lanemask_lt);
        if (valid && rank == 0) wc[warp][d] = __popc(peers);
        __syncthreads();
        {
            uint32_t r = run[tid];
#pragma unroll
            for (int w = 0; w < RS_WARPS; w++) {
                const uint32_t c = wc[w][tid];
                wc[w][tid] = r;
                r += c;
            }
            run[tid] = r;
        }
        __syncthreads();
        if (valid) {
            const uint32_t pos = wc[warp][d] + rank;
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) wc[w][tid] = 0;
        __syncthreads();
    }
}

template <typename K>
cudaError_t sort_impl(K *keys, uint32_t *vals, uint64_t n, int begin_bit, int end_bit, void *scratch, cudaStream_t st) {
    if (n <= 1) return cudaSuccess;
    const uint32_t num_tiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    char *p = static_cast<char *>(scratch);
    K *keys_alt = reinterpret_cast<K *>(p);
    p += ((n * sizeof(K) + 255) / 256) * 256;
    uint32_t *vals_alt = reinterpret_cast<uint32_t *>(p);
    p += ((n * 4 + 255) / 256) * 256;
    uint32_t *hist = reinterpret_cast<uint32_t *>(p);
    K *src_k = keys, *dst_k = keys_alt;
    uint32_t *src_v = vals, *dst_v = vals_alt;
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        k_rs_hist<K><<<num_tiles, RS_THREADS, 0, st>>>(src_k, n, shift, num_tiles, hist);
        k_rs_scan<<<1, 1024, 0, st>>>(hist, 256u * num_tiles);
        k_rs_scatter<K><<<num_tiles, RS_THREADS, 0, st>>>(src_k, src_v, dst_k, dst_v, n, shift, num_tiles, hist);
        K *tk = src_k; src_k = dst_k; dst_k = tk;
        uint32_t *tv = src_v; src_v = dst_v; dst_v = tv;
        passes++;
    }
    if (passes & 1) {
        cudaError_t e = cudaMemcpyAsync(keys, src_k, n * sizeof(K), cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
        e = cudaMemcpyAsync(vals, src_v, n * 4, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

} // namespace

size_t radix_sort_scratch_bytes(uint64_t n, int key_bytes) {
    const uint64_t num_tiles = (n + RS_TILE - 1) / RS_TILE;
    return ((n * key_bytes + 255) / 256) * 256 + ((n * 4 + 255) / 256) * 256 + 256 * num_tiles * 4 + 256;
}

cudaError_t radix_sort_pairs(void *keys, uint32_t *vals, uint64_t n, int key_bytes, int begin_bit, int end_bit, void *scratch,
                             cudaStream_t stream) {
    if (key_bytes == 8) return sort_impl<uint64_t>(static_cast<uint64_t *>(keys), vals, n, begin_bit, end_bit, scratch, stream);
    if (key_bytes == 4) return sort_impl<uint32_t>(static_cast<uint32_t *>(keys), vals, n, begin_bit, end_bit, scratch, stream);
    return cudaErrorInvalidValue;
}

} // namespace rg
