// Stable one-sweep LSD radix sort, 8-bit digits (see radix_sort.cuh).
//
// Launches per sort: one memset of the counters, one histogram launch for
// all digit passes, then one launch per pass (plus a copy when the number of
// passes is odd, so that the result ends in the caller's arrays).
//
// A pass, per tile of RS_TILE = 256 x 16 keys (tiles are numbered in the
// order their
// blocks start, through an atomic counter, so every tile's predecessors are
// running or done):
//   1. each warp ranks its 32 x ITEMS keys stably (index order): the lanes
//      of one digit found with one ballot per digit bit, per-warp digit
//      counters in shared memory;
//   2. thread d sums digit d over the warps and publishes the tile's count of
//      d (flag AGG; tile 0 publishes it as INC, an inclusive prefix);
//   3. thread d walks back over the preceding tiles' status words of digit d,
//      LOOKBACK words per round, adding AGG counts until it meets an INC
//      prefix, then publishes its own inclusive prefix (decoupled look-back;
//      with every tile resident at once the walks are long, so a round has
//      its loads in flight together); the wait on an unpublished word is
//      bounded and reports SORT_ERR_LOOKBACK when it runs out;
//   4. keys, then values, are placed in shared memory in digit order and
//      written out by consecutive threads, so each digit's run of the tile is
//      one contiguous stretch of the output.
// A status word is 30 bits of count under 2 flag bits, written and read as
// one 32-bit word, so a reader sees either nothing or a complete entry.
#include "radix_sort.cuh"

namespace rg {
namespace {

constexpr uint32_t ST_AGG = 1u << 30, ST_INC = 2u << 30, ST_COUNT = (1u << 30) - 1u;
constexpr uint32_t LOOKBACK_SPIN_LIMIT = 1u << 21; // polls of one word (with a short sleep) before giving up
constexpr uint32_t HIST_MAX_BLOCKS = 148 * 8;
constexpr int LOOKBACK = 24; // preceding tiles read per look-back round

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t item_count(uint64_t cap, const uint32_t *n_dev) {
    return n_dev ? (uint32_t)min(cap, (uint64_t)*n_dev) : (uint32_t)cap;
}

template <typename K>
__device__ __forceinline__ uint32_t digit(K k, int shift) {
    return (uint32_t)(k >> shift) & 0xFFu;
}

// Exclusive scan of one value per thread over the block (RS_THREADS threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *s_warp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t before = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++)
        if (w < warp) before += s_warp[w];
    __syncthreads();
    return before + x - v;
}

// Digit counts of every pass in one read of the keys.
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const K *__restrict__ keys, uint64_t cap, const uint32_t *__restrict__ n_dev,
                                                        int begin_bit, int passes, uint32_t *__restrict__ ghist) {
    __shared__ uint32_t h[RS_MAX_PASSES * 256];
    for (int i = threadIdx.x; i < passes * 256; i += RS_THREADS) h[i] = 0;
    __syncthreads();
    const uint32_t n = item_count(cap, n_dev);
    for (uint32_t i = blockIdx.x * RS_THREADS + threadIdx.x; i < n; i += gridDim.x * RS_THREADS) {
        const K k = keys[i];
        for (int p = 0; p < passes; p++) atomicAdd(&h[p * 256 + digit(k, begin_bit + 8 * p)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += RS_THREADS)
        if (h[i]) atomicAdd(&ghist[i], h[i]);
}

// One digit pass. vals_in null: the values are the items' input indices.
template <typename K, int ITEMS>
__global__ void __launch_bounds__(RS_THREADS, 2) k_rs_onesweep(const K *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                                            K *__restrict__ keys_out, uint32_t *__restrict__ vals_out, uint64_t cap,
                                                            const uint32_t *__restrict__ n_dev, int shift, const uint32_t *__restrict__ ghist,
                                                            uint32_t *__restrict__ tile_counter, uint32_t *__restrict__ status,
                                                            uint32_t *__restrict__ err) {
    __shared__ uint32_t s_whist[RS_WARPS][256]; // per-warp digit counts, then the warps' exclusive offsets
    __shared__ uint32_t s_dstart[256];          // first tile position of each digit
    __shared__ uint32_t s_gofs[256];            // output index of tile position 0 of each digit
    __shared__ uint32_t s_warp[RS_WARPS];
    __shared__ uint32_t s_tile;
    __shared__ __align__(16) K s_x[(RS_THREADS * ITEMS)]; // the tile in digit order: keys, then values
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) s_tile = atomicAdd(tile_counter, 1u);
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) s_whist[w][t] = 0;
    __syncthreads();
    const uint32_t n = item_count(cap, n_dev);
    const uint32_t tile = s_tile;
    const uint64_t tile_base = (uint64_t)tile * (RS_THREADS * ITEMS);
    if (tile_base >= n) return; // past the items (block-uniform)
    const uint32_t tile_n = (uint32_t)min((uint64_t)(RS_THREADS * ITEMS), (uint64_t)n - tile_base);

    // warp w holds tile positions [w * 32 * ITEMS, (w + 1) * 32 * ITEMS), lane-striped
    const uint32_t wbase = (uint32_t)warp * 32u * ITEMS;
    K k[ITEMS];
    uint32_t v[ITEMS], pos[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        const uint32_t li = wbase + (uint32_t)j * 32u + lane;
        const bool ok = li < tile_n;
        k[j] = ok ? keys_in[tile_base + li] : (K)0;
        v[j] = ok ? (vals_in ? vals_in[tile_base + li] : (uint32_t)(tile_base + li)) : 0u;
    }
    // stable rank among the warp's keys of the same digit: the lanes of one
    // digit (a group, found with one ballot per digit bit) take their places
    // in lane order after the group's earlier keys, whose count the group's
    // lowest lane reads and advances with one shared atomic; the warp is
    // synchronised after each key, so the counts advance in key order
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        const uint32_t li = wbase + (uint32_t)j * 32u + lane;
        const bool ok = li < tile_n;
        const uint32_t d = ok ? digit(k[j], shift) : 0u;
        uint32_t peers = __ballot_sync(0xffffffffu, ok);
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const uint32_t m = __ballot_sync(0xffffffffu, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? m : ~m;
        }
        const uint32_t leader = __ffs(peers) - 1u; // invalid lanes get a group of valid lanes or none; they use nothing
        uint32_t before = 0;
        if (ok && lane == leader) before = atomicAdd(&s_whist[warp][d], (uint32_t)__popc(peers));
        before = __shfl_sync(0xffffffffu, before, ok ? leader : lane);
        pos[j] = before + __popc(peers & lt);
        __syncwarp(); // this key's atomic is done before the next key's
    }
    __syncthreads();
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) {
        const uint32_t c = s_whist[w][t];
        s_whist[w][t] = cnt;
        cnt += c;
    }
    uint32_t *mine = status + (uint64_t)tile * 256u + (uint32_t)t;
    st_relaxed(mine, (tile == 0 ? ST_INC : ST_AGG) | cnt);
    const uint32_t gstart = block_exclusive_scan(ghist[t], s_warp);
    const uint32_t dstart = block_exclusive_scan(cnt, s_warp);
    uint32_t excl = 0;
    if (tile > 0) {
        // walk back over the preceding tiles' words of digit t, LOOKBACK
        // tiles per round (independent loads in flight together), adding
        // counts until an inclusive prefix; a word not yet published is
        // polled again from there on the next round
        int32_t pred = (int32_t)tile - 1;
        uint32_t spins = 0;
        bool done = false;
        while (!done) {
            uint32_t w[LOOKBACK];
#pragma unroll
            for (int q = 0; q < LOOKBACK; q++)
                w[q] = pred - q >= 0 ? ld_relaxed(status + (uint64_t)(pred - q) * 256u + (uint32_t)t) : ST_INC;
            int used = 0;
#pragma unroll
            for (int q = 0; q < LOOKBACK; q++) {
                if (done || used < q) continue; // stopped earlier in this round
                const uint32_t s = w[q];
                if ((s & ~ST_COUNT) == 0u) continue; // unpublished: the next round starts here
                excl += s & ST_COUNT;
                used = q + 1;
                if (s & ST_INC) done = true; // tile 0 (and past it, the sentinel) is inclusive
            }
            pred -= used;
            if (!done && used == 0) {
                if (++spins > LOOKBACK_SPIN_LIMIT) {
                    if (err) atomicOr(err, SORT_ERR_LOOKBACK);
                    break;
                }
                if (spins > 8u) __nanosleep(64);
            }
        }
        st_relaxed(mine, ST_INC | ((excl + cnt) & ST_COUNT));
    }
    s_dstart[t] = dstart;
    s_gofs[t] = gstart + excl - dstart;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        const uint32_t li = wbase + (uint32_t)j * 32u + lane;
        if (li < tile_n) {
            const uint32_t d = digit(k[j], shift);
            pos[j] += s_dstart[d] + s_whist[warp][d];
            s_x[pos[j]] = k[j];
        }
    }
    __syncthreads();
    uint32_t dst[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        const uint32_t i = (uint32_t)j * RS_THREADS + (uint32_t)t;
        if (i < tile_n) {
            const K key = s_x[i];
            dst[j] = s_gofs[digit(key, shift)] + i;
            keys_out[dst[j]] = key;
        }
    }
    __syncthreads();
    uint32_t *s_v = reinterpret_cast<uint32_t *>(s_x);
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        const uint32_t li = wbase + (uint32_t)j * 32u + lane;
        if (li < tile_n) s_v[pos[j]] = v[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        const uint32_t i = (uint32_t)j * RS_THREADS + (uint32_t)t;
        if (i < tile_n) vals_out[dst[j]] = s_v[i];
    }
}

template <typename K>
__global__ void k_rs_copy(const K *__restrict__ ks, const uint32_t *__restrict__ vs, K *__restrict__ kd, uint32_t *__restrict__ vd,
                          uint64_t cap, const uint32_t *__restrict__ n_dev) {
    const uint32_t n = item_count(cap, n_dev);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        kd[i] = ks[i];
        vd[i] = vs[i];
    }
}

constexpr uint64_t kCounterWords = RS_COUNTER_WORDS; // digit counts of every pass, then the tile counters

inline uint32_t tile_count(uint64_t n) { return (uint32_t)((n + RS_TILE - 1) / RS_TILE); }
inline uint32_t *counts_of(void *scratch, uint64_t n, int key_bytes) {
    return reinterpret_cast<uint32_t *>(static_cast<char *>(scratch) + rs_align256(n * key_bytes) + rs_align256(n * 4));
}
inline cudaError_t zero_counters(void *scratch, uint64_t n, int key_bytes, int passes, cudaStream_t st) {
    return cudaMemsetAsync(counts_of(scratch, n, key_bytes), 0, (kCounterWords + (uint64_t)passes * tile_count(n) * 256) * 4, st);
}

template <typename K>
cudaError_t sort_impl(K *keys, uint32_t *vals, uint64_t n, int begin_bit, int end_bit, void *scratch, cudaStream_t st, const uint32_t *n_dev,
                      bool ident, uint32_t *err, bool counted) {
    const int passes = (end_bit - begin_bit + 7) / 8;
    if (passes < 1 || passes > (int)sizeof(K) || begin_bit < 0 || end_bit > (int)(8 * sizeof(K)) || n > RS_MAX_ITEMS)
        return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    const uint32_t num_tiles = tile_count(n);
    char *p = static_cast<char *>(scratch);
    K *keys_alt = reinterpret_cast<K *>(p);
    p += rs_align256(n * sizeof(K));
    uint32_t *vals_alt = reinterpret_cast<uint32_t *>(p);
    p += rs_align256(n * 4);
    uint32_t *ghist = reinterpret_cast<uint32_t *>(p);
    uint32_t *counters = ghist + RS_MAX_PASSES * 256;
    uint32_t *status = ghist + kCounterWords;
    if (!counted) { // else radix_sort_begin zeroed them and the key kernel counted the digits
        cudaError_t e = zero_counters(scratch, n, (int)sizeof(K), passes, st);
        if (e != cudaSuccess) return e;
        // one block per tile up to HIST_MAX_BLOCKS, each striding over the keys
        k_rs_hist<K><<<num_tiles < HIST_MAX_BLOCKS ? num_tiles : HIST_MAX_BLOCKS, RS_THREADS, 0, st>>>(keys, n, n_dev, begin_bit, passes,
                                                                                                      ghist);
    }
    K *src_k = keys, *dst_k = keys_alt;
    const uint32_t *src_v = ident ? nullptr : vals;
    uint32_t *dst_v = vals_alt;
    for (int q = 0; q < passes; q++) {
        k_rs_onesweep<K, RS_ITEMS><<<num_tiles, RS_THREADS, 0, st>>>(src_k, src_v, dst_k, dst_v, n, n_dev, begin_bit + 8 * q, ghist + 256 * q,
                                                                    counters + q, status + (uint64_t)q * num_tiles * 256, err);
        K *tk = src_k;
        src_k = dst_k;
        dst_k = tk;
        uint32_t *nv = dst_v;
        dst_v = (dst_v == vals_alt) ? vals : vals_alt;
        src_v = nv;
    }
    if (passes & 1) {
        const uint64_t want = (n + 255) / 256;
        const uint32_t blocks = (uint32_t)(want < 148 * 16 ? want : 148 * 16);
        k_rs_copy<K><<<blocks, 256, 0, st>>>(src_k, src_v, keys, vals, n, n_dev);
    }
    return cudaGetLastError();
}

} // namespace

size_t radix_sort_scratch_bytes(uint64_t n, int key_bytes) { return radix_sort_scratch_bytes_c(n, key_bytes); }

cudaError_t radix_sort_begin(void *scratch, uint64_t n, int key_bytes, int begin_bit, int end_bit, cudaStream_t st) {
    const int passes = (end_bit - begin_bit + 7) / 8;
    if (passes < 1 || passes > key_bytes || n > RS_MAX_ITEMS) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    return zero_counters(scratch, n, key_bytes, passes, st);
}

uint32_t *radix_sort_counts(void *scratch, uint64_t n, int key_bytes) { return counts_of(scratch, n, key_bytes); }

cudaError_t radix_sort_pairs(void *keys, uint32_t *vals, uint64_t n, int key_bytes, int begin_bit, int end_bit, void *scratch,
                             cudaStream_t stream, const uint32_t *n_dev, bool vals_identity, uint32_t *err, bool counted) {
    if (key_bytes == 8)
        return sort_impl<uint64_t>(static_cast<uint64_t *>(keys), vals, n, begin_bit, end_bit, scratch, stream, n_dev, vals_identity, err,
                                   counted);
    if (key_bytes == 4)
        return sort_impl<uint32_t>(static_cast<uint32_t *>(keys), vals, n, begin_bit, end_bit, scratch, stream, n_dev, vals_identity, err,
                                   counted);
    return cudaErrorInvalidValue;
}

} // namespace rg
