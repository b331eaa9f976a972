// GPU BVH construction (see bvh.cuh). Compiled with --fmad=false: the
// triangle precompute must round every product and sum on its own, as the
// reference build does.
//
// Pipeline for one mesh of n triangles:
//   1. k_preprocess  PreprocessTri per triangle + triangle boxes
//   2. k_bounds      centroid bounds
//   3. k_morton      63-bit Morton keys (21 bits per axis), value = triangle id
//   4. radix sort    (key, id), stable
//   5. k_karras      binary radix tree over the sorted keys (Karras 2012,
//                    duplicate keys split by index)
//   6. k_bottom_up   node boxes, leaves to root with arrival counters
//   7. k_wide_cost   bottom-up SAH cost of every binary subtree written as
//                    1..8 slots of a wide node (the dynamic programme of
//                    Ylitie, Karras and Laine 2017): a slot is a leaf (<= 3
//                    triangles) or a wide node, or the subtree is opened and
//                    its two children share the slots
//   8. k_collapse    level by level: each wide node takes the slots the
//                    programme chose for its binary node, children with
//                    <= 3 triangles become leaves, the others wide nodes of
//                    the next level; children are assigned to the 8 slots
//                    by octant so that a ray visits them roughly front to
//                    back, and their boxes are quantised to 8 bits.
#include <algorithm>
#include <vector>

#include "../../include/raygpu.h"
#include "bvh.cuh"
#include "radix_sort.cuh"

namespace rg {
namespace {

constexpr uint32_t LEAF = 0x80000000u;

__device__ __forceinline__ float comp(const float3 &v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__global__ void k_preprocess(const float *__restrict__ verts, const uint32_t *__restrict__ mat, uint32_t n, TriRec *__restrict__ out,
                             float *__restrict__ aabb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *v = verts + 9ull * i;
    const float3 p0 = make_float3(v[0], v[1], v[2]), p1 = make_float3(v[3], v[4], v[5]), p2 = make_float3(v[6], v[7], v[8]);
    // PreprocessTri, src/Ray/internal/Core.cpp:162-214
    const float3 e0 = make_float3(__fsub_rn(p1.x, p0.x), __fsub_rn(p1.y, p0.y), __fsub_rn(p1.z, p0.z));
    const float3 e1 = make_float3(__fsub_rn(p2.x, p0.x), __fsub_rn(p2.y, p0.y), __fsub_rn(p2.z, p0.z));
    const float3 nrm = make_float3(__fsub_rn(__fmul_rn(e0.y, e1.z), __fmul_rn(e0.z, e1.y)),
                                   __fsub_rn(__fmul_rn(e0.z, e1.x), __fmul_rn(e0.x, e1.z)),
                                   __fsub_rn(__fmul_rn(e0.x, e1.y), __fmul_rn(e0.y, e1.x)));
    int w = 2, u = 0, vv = 1;
    if (fabsf(nrm.x) >= fabsf(nrm.y) && fabsf(nrm.x) >= fabsf(nrm.z)) {
        w = 0; u = 1; vv = 2;
    } else if (fabsf(nrm.y) >= fabsf(nrm.x) && fabsf(nrm.y) >= fabsf(nrm.z)) {
        w = 1; u = 0; vv = 2;
    }
    TriRec t;
    const float nw = comp(nrm, w);
    if (fabsf(nw) > FLT_EPS_) {
        t.nu = __fdiv_rn(comp(nrm, u), nw);
        t.nv = __fdiv_rn(comp(nrm, vv), nw);
        t.pu = comp(p0, u);
        t.pv = comp(p0, vv);
        t.np = __fadd_rn(__fadd_rn(__fmul_rn(t.nu, t.pu), __fmul_rn(t.nv, t.pv)), comp(p0, w));
        const float sign = (w == 1) ? -1.0f : 1.0f;
        t.e0u = __fdiv_rn(__fmul_rn(sign, comp(e0, u)), nw);
        t.e0v = __fdiv_rn(__fmul_rn(sign, comp(e0, vv)), nw);
        t.e1u = __fdiv_rn(__fmul_rn(sign, comp(e1, u)), nw);
        t.e1v = __fdiv_rn(__fmul_rn(sign, comp(e1, vv)), nw);
        int ci = w;
        if (fabsf(t.nu) < 0.000001f && fabsf(t.nv) < 0.000001f) ci |= TRI_AXIS_ALIGNED_BIT;
        if (nw < 0) ci |= TRI_INV_NORMAL_BIT;
        if (mat[3ull * i + 2]) ci |= TRI_SOLID_BIT;
        t.ci = ci;
    } else {
        // InvalidTriangle (Core.cpp:98-105): never intersects
        t.nu = t.nv = t.np = t.pu = t.pv = __int_as_float(0x7fc00000);
        t.e0u = t.e0v = t.e1u = t.e1v = __int_as_float(0x7fc00000);
        t.ci = mat[3ull * i + 2] ? TRI_SOLID_BIT : 0;
    }
    t.mi = mat[3ull * i + 0];
    t.back_mi = mat[3ull * i + 1];
    out[i] = t;
    float lo[3] = {fminf(p0.x, fminf(p1.x, p2.x)), fminf(p0.y, fminf(p1.y, p2.y)), fminf(p0.z, fminf(p1.z, p2.z))};
    float hi[3] = {fmaxf(p0.x, fmaxf(p1.x, p2.x)), fmaxf(p0.y, fmaxf(p1.y, p2.y)), fmaxf(p0.z, fmaxf(p1.z, p2.z))};
    bool finite = true;
    for (int k = 0; k < 3; k++) finite = finite && isfinite(lo[k]) && isfinite(hi[k]);
    for (int k = 0; k < 3; k++) {
        aabb[6ull * i + k] = finite ? lo[k] : 0.0f;
        aabb[6ull * i + 3 + k] = finite ? hi[k] : 0.0f;
    }
}

__device__ __forceinline__ uint32_t f2ord(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ord2f(uint32_t u) {
    const uint32_t v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(v);
#else
    float f;
    memcpy(&f, &v, 4);
    return f;
#endif
}

// bounds[0..2] = ordered min of the centroids, [3..5] = ordered max
__global__ void k_bounds(const float *__restrict__ aabb, uint32_t n, uint32_t *__restrict__ bounds) {
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int k = 0; k < 3; k++) {
            const uint32_t c = f2ord(0.5f * (aabb[6ull * i + k] + aabb[6ull * i + 3 + k]));
            mn[k] = min(mn[k], c);
            mx[k] = max(mx[k], c);
        }
    }
    for (int k = 0; k < 3; k++) {
        for (int off = 16; off; off >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], off));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; k++) {
            atomicMin(&bounds[k], mn[k]);
            atomicMax(&bounds[3 + k], mx[k]);
        }
    }
}

__device__ __forceinline__ uint64_t spread21(uint64_t x) {
    x &= 0x1fffffull;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void k_morton(const float *__restrict__ aabb, uint32_t n, const uint32_t *__restrict__ bounds, uint64_t *__restrict__ keys,
                         uint32_t *__restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t code = 0;
    for (int k = 0; k < 3; k++) {
        const float lo = ord2f(bounds[k]), hi = ord2f(bounds[3 + k]);
        const float c = 0.5f * (aabb[6ull * i + k] + aabb[6ull * i + 3 + k]);
        const float ext = hi - lo;
        float f = ext > 0.0f ? (c - lo) / ext : 0.0f;
        f = fminf(fmaxf(f, 0.0f), 1.0f);
        const uint32_t q = min((uint32_t)(f * 2097152.0f), 2097151u);
        code |= spread21(q) << k;
    }
    keys[i] = code;
    vals[i] = i;
}

__device__ __forceinline__ int kdelta(const uint64_t *__restrict__ k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = k[i], b = k[j];
    if (a == b) return 64 + __clz((uint32_t)(i ^ j));
    return __clzll(a ^ b);
}

// Binary radix tree (Karras 2012): internal node i in [0, n-2]; a child id
// with the LEAF bit set is the sorted leaf j. parent[] covers 2n-1 ids
// (internal i -> i, leaf j -> n-1+j).
__global__ void k_karras(const uint64_t *__restrict__ keys, int n, uint32_t *__restrict__ left, uint32_t *__restrict__ right,
                         uint32_t *__restrict__ parent, uint32_t *__restrict__ first, uint32_t *__restrict__ last) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = kdelta(keys, n, i, i - d);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = kdelta(keys, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    const uint32_t lc = (lo == gamma) ? (LEAF | (uint32_t)gamma) : (uint32_t)gamma;
    const uint32_t rc = (hi == gamma + 1) ? (LEAF | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
    left[i] = lc;
    right[i] = rc;
    first[i] = (uint32_t)lo;
    last[i] = (uint32_t)hi;
    parent[(lc & LEAF) ? (n - 1 + (lc & ~LEAF)) : lc] = (uint32_t)i;
    parent[(rc & LEAF) ? (n - 1 + (rc & ~LEAF)) : rc] = (uint32_t)i;
}

__device__ __forceinline__ void child_box(uint32_t c, const float *__restrict__ aabb, const uint32_t *__restrict__ sorted,
                                          const float *nb, float lo[3], float hi[3]) {
    if (c & LEAF) {
        const float *b = aabb + 6ull * sorted[c & ~LEAF];
        for (int k = 0; k < 3; k++) { lo[k] = b[k]; hi[k] = b[3 + k]; }
    } else {
        for (int k = 0; k < 3; k++) { lo[k] = __ldcg(nb + 6ull * c + k); hi[k] = __ldcg(nb + 6ull * c + 3 + k); }
    }
}

__global__ void k_bottom_up(const float *__restrict__ aabb, const uint32_t *__restrict__ sorted, int n, const uint32_t *__restrict__ left,
                            const uint32_t *__restrict__ right, const uint32_t *__restrict__ parent, float *nb, uint32_t *flags) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t node = parent[n - 1 + j];
    for (int climb = 0; climb < n; climb++) { // a path to the root has fewer than n nodes
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0) return; // the sibling subtree is not done yet
        float a0[3], a1[3], b0[3], b1[3];
        child_box(left[node], aabb, sorted, nb, a0, a1);
        child_box(right[node], aabb, sorted, nb, b0, b1);
        for (int k = 0; k < 3; k++) {
            __stcg(nb + 6ull * node + k, fminf(a0[k], b0[k]));
            __stcg(nb + 6ull * node + 3 + k, fmaxf(a1[k], b1[k]));
        }
        if (node == 0) return;
        node = parent[node];
    }
}

// Instance tree nodes from the binary radix tree and its node boxes: both
// children's boxes (an instance's world box, or the child node's box) and
// ids (TLAS_LEAF | instance index, or the node index).
__global__ void k_tlas_pack(const float *__restrict__ aabb, const uint32_t *__restrict__ sorted, int n, const uint32_t *__restrict__ left,
                            const uint32_t *__restrict__ right, const float *__restrict__ nb, TlasNode *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    TlasNode t;
    for (int c = 0; c < 2; c++) {
        const uint32_t id = c == 0 ? left[i] : right[i];
        float lo[3], hi[3];
        child_box(id, aabb, sorted, nb, lo, hi);
        for (int k = 0; k < 3; k++) {
            t.lo[c][k] = lo[k];
            t.hi[c][k] = hi[k];
        }
        t.child[c] = (id & LEAF) ? (TLAS_LEAF | sorted[id & ~LEAF]) : id;
    }
    t.pad[0] = t.pad[1] = 0;
    out[i] = t;
}

// SAH weights of the cost programme: a wide node's box test and fetch, and one triangle test.
constexpr float SAH_NODE = 1.0f, SAH_TRI = 1.2f;

__device__ __forceinline__ float box_area(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// C(c, j): the cost of binary subtree c in at most j slots (a single triangle: a leaf).
__device__ __forceinline__ float slot_cost(uint32_t c, int j, const float *__restrict__ aabb, const uint32_t *__restrict__ sorted,
                                           const float *cost) {
    if (c & LEAF) {
        const float *b = aabb + 6ull * sorted[c & ~LEAF];
        const float lo[3] = {b[0], b[1], b[2]}, hi[3] = {b[3], b[4], b[5]};
        return box_area(lo, hi) * SAH_TRI;
    }
    return __ldcg(cost + 8ull * c + (j - 1));
}

// Bottom-up over the binary tree (arrival counters, after k_bottom_up): for
// every internal node, C(node, j) for j = 1..8 and its choice: j = 1 a leaf
// (<= LEAF_MAX_TRIS triangles) or a wide node (its box's area times
// SAH_NODE plus the best use of 8 slots by its children); j >= 2 the better
// of one slot and the best split of the j slots between the two children
// (dec = the left child's share, 0 for one slot). open_k: the best split of
// 8 slots when the node is opened as a wide node.
__global__ void k_wide_cost(const float *__restrict__ aabb, const uint32_t *__restrict__ sorted, int n, const uint32_t *__restrict__ left,
                            const uint32_t *__restrict__ right, const uint32_t *__restrict__ parent, const uint32_t *__restrict__ first,
                            const uint32_t *__restrict__ last, const float *__restrict__ nb, uint32_t *flags, float *cost,
                            uint8_t *dec, uint8_t *open_k) {
    const int j0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (j0 >= n) return;
    uint32_t node = parent[n - 1 + j0];
    for (int climb = 0; climb < n; climb++) {
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0) return; // the sibling subtree is not done yet
        const uint32_t l = left[node], r = right[node];
        float cl[8], cr[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            cl[k] = slot_cost(l, k + 1, aabb, sorted, cost);
            cr[k] = slot_cost(r, k + 1, aabb, sorted, cost);
        }
        float lo[3], hi[3];
        for (int k = 0; k < 3; k++) {
            lo[k] = __ldcg(nb + 6ull * node + k);
            hi[k] = __ldcg(nb + 6ull * node + 3 + k);
        }
        const float area = box_area(lo, hi);
        const uint32_t cnt = last[node] - first[node] + 1u;
        float dist[9];
        uint8_t dk[9];
        for (int j = 2; j <= 8; j++) {
            float best = INFINITY;
            uint8_t bk = 1;
            for (int k = 1; k < j; k++) {
                const float v = cl[k - 1] + cr[j - k - 1];
                if (v < best) {
                    best = v;
                    bk = (uint8_t)k;
                }
            }
            dist[j] = best;
            dk[j] = bk;
        }
        const bool as_leaf = cnt <= (uint32_t)LEAF_MAX_TRIS;
        const float c1 = as_leaf ? area * (float)cnt * SAH_TRI : area * SAH_NODE + dist[8];
        __stcg(cost + 8ull * node, c1);
        dec[8ull * node] = as_leaf ? 0 : 1;
        for (int j = 2; j <= 8; j++) {
            const bool split = dist[j] < c1;
            __stcg(cost + 8ull * node + (j - 1), split ? dist[j] : c1);
            dec[8ull * node + (j - 1)] = split ? dk[j] : 0;
        }
        open_k[node] = dk[8];
        if (node == 0) return;
        node = parent[node];
    }
}

struct QItem {
    uint32_t bin, wide, depth;
};

__device__ __forceinline__ uint32_t bin_count(uint32_t c, const uint32_t *first, const uint32_t *last) {
    return (c & LEAF) ? 1u : (last[c] - first[c] + 1u);
}

__global__ void k_collapse(const QItem *__restrict__ in, uint32_t n_in, QItem *__restrict__ out, uint32_t *__restrict__ counters,
                           const float *__restrict__ aabb, const uint32_t *__restrict__ sorted, const TriRec *__restrict__ tris_ref,
                           const uint32_t *__restrict__ left, const uint32_t *__restrict__ right, const uint32_t *__restrict__ first,
                           const uint32_t *__restrict__ last, const float *__restrict__ nb, const uint8_t *__restrict__ dec,
                           const uint8_t *__restrict__ open_k, WideNode *__restrict__ nodes, TriRec *__restrict__ leaf_tris) {
    // counters: [0] wide nodes allocated, [1] leaf triangles allocated,
    //           [2] items written to `out`, [3] maximum depth
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_in) return;
    const QItem it = in[t];
    uint32_t c[8];
    int nc;
    if (it.bin & LEAF) {
        c[0] = it.bin;
        nc = 1;
    } else {
        // the slots the cost programme chose: open it.bin into 8 slots, then
        // follow each subtree's choice for its share of them
        uint32_t sn[16];
        int sj[16], sp = 0;
        const int k0 = min(max((int)open_k[it.bin], 1), 7);
        sn[sp] = right[it.bin];
        sj[sp++] = 8 - k0;
        sn[sp] = left[it.bin];
        sj[sp++] = k0;
        nc = 0;
        while (sp > 0 && nc < 8) {
            sp--;
            const uint32_t m = sn[sp];
            const int j = sj[sp];
            const int k = (m & LEAF) || j <= 1 ? 0 : (int)dec[8ull * m + (j - 1)];
            if (k <= 0 || k >= j || sp + 2 > 16) {
                c[nc++] = m;
            } else {
                sn[sp] = right[m];
                sj[sp++] = j - k;
                sn[sp] = left[m];
                sj[sp++] = k;
            }
        }
    }
    float clo[8][3], chi[8][3];
    float nlo[3] = {INFINITY, INFINITY, INFINITY}, nhi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < nc; k++) {
        child_box(c[k], aabb, sorted, nb, clo[k], chi[k]);
        for (int a = 0; a < 3; a++) {
            nlo[a] = fminf(nlo[a], clo[k][a]);
            nhi[a] = fmaxf(nhi[a], chi[k][a]);
        }
    }
    // octant slot assignment: slot bit a set <=> child lies on the high side of axis a
    int slot_of[8];
    int child_in_slot[8];
    for (int s = 0; s < 8; s++) child_in_slot[s] = -1;
    for (int k = 0; k < 8; k++) slot_of[k] = -1;
    float ctr[3];
    for (int a = 0; a < 3; a++) ctr[a] = 0.5f * (nlo[a] + nhi[a]);
    for (int r = 0; r < nc; r++) {
        float best = -INFINITY;
        int bk = -1, bs = -1;
        for (int k = 0; k < nc; k++) {
            if (slot_of[k] >= 0) continue;
            float off[3];
            for (int a = 0; a < 3; a++) off[a] = 0.5f * (clo[k][a] + chi[k][a]) - ctr[a];
            for (int s = 0; s < 8; s++) {
                if (child_in_slot[s] >= 0) continue;
                const float sc = ((s & 1) ? off[0] : -off[0]) + ((s & 2) ? off[1] : -off[1]) + ((s & 4) ? off[2] : -off[2]);
                if (bk < 0 || sc > best) { best = sc; bk = k; bs = s; }
            }
        }
        slot_of[bk] = bs;
        child_in_slot[bs] = bk;
    }
    int n_internal = 0, n_leaf_tris = 0;
    for (int k = 0; k < nc; k++) {
        const uint32_t cnt = bin_count(c[k], first, last);
        if (cnt > (uint32_t)LEAF_MAX_TRIS) n_internal++;
        else n_leaf_tris += (int)cnt;
    }
    const uint32_t child_base = n_internal ? atomicAdd(&counters[0], (uint32_t)n_internal) : 0u;
    const uint32_t tri_base = n_leaf_tris ? atomicAdd(&counters[1], (uint32_t)n_leaf_tris) : 0u;
    WideNode nd;
    // quantisation frame per axis (exact decode, one quantum of margin)
    double qs[3], qp[3];
    for (int a = 0; a < 3; a++) {
        const float lo = nlo[a], hi = nhi[a];
        const float M = fmaxf(fabsf(lo), fabsf(hi));
        int ex = 0;
        frexpf(M, &ex);
        const int e_ulp = (M > 0.0f) ? ex - 23 : -126;
        const double ext = (double)hi - (double)lo;
        int e_ext = -126;
        if (ext > 0.0) {
            int ex2 = 0;
            frexp(ext / 252.0, &ex2);
            e_ext = ex2;
        }
        const int e = max(max(e_ulp, e_ext), -126);
        const double s = ldexp(1.0, e);
        const double p = floor((double)lo / s) * s - s;
        qs[a] = s;
        qp[a] = p;
        nd.p[a] = (float)p;
        nd.e[a] = (uint8_t)(e + 127);
    }
    nd.imask = 0;
    nd.child_base = child_base;
    nd.tri_base = tri_base;
    int rank = 0, toff = 0;
    for (int s = 0; s < 8; s++) {
        const int k = child_in_slot[s];
        if (k < 0) {
            nd.meta[s] = 0;
            for (int a = 0; a < 3; a++) { nd.qlo[a][s] = 0; nd.qhi[a][s] = 0; }
            continue;
        }
        for (int a = 0; a < 3; a++) {
            int ql = (int)floor(__dsub_rd((double)clo[k][a], qp[a]) / qs[a]) - 1;
            int qh = (int)ceil(__dsub_ru((double)chi[k][a], qp[a]) / qs[a]) + 1;
            nd.qlo[a][s] = (uint8_t)min(max(ql, 0), 255);
            nd.qhi[a][s] = (uint8_t)min(max(qh, 0), 255);
        }
        const uint32_t cnt = bin_count(c[k], first, last);
        if (cnt > (uint32_t)LEAF_MAX_TRIS) {
            nd.imask |= (uint8_t)(1u << s);
            nd.meta[s] = (uint8_t)((1u << 5) | (24u + (uint32_t)s));
            const uint32_t slot = atomicAdd(&counters[2], 1u);
            out[slot] = QItem{c[k], child_base + (uint32_t)rank, it.depth + 1};
            rank++;
        } else {
            nd.meta[s] = (uint8_t)((((1u << cnt) - 1u) << 5) | (uint32_t)toff);
            const uint32_t f = (c[k] & LEAF) ? (c[k] & ~LEAF) : first[c[k]];
            for (uint32_t j = 0; j < cnt; j++) {
                const uint32_t src = sorted[f + j];
                TriRec tr = tris_ref[src];
                tr.mi = src;
                tr.back_mi = 0;
                leaf_tris[tri_base + toff + j] = tr;
            }
            toff += (int)cnt;
        }
    }
    nodes[it.wide] = nd;
    atomicMax(&counters[3], it.depth + 1);
}

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
    return device_alloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T));
}

// Scratch allocations of one build, released when the build returns.
struct TmpAllocs {
    void *p[16] = {};
    int k = 0;
    ~TmpAllocs() {
        for (int i = 0; i < k; i++) cudaFree(p[i]);
    }
    template <typename T>
    cudaError_t get(T **ptr, size_t count) {
        cudaError_t e = dalloc(ptr, count);
        if (e == cudaSuccess) p[k++] = *ptr;
        return e;
    }
};

} // namespace

cudaError_t launch_preprocess_tris(const float *verts, const uint32_t *mat, uint32_t n, TriRec *tris_out, float *aabb_out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_preprocess<<<(n + 255) / 256, 256, 0, st>>>(verts, mat, n, tris_out, aabb_out);
    return cudaGetLastError();
}

void free_mesh_bvh(MeshBvh &b) {
    if (b.nodes) cudaFree(b.nodes);
    if (b.leaf_tris) cudaFree(b.leaf_tris);
    b.nodes = nullptr;
    b.leaf_tris = nullptr;
    b.node_count = b.tri_count = b.depth = 0;
}

int build_mesh_bvh(const TriRec *tris_ref, const float *aabb, uint32_t n, MeshBvh &out, cudaStream_t st) {
    free_mesh_bvh(out);
    if (n == 0) return RAY_OK;
    if (n > 0x7fffffffu) {
        set_error("mesh too large for the BVH builder");
        return RAY_ERR_INVALID_ARG;
    }
    TmpAllocs tmp;
    uint64_t *keys;
    uint32_t *vals, *bounds, *left, *right, *parent, *first, *last, *flags, *counters;
    float *nb, *cost;
    uint8_t *dec, *open_k;
    QItem *qa, *qb;
    void *scratch;
    const size_t ni = n > 1 ? n - 1 : 1;
    RG_CUDA_TRY(tmp.get(&keys, n));
    RG_CUDA_TRY(tmp.get(&vals, n));
    RG_CUDA_TRY(tmp.get(&bounds, 6));
    RG_CUDA_TRY(tmp.get(&left, ni));
    RG_CUDA_TRY(tmp.get(&right, ni));
    RG_CUDA_TRY(tmp.get(&parent, 2 * (size_t)n));
    RG_CUDA_TRY(tmp.get(&first, ni));
    RG_CUDA_TRY(tmp.get(&last, ni));
    RG_CUDA_TRY(tmp.get(&flags, ni));
    RG_CUDA_TRY(tmp.get(&counters, 4));
    RG_CUDA_TRY(tmp.get(&nb, 6 * ni));
    RG_CUDA_TRY(tmp.get(&cost, 8 * ni));
    RG_CUDA_TRY(tmp.get(&dec, 8 * ni));
    RG_CUDA_TRY(tmp.get(&open_k, ni));
    RG_CUDA_TRY(tmp.get(&qa, n));
    RG_CUDA_TRY(tmp.get(&qb, n));
    RG_CUDA_TRY(tmp.get(reinterpret_cast<char **>(&scratch), radix_sort_scratch_bytes(n, 8)));
    const uint32_t init_bounds[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    RG_CUDA_TRY(cudaMemcpyAsync(bounds, init_bounds, sizeof(init_bounds), cudaMemcpyHostToDevice, st));
    k_bounds<<<std::min<uint32_t>((n + 255) / 256, 1184), 256, 0, st>>>(aabb, n, bounds);
    k_morton<<<(n + 255) / 256, 256, 0, st>>>(aabb, n, bounds, keys, vals);
    RG_CUDA_TRY(cudaGetLastError());
    RG_CUDA_TRY(radix_sort_pairs(keys, vals, n, 8, 0, 64, scratch, st));
    uint32_t root_bin = LEAF | 0u;
    if (n > 1) {
        RG_CUDA_TRY(cudaMemsetAsync(flags, 0, ni * sizeof(uint32_t), st));
        k_karras<<<(uint32_t)((ni + 255) / 256), 256, 0, st>>>(keys, (int)n, left, right, parent, first, last);
        k_bottom_up<<<(n + 255) / 256, 256, 0, st>>>(aabb, vals, (int)n, left, right, parent, nb, flags);
        RG_CUDA_TRY(cudaGetLastError());
        RG_CUDA_TRY(cudaMemsetAsync(flags, 0, ni * sizeof(uint32_t), st));
        k_wide_cost<<<(n + 255) / 256, 256, 0, st>>>(aabb, vals, (int)n, left, right, parent, first, last, nb, flags, cost, dec, open_k);
        RG_CUDA_TRY(cudaGetLastError());
        root_bin = 0;
    }
    // Wide nodes <= binary internal nodes with more than LEAF_MAX_TRIS triangles + 1.
    RG_CUDA_TRY(dalloc(&out.nodes, n));
    RG_CUDA_TRY(dalloc(&out.leaf_tris, n));
    const uint32_t init_counters[4] = {1u, 0u, 0u, 0u}; // node 0 (the root) is taken
    RG_CUDA_TRY(cudaMemcpyAsync(counters, init_counters, sizeof(init_counters), cudaMemcpyHostToDevice, st));
    const QItem root{root_bin, 0u, 0u};
    RG_CUDA_TRY(cudaMemcpyAsync(qa, &root, sizeof(root), cudaMemcpyHostToDevice, st));
    uint32_t n_in = 1;
    for (int level = 0; n_in > 0; level++) {
        if (level > 200) {
            set_error("BVH collapse did not terminate");
            return RAY_ERR_CUDA;
        }
        RG_CUDA_TRY(cudaMemsetAsync(counters + 2, 0, sizeof(uint32_t), st));
        k_collapse<<<(n_in + 127) / 128, 128, 0, st>>>(qa, n_in, qb, counters, aabb, vals, tris_ref, left, right, first, last, nb, dec,
                                                      open_k, out.nodes, out.leaf_tris);
        RG_CUDA_TRY(cudaGetLastError());
        RG_CUDA_TRY(cudaMemcpyAsync(&n_in, counters + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        RG_CUDA_TRY(wait_stream(st));
        std::swap(qa, qb);
    }
    uint32_t cnt[4];
    RG_CUDA_TRY(cudaMemcpyAsync(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    float rootbox[6];
    if (n > 1) {
        RG_CUDA_TRY(cudaMemcpyAsync(rootbox, nb, sizeof(rootbox), cudaMemcpyDeviceToHost, st));
    } else {
        RG_CUDA_TRY(cudaMemcpyAsync(rootbox, aabb, sizeof(rootbox), cudaMemcpyDeviceToHost, st));
    }
    RG_CUDA_TRY(wait_stream(st));
    out.node_count = cnt[0];
    out.tri_count = cnt[1];
    out.depth = cnt[3];
    for (int k = 0; k < 3; k++) {
        out.bmin[k] = rootbox[k];
        out.bmax[k] = rootbox[3 + k];
    }
    if (out.tri_count != n) {
        set_error("BVH build lost triangles");
        return RAY_ERR_CUDA;
    }
    return RAY_OK;
}

void free_inst_tree(InstTree &t) {
    void *ps[] = {t.aabb, t.sorted, t.left, t.right, t.parent, t.first, t.last, t.nb, t.flags, t.nodes};
    for (void *p : ps)
        if (p) cudaFree(p);
    t = InstTree{};
}

int build_inst_tree(const float *boxes, uint32_t n, bool refit, InstTree &t, cudaStream_t st) {
    if (n < 2) { // one instance or none: the traversal tests it directly
        free_inst_tree(t);
        return RAY_OK;
    }
    const uint32_t ni = n - 1;
    if (!refit || t.n != n) {
        free_inst_tree(t);
        RG_CUDA_TRY(dalloc(&t.aabb, 6 * (size_t)n));
        RG_CUDA_TRY(dalloc(&t.sorted, n));
        RG_CUDA_TRY(dalloc(&t.left, ni));
        RG_CUDA_TRY(dalloc(&t.right, ni));
        RG_CUDA_TRY(dalloc(&t.parent, 2 * (size_t)n));
        RG_CUDA_TRY(dalloc(&t.first, ni));
        RG_CUDA_TRY(dalloc(&t.last, ni));
        RG_CUDA_TRY(dalloc(&t.nb, 6 * (size_t)ni));
        RG_CUDA_TRY(dalloc(&t.flags, ni));
        RG_CUDA_TRY(dalloc(&t.nodes, ni));
        TmpAllocs tmp;
        uint64_t *keys = nullptr;
        uint32_t *bounds = nullptr;
        char *scratch = nullptr;
        RG_CUDA_TRY(tmp.get(&keys, n));
        RG_CUDA_TRY(tmp.get(&bounds, 6));
        RG_CUDA_TRY(tmp.get(&scratch, radix_sort_scratch_bytes(n, 8)));
        RG_CUDA_TRY(cudaMemcpyAsync(t.aabb, boxes, 6 * sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, st));
        const uint32_t init_bounds[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        RG_CUDA_TRY(cudaMemcpyAsync(bounds, init_bounds, sizeof(init_bounds), cudaMemcpyHostToDevice, st));
        k_bounds<<<std::min<uint32_t>((n + 255) / 256, 1184), 256, 0, st>>>(t.aabb, n, bounds);
        k_morton<<<(n + 255) / 256, 256, 0, st>>>(t.aabb, n, bounds, keys, t.sorted);
        RG_CUDA_TRY(cudaGetLastError());
        RG_CUDA_TRY(radix_sort_pairs(keys, t.sorted, n, 8, 0, 64, scratch, st));
        k_karras<<<(ni + 255) / 256, 256, 0, st>>>(keys, (int)n, t.left, t.right, t.parent, t.first, t.last);
        RG_CUDA_TRY(cudaGetLastError());
        RG_CUDA_TRY(wait_stream(st)); // before the temporaries are freed
        t.n = n;
    } else {
        RG_CUDA_TRY(cudaMemcpyAsync(t.aabb, boxes, 6 * sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, st));
    }
    // node boxes bottom-up (a refit: the same topology, the instances' new boxes), then the packed nodes
    RG_CUDA_TRY(cudaMemsetAsync(t.flags, 0, ni * sizeof(uint32_t), st));
    k_bottom_up<<<(n + 255) / 256, 256, 0, st>>>(t.aabb, t.sorted, (int)n, t.left, t.right, t.parent, t.nb, t.flags);
    k_tlas_pack<<<(ni + 255) / 256, 256, 0, st>>>(t.aabb, t.sorted, (int)n, t.left, t.right, t.nb, t.nodes);
    RG_CUDA_TRY(cudaGetLastError());
    return RAY_OK;
}

} // namespace rg
