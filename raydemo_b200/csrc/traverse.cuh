// Device-side traversal shared by the trace kernels and the shading kernels:
// the instance-level test and transform, the compressed wide-BVH node step,
// the triangle test and whole-mesh traversal. See trace.cu for the design.
#pragma once

#include "trace.cuh"

namespace rg {
namespace trav {

constexpr int TRACE_BLOCK = 128;
constexpr int SMEM_STACK = 24; // entries per thread in shared memory
constexpr int LMEM_STACK = 40; // further entries in a local array (DEEP instances only)
constexpr uint32_t NO_RAY = 0xffffffffu;

// Three-input max / min (sm_100). NaN inputs are dropped, as fmaxf/fminf drop them.
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Byte k of word as the float 1 + byte * 2^-15 (0x3F80bb00): exact, one permute.
__device__ __forceinline__ float byte_to_unit(uint32_t word, uint32_t k) {
    return __uint_as_float(__byte_perm(word, 0x3F800000u, 0x7604u | (k << 4)));
}

// The reference's slab test, exactly (bbox_test, CoreRef.cpp:64-86).
__device__ __forceinline__ bool ref_bbox_test(float ox, float oy, float oz, float ix, float iy, float iz, float t, const float *bmin,
                                              const float *bmax) {
    float lo_x = __fmul_rn(ix, __fsub_rn(bmin[0], ox)), hi_x = __fmul_rn(ix, __fsub_rn(bmax[0], ox));
    if (lo_x > hi_x) { const float tmp = lo_x; lo_x = hi_x; hi_x = tmp; }
    float lo_y = __fmul_rn(iy, __fsub_rn(bmin[1], oy)), hi_y = __fmul_rn(iy, __fsub_rn(bmax[1], oy));
    if (lo_y > hi_y) { const float tmp = lo_y; lo_y = hi_y; hi_y = tmp; }
    float lo_z = __fmul_rn(iz, __fsub_rn(bmin[2], oz)), hi_z = __fmul_rn(iz, __fsub_rn(bmax[2], oz));
    if (lo_z > hi_z) { const float tmp = lo_z; lo_z = hi_z; hi_z = tmp; }
    float tmin = lo_x > lo_y ? lo_x : lo_y;
    if (lo_z > tmin) tmin = lo_z;
    float tmax = hi_x < hi_y ? hi_x : hi_y;
    if (hi_z < tmax) tmax = hi_z;
    tmax = __fmul_rn(tmax, 1.00000024f);
    return tmin <= tmax && tmin <= t && tmax > 0;
}

// The same slab test, also giving the entry distance (for visiting order).
// For a box containing another, it accepts whenever the test on the inner
// box accepts (every rounding step is monotonic), so an instance-tree node
// is never culled where the reference's test enters one of its instances.
__device__ __forceinline__ bool ref_bbox_entry(float ox, float oy, float oz, float ix, float iy, float iz, float t, const float *bmin,
                                               const float *bmax, float &tmin_out) {
    float lo_x = __fmul_rn(ix, __fsub_rn(bmin[0], ox)), hi_x = __fmul_rn(ix, __fsub_rn(bmax[0], ox));
    if (lo_x > hi_x) { const float tmp = lo_x; lo_x = hi_x; hi_x = tmp; }
    float lo_y = __fmul_rn(iy, __fsub_rn(bmin[1], oy)), hi_y = __fmul_rn(iy, __fsub_rn(bmax[1], oy));
    if (lo_y > hi_y) { const float tmp = lo_y; lo_y = hi_y; hi_y = tmp; }
    float lo_z = __fmul_rn(iz, __fsub_rn(bmin[2], oz)), hi_z = __fmul_rn(iz, __fsub_rn(bmax[2], oz));
    if (lo_z > hi_z) { const float tmp = lo_z; lo_z = hi_z; hi_z = tmp; }
    float tmin = lo_x > lo_y ? lo_x : lo_y;
    if (lo_z > tmin) tmin = lo_z;
    float tmax = hi_x < hi_y ? hi_x : hi_y;
    if (hi_z < tmax) tmax = hi_z;
    tmax = __fmul_rn(tmax, 1.00000024f);
    tmin_out = tmin;
    return tmin <= tmax && tmin <= t && tmax > 0;
}

// safe_invert, CoreRef.cpp:272-294
__device__ __forceinline__ float safe_inv(float v) {
    float r = __frcp_rn(v);
    if (v <= FLT_EPS_ && v >= 0) r = 3.402823466e+38F;
    else if (v >= -FLT_EPS_ && v < 0) r = -3.402823466e+38F;
    return r;
}

struct Best {
    float t, u, v;
    int prim, obj;
};

// Ray in the space of the instance being traversed.
struct LocalRay {
    float ox, oy, oz, dx, dy, dz, ix, iy, iz;
    uint32_t oct; // bit a set: direction negative on axis a
};

struct MeshRef {
    const WideNode *nodes;
    const TriRec *tris;
    uint32_t prim_base, node_count, tri_count;
    int obj;
};

// Per-thread stack of node groups: entry k of this thread at
// smem[k * STRIDE] (STRIDE = the block's thread count), DEPTH entries in
// shared memory; the DEEP variant continues it in a local array, to
// SMEM_STACK + LMEM_STACK entries in all.
template <bool DEEP, int STRIDE = TRACE_BLOCK, int DEPTH = SMEM_STACK>
struct Stack;

template <int STRIDE, int DEPTH>
struct Stack<false, STRIDE, DEPTH> {
    uint2 *smem;
    int sp;
    __device__ __forceinline__ bool push(uint2 e) {
        if (sp >= DEPTH) return false;
        smem[sp * STRIDE] = e;
        sp++;
        return true;
    }
    __device__ __forceinline__ uint2 pop() {
        sp--;
        return smem[sp * STRIDE];
    }
};

template <int STRIDE, int DEPTH>
struct Stack<true, STRIDE, DEPTH> {
    static constexpr int LOCAL = SMEM_STACK + LMEM_STACK - DEPTH;
    uint2 *smem;
    uint2 lmem[LOCAL];
    int sp;
    __device__ __forceinline__ bool push(uint2 e) {
        if (sp >= DEPTH + LOCAL) return false;
        if (sp < DEPTH) smem[sp * STRIDE] = e;
        else lmem[sp - DEPTH] = e;
        sp++;
        return true;
    }
    __device__ __forceinline__ uint2 pop() {
        sp--;
        return sp < DEPTH ? smem[sp * STRIDE] : lmem[sp - DEPTH];
    }
};

__device__ __forceinline__ LocalRay make_local_ray(float ox, float oy, float oz, float dx, float dy, float dz) {
    LocalRay r;
    r.ox = ox; r.oy = oy; r.oz = oz;
    r.dx = dx; r.dy = dy; r.dz = dz;
    r.ix = __frcp_rn(dx); // 1.0f / d, CoreRef.cpp:1215
    r.iy = __frcp_rn(dy);
    r.iz = __frcp_rn(dz);
    r.oct = (r.ix < 0.0f ? 1u : 0u) | (r.iy < 0.0f ? 2u : 0u) | (r.iz < 0.0f ? 4u : 0u);
    return r;
}

// TransformRay, CoreRef.cpp:1605-1617, with the instance's inverse transform.
__device__ __forceinline__ LocalRay transform_ray(const InstanceRec *ir, float4 r0, float4 r1) {
    float x[12];
#pragma unroll
    for (int k = 0; k < 12; k++) x[k] = __ldg(&ir->inv_xform[k]);
    const float tox = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x[0], r0.x), __fmul_rn(x[3], r0.y)), __fmul_rn(x[6], r0.z)), x[9]);
    const float toy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x[1], r0.x), __fmul_rn(x[4], r0.y)), __fmul_rn(x[7], r0.z)), x[10]);
    const float toz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x[2], r0.x), __fmul_rn(x[5], r0.y)), __fmul_rn(x[8], r0.z)), x[11]);
    const float tdx = __fadd_rn(__fadd_rn(__fmul_rn(x[0], r1.x), __fmul_rn(x[3], r1.y)), __fmul_rn(x[6], r1.z));
    const float tdy = __fadd_rn(__fadd_rn(__fmul_rn(x[1], r1.x), __fmul_rn(x[4], r1.y)), __fmul_rn(x[7], r1.z));
    const float tdz = __fadd_rn(__fadd_rn(__fmul_rn(x[2], r1.x), __fmul_rn(x[5], r1.y)), __fmul_rn(x[8], r1.z));
    return make_local_ray(tox, toy, toz, tdx, tdy, tdz);
}

__device__ __forceinline__ MeshRef mesh_of(const SceneView &sv, const InstanceRec *ir, int m) {
    MeshRef mr;
    mr.nodes = sv.nodes + __ldg(&ir->node_base);
    mr.tris = sv.leaf_tris + __ldg(&ir->tri_base);
    mr.prim_base = __ldg(&ir->prim_base);
    mr.node_count = __ldg(&ir->node_count);
    mr.tri_count = __ldg(&ir->tri_count);
    mr.obj = m;
    return mr;
}

// Instance-tree walk, one ray: pops entries of the ray's instance stack
// (stk, sp) until an instance whose world box the ray enters with the
// current best t -- the reference's instance test, bbox_test with the
// safe-inverted direction -- and returns its index; -1 when the walk is
// done. An internal node pushes the children whose boxes the ray enters,
// the nearer on top; an instance pushed this way is tested again when popped
// (best t may have shrunk). Indices outside the tree and a full stack set
// TRACE_ERR_TLAS (the walk goes on without the entry).
constexpr int TLAS_STACK = 48;
__device__ __forceinline__ int tlas_next(const SceneView &sv, float4 r0, float sx, float sy, float sz, float best_t, uint32_t *stk, int &sp,
                                         uint32_t &err) {
    while (sp > 0) {
        const uint32_t e = stk[--sp];
        if (e & TLAS_LEAF) {
            const uint32_t m = e & ~TLAS_LEAF;
            if (m >= sv.n_inst) {
                err |= TRACE_ERR_TLAS;
                continue;
            }
            const InstanceRec *ir = sv.inst + m;
            float bmin[3], bmax[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                bmin[k] = __ldg(&ir->bbox_min[k]);
                bmax[k] = __ldg(&ir->bbox_max[k]);
            }
            if (ref_bbox_test(r0.x, r0.y, r0.z, sx, sy, sz, best_t, bmin, bmax)) return (int)m;
            continue;
        }
        if (e + 1 >= sv.n_inst) {
            err |= TRACE_ERR_TLAS;
            continue;
        }
        const float4 *np = reinterpret_cast<const float4 *>(sv.tlas + e);
        const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
        const uint4 ids = __ldg(reinterpret_cast<const uint4 *>(np + 3));
        const float lo0[3] = {a.x, a.y, a.z}, lo1[3] = {a.w, b.x, b.y}, hi0[3] = {b.z, b.w, c.x}, hi1[3] = {c.y, c.z, c.w};
        float t0 = 0.0f, t1 = 0.0f;
        const bool h0 = ref_bbox_entry(r0.x, r0.y, r0.z, sx, sy, sz, best_t, lo0, hi0, t0);
        const bool h1 = ref_bbox_entry(r0.x, r0.y, r0.z, sx, sy, sz, best_t, lo1, hi1, t1);
        const bool near1 = h1 && (!h0 || t1 < t0); // child 1 first when it is the nearer (or the only) one
        const uint32_t first = near1 ? ids.y : ids.x, second = near1 ? ids.x : ids.y;
        const bool has_second = h0 && h1;
        if (has_second) {
            if (sp < TLAS_STACK) stk[sp++] = second;
            else err |= TRACE_ERR_TLAS;
        }
        if (h0 || h1) {
            if (sp < TLAS_STACK) stk[sp++] = first;
            else err |= TRACE_ERR_TLAS;
        }
    }
    return -1;
}

// Node step: takes the next child of node group (ng_base, ng_bits), tests
// its 8 children and returns their hits as a node group (internal children,
// bits 24..31, with the node's imask in bits 0..7) and a triangle group
// (bits 0..23). Returns false (and sets err) on a corrupt index.
template <bool COUNT, typename ST>
__device__ __forceinline__ bool node_step(const MeshRef &mr, const LocalRay &r, float best_t, uint32_t &ng_base, uint32_t &ng_bits,
                                          uint32_t &tg_base, uint32_t &tg_bits, ST &st, uint32_t &visits, uint32_t &err,
                                          uint32_t &nvis) {
    const uint32_t j = __ffs(ng_bits >> 24) - 1;
    ng_bits &= ~(1u << (24 + j));
    const uint32_t s = j ^ r.oct;
    const uint32_t ni = ng_base + __popc((ng_bits & 0xFFu) & ((1u << s) - 1u));
    if (ng_bits > 0x00FFFFFFu && !st.push(make_uint2(ng_base, ng_bits))) {
        err |= TRACE_ERR_STACK;
        return false;
    }
    // A tree visits each node at most once; a bad index or a longer walk
    // means a corrupt structure: flag it and stop this ray.
    if (ni >= mr.node_count || ++visits > mr.node_count) {
        err |= (ni >= mr.node_count) ? TRACE_ERR_BOUNDS : TRACE_ERR_LIMIT;
        return false;
    }
    const uint4 *np = reinterpret_cast<const uint4 *>(mr.nodes + ni);
    const uint4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
    if (COUNT) nvis++;
    const uint32_t imask = w0.w >> 24;
    // Slab parameter of plane q on one axis: t(q) = q * A + B with
    // A = 2^e * inv_d (exact: a power-of-two scaling) and B = (p - o) * inv_d.
    // It is evaluated as one FMA on the byte read as the float
    // v = 1 + q * 2^-15: t = v * (2^15 A) + (B - 2^15 A), where 2^15 A is
    // exact and v * 2^15 A = 2^15 A + q A exactly inside the FMA. Rounding
    // B - 2^15 A, then -/+ slack, then the FMA's result errs by less than
    // 3u(|B| + 33024|A|) (u = 2^-24); the slack 2^-21 (|B| + 33024|A|)
    // moves the near planes down and the far planes up by more than that,
    // so the test accepts every box that the exact slab test on the decoded
    // box accepts. (An overflowing 2^15 A gives NaN planes: that axis is
    // left unbounded, still conservative.)
    float A[3], Bn[3], Bf[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float p = __uint_as_float(a == 0 ? w0.x : (a == 1 ? w0.y : w0.z));
        const float sc = __uint_as_float(((w0.w >> (8 * a)) & 0xFFu) << 23);
        const float inv = a == 0 ? r.ix : (a == 1 ? r.iy : r.iz);
        const float o = a == 0 ? r.ox : (a == 1 ? r.oy : r.oz);
        const float Aa = __fmul_rn(sc, inv);
        const float B = __fmul_rn(__fsub_rn(p, o), inv);
        const float slack = __fmul_rn(__fmaf_rn(fabsf(Aa), 33024.0f, fabsf(B)), 4.76837158203125e-07f);
        const float B0 = __fmaf_rn(-32768.0f, Aa, B);
        A[a] = __fmul_rn(Aa, 32768.0f);
        Bn[a] = __fsub_rn(B0, slack);
        Bf[a] = __fadd_rn(B0, slack);
    }
    // Near/far plane words by direction sign, so that a NaN slab value
    // (origin on a plane of a box the ray runs parallel to) leaves that axis
    // unbounded, which keeps the test conservative. Planes: lo x = w2.xy,
    // lo y = w2.zw, lo z = w3.xy, hi x = w3.zw, hi y = w4.xy, hi z = w4.zw.
    const bool nx = r.oct & 1u, ny = r.oct & 2u, nz = r.oct & 4u;
    const uint32_t nxa = nx ? w3.z : w2.x, nxb = nx ? w3.w : w2.y, fxa = nx ? w2.x : w3.z, fxb = nx ? w2.y : w3.w;
    const uint32_t nya = ny ? w4.x : w2.z, nyb = ny ? w4.y : w2.w, fya = ny ? w2.z : w4.x, fyb = ny ? w2.w : w4.y;
    const uint32_t nza = nz ? w4.z : w3.x, nzb = nz ? w4.w : w3.y, fza = nz ? w3.x : w4.z, fzb = nz ? w3.y : w4.w;
    uint32_t hit8 = 0; // slots whose box the ray enters
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const uint32_t k = (uint32_t)(c & 3);
        const float tnx = __fmaf_rn(byte_to_unit(c < 4 ? nxa : nxb, k), A[0], Bn[0]);
        const float tfx = __fmaf_rn(byte_to_unit(c < 4 ? fxa : fxb, k), A[0], Bf[0]);
        const float tny = __fmaf_rn(byte_to_unit(c < 4 ? nya : nyb, k), A[1], Bn[1]);
        const float tfy = __fmaf_rn(byte_to_unit(c < 4 ? fya : fyb, k), A[1], Bf[1]);
        const float tnz = __fmaf_rn(byte_to_unit(c < 4 ? nza : nzb, k), A[2], Bn[2]);
        const float tfz = __fmaf_rn(byte_to_unit(c < 4 ? fza : fzb, k), A[2], Bf[2]);
        // [max(near planes, 0), min(far planes, best_t)] non-empty: the slab
        // test with the ray's interval folded in (best_t >= 0)
        const float tmin = max3f(tnx, tny, fmaxf(tnz, 0.0f));
        const float tmax = min3f(tfx, tfy, fminf(tfz, best_t));
        if (tmin <= tmax) hit8 |= 1u << c;
    }
    // internal children: bit 24 + (slot ^ octant), so that the node group
    // is taken in the ray's octant order
    uint32_t inner = hit8 & imask;
    if (r.oct & 1u) inner = ((inner & 0x55u) << 1) | ((inner >> 1) & 0x55u);
    if (r.oct & 2u) inner = ((inner & 0x33u) << 2) | ((inner >> 2) & 0x33u);
    if (r.oct & 4u) inner = ((inner & 0x0Fu) << 4) | ((inner >> 4) & 0x0Fu);
    uint32_t hitmask = inner << 24;
    // leaf children: their triangle bits (an empty slot has meta 0 and adds nothing)
    for (uint32_t lv = hit8 & ~imask; lv; lv &= lv - 1u) {
        const uint32_t sl = __ffs(lv) - 1u;
        const uint32_t meta = ((sl < 4u ? w1.z : w1.w) >> (8u * (sl & 3u))) & 0xFFu;
        hitmask |= (meta >> 5) << (meta & 31u);
    }
    ng_base = w1.x;
    ng_bits = (hitmask & 0xFF000000u) | imask;
    tg_base = w1.y;
    tg_bits = hitmask & 0x00FFFFFFu;
    return true;
}

// The reference's triangle arithmetic (_IntersectTri, CoreRef.cpp:18-40) on
// one precomputed record (t0, t1, t2) and a ray given by origin and
// direction: true when the ray's line passes the edge tests; then
// t = dett / det, u = detu / det and v = detv / det, each as the product with
// the correctly rounded reciprocal rdet, as the reference computes them.
__device__ __forceinline__ bool tri_core(const float4 &t0, const float4 &t1, const float4 &t2, float ox, float oy, float oz, float dx,
                                         float dy, float dz, float &rdet, float &dett, float &detu, float &detv) {
    const float nu = t0.x, nv = t0.y, npl = t0.z, pu = t0.w, pv = t1.x, e0u = t1.z, e0v = t1.w, e1u = t2.x, e1v = t2.y;
    const int iw = __float_as_int(t1.y) & TRI_W_BITS;
    const float du = iw == 0 ? dy : dx, dv = iw == 2 ? dy : dz, dw = iw == 0 ? dx : (iw == 1 ? dy : dz);
    const float ou = iw == 0 ? oy : ox, ov = iw == 2 ? oy : oz, ow = iw == 0 ? ox : (iw == 1 ? oy : oz);
    const float det = __fadd_rn(__fadd_rn(__fmul_rn(du, nu), __fmul_rn(dv, nv)), dw);
    dett = __fsub_rn(npl, __fadd_rn(__fadd_rn(__fmul_rn(ou, nu), __fmul_rn(ov, nv)), ow));
    const float Du = __fsub_rn(__fmul_rn(du, dett), __fmul_rn(__fsub_rn(pu, ou), det));
    const float Dv = __fsub_rn(__fmul_rn(dv, dett), __fmul_rn(__fsub_rn(pv, ov), det));
    detu = __fsub_rn(__fmul_rn(e1v, Du), __fmul_rn(e1u, Dv));
    detv = __fsub_rn(__fmul_rn(e0u, Dv), __fmul_rn(e0v, Du));
    const float tmpdet0 = __fsub_rn(__fsub_rn(det, detu), detv);
    if ((tmpdet0 > -HIT_EPS && detu > -HIT_EPS && detv > -HIT_EPS) || (tmpdet0 < HIT_EPS && detu < HIT_EPS && detv < HIT_EPS)) {
        rdet = __frcp_rn(det); // 1.0f / det, correctly rounded
        return true;
    }
    return false;
}

// One triangle test; updates best when it is the closer hit. With SOLID,
// returns whether that hit is on a solid triangle (TRI_SOLID_BIT), which ends
// a shadow ray's search (IntersectTris_AnyHit, CoreRef.cpp:804-829).
template <bool COUNT, bool SOLID = false>
__device__ __forceinline__ bool tri_test(const MeshRef &mr, const LocalRay &r, uint32_t li, Best &best, uint32_t &err, uint32_t &ntri) {
    if (li >= mr.tri_count) {
        err |= TRACE_ERR_BOUNDS;
        return false;
    }
    const float4 *tp = reinterpret_cast<const float4 *>(mr.tris + li);
    const float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
    if (COUNT) ntri++;
    float rdet, dett, detu, detv;
    if (tri_core(t0, t1, t2, r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, rdet, dett, detu, detv)) {
        const float t = __fmul_rn(dett, rdet);
        const int gp = (int)(mr.prim_base + __float_as_uint(t2.z));
        if (t > 0.0f && (t < best.t || (t == best.t && best.prim >= 0 && gp < best.prim))) {
            best.t = t;
            best.u = __fmul_rn(detu, rdet);
            best.v = __fmul_rn(detv, rdet);
            best.prim = gp;
            best.obj = mr.obj;
            if (SOLID) return (__float_as_int(t1.y) & TRI_SOLID_BIT) != 0;
        }
    }
    return false;
}

// Whole traversal of one mesh for one ray (the one-thread-per-ray kernel).
// The current node group always has a child left at the top of the loop: the
// root's, then the group a node step returns or one taken from the stack.
template <bool COUNT, typename ST>
__device__ __forceinline__ void trace_mesh(const MeshRef &mr, const LocalRay &r, Best &best, ST &st, uint32_t &err,
                                           uint32_t &nvis, uint32_t &ntri) {
    uint32_t ng_base = 0, ng_bits = (1u << (24 + r.oct)) | 1u; // the root as slot 0 of a virtual parent
    uint32_t tg_base = 0, tg_bits = 0, visits = 0;
    st.sp = 0;
    while (true) {
        if (!node_step<COUNT>(mr, r, best.t, ng_base, ng_bits, tg_base, tg_bits, st, visits, err, nvis)) return;
        while (tg_bits) {
            const uint32_t k = __ffs(tg_bits) - 1;
            tg_bits &= tg_bits - 1;
            tri_test<COUNT>(mr, r, tg_base + k, best, err, ntri);
        }
        if (ng_bits <= 0x00FFFFFFu) {
            if (st.sp == 0) return;
            const uint2 e = st.pop();
            ng_base = e.x;
            ng_bits = e.y;
        }
    }
}

// Shadow-ray traversal of one mesh (Traverse_MicroTree_WithStack_AnyHit,
// CoreRef.cpp:1470-1577): closest-hit order, stopping at the first accepted
// hit on a solid triangle. Returns true when it stopped there.
template <typename ST>
__device__ __forceinline__ bool trace_mesh_any(const MeshRef &mr, const LocalRay &r, Best &best, ST &st, uint32_t &err) {
    uint32_t ng_base = 0, ng_bits = (1u << (24 + r.oct)) | 1u;
    uint32_t tg_base = 0, tg_bits = 0, visits = 0, nvis = 0, ntri = 0;
    st.sp = 0;
    while (true) {
        if (!node_step<false>(mr, r, best.t, ng_base, ng_bits, tg_base, tg_bits, st, visits, err, nvis)) return false;
        while (tg_bits) {
            const uint32_t k = __ffs(tg_bits) - 1;
            tg_bits &= tg_bits - 1;
            if (tri_test<false, true>(mr, r, tg_base + k, best, err, ntri)) return true;
        }
        if (ng_bits <= 0x00FFFFFFu) {
            if (st.sp == 0) return false;
            const uint2 e = st.pop();
            ng_base = e.x;
            ng_bits = e.y;
        }
    }
}

} // namespace trav
} // namespace rg
