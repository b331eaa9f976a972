/*
 * CPU oracle (test infrastructure only) -- restates the Ray library's hot-path
 * arithmetic in plain C. Every function cites the reference lines it follows;
 * paths are relative to the SerhiiY-94/RayDemo tree. Compile with
 * -ffp-contract=off so that every product and sum is rounded on its own, as in
 * the reference build.
 */
#include "ray_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define ORC_HIT_EPS 0.000001f  /* HIT_EPS, src/Ray/internal/Core.h:46 */
#define ORC_FLT_EPS 0.0000001f /* FLT_EPS, src/Ray/internal/Core.h:47 */
#define ORC_PI 3.141592653589793238463f

/* ---------------------------------------------------------------- helpers */

/* x86 cvttss2si semantics for (int)f: NaN and out-of-range give INT_MIN.
 * The reference's (int) casts compile to that instruction; C leaves it
 * undefined, so it is spelled out here. */
static int32_t f2i_x86(float f) {
    if (f != f || f >= 2147483648.0f || f < -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)f;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

int32_t orc_hash(int32_t x) { /* CoreRef.cpp:264-270 */
    uint32_t ret = (uint32_t)x;
    ret = ((ret >> 16) ^ ret) * 0x45d9f3bu;
    ret = ((ret >> 16) ^ ret) * 0x45d9f3bu;
    ret = (ret >> 16) ^ ret;
    return (int32_t)ret;
}

float orc_construct_float(uint32_t m) { /* CoreRef.cpp:359-368 */
    m &= 0x007FFFFFu;
    m |= 0x3F800000u;
    float f;
    memcpy(&f, &m, 4);
    return f - 1.0f;
}

static float fract_pos(float v) { /* std::modf fractional part */
    float ip;
    return modff(v, &ip);
}

/* ------------------------------------------------------ triangle precompute */

static int preprocess_tri(const float *p0, const float *p1, const float *p2, orc_tri *acc) {
    /* PreprocessTri, src/Ray/internal/Core.cpp:162-214 */
    const float e0[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const float e1[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    const float n[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0]};
    int w = 2, u = 0, v = 1;
    if (fabsf(n[0]) >= fabsf(n[1]) && fabsf(n[0]) >= fabsf(n[2])) {
        w = 0; u = 1; v = 2;
    } else if (fabsf(n[1]) >= fabsf(n[0]) && fabsf(n[1]) >= fabsf(n[2])) {
        w = 1; u = 0; v = 2;
    }
    if (fabsf(n[w]) > ORC_FLT_EPS) {
        acc->nu = n[u] / n[w];
        acc->nv = n[v] / n[w];
        acc->pu = p0[u];
        acc->pv = p0[v];
        acc->np = acc->nu * acc->pu + acc->nv * acc->pv + p0[w];
        const float sign = (w == 1) ? -1.0f : 1.0f;
        acc->e0u = sign * e0[u] / n[w];
        acc->e0v = sign * e0[v] / n[w];
        acc->e1u = sign * e1[u] / n[w];
        acc->e1v = sign * e1[v] / n[w];
        acc->ci = w;
        if (fabsf(acc->nu) < 0.000001f && fabsf(acc->nv) < 0.000001f) acc->ci |= 4; /* TRI_AXIS_ALIGNED_BIT */
        if (n[w] < 0) acc->ci |= 8;                                                 /* TRI_INV_NORMAL_BIT */
        acc->mi = 0;
        acc->back_mi = 0;
        return 1;
    }
    /* InvalidTriangle, src/Ray/internal/Core.cpp:98-105 */
    acc->nu = acc->nv = acc->np = acc->pu = acc->pv = NAN;
    acc->ci = 0;
    acc->e0u = acc->e0v = acc->e1u = acc->e1v = NAN;
    acc->mi = acc->back_mi = 0xffffffffu;
    return 0;
}

int64_t orc_preprocess_tris(const float *pos, int64_t stride, const uint32_t *idx, int64_t ntris, orc_tri *out) {
    int64_t bad = 0;
    for (int64_t i = 0; i < ntris; i++) {
        const float *p0 = pos + (int64_t)idx[3 * i + 0] * stride;
        const float *p1 = pos + (int64_t)idx[3 * i + 1] * stride;
        const float *p2 = pos + (int64_t)idx[3 * i + 2] * stride;
        if (!preprocess_tri(p0, p1, p2, &out[i])) bad++;
    }
    return bad;
}

/* ------------------------------------------------------------ intersection */

/* _IntersectTri, src/Ray/internal/CoreRef.cpp:11-42, with the tie on equal t
 * resolved to the lower triangle index so the result does not depend on the
 * order in which triangles are visited. */
static inline void intersect_tri(const float *o, const float *d, const orc_tri *tri, int32_t i, orc_hit *h) {
    static const int next_u[3] = {1, 0, 0}, next_v[3] = {2, 2, 1};
    const int iw = tri->ci & 3, iu = next_u[iw], iv = next_v[iw];
    const float det = d[iu] * tri->nu + d[iv] * tri->nv + d[iw];
    const float dett = tri->np - (o[iu] * tri->nu + o[iv] * tri->nv + o[iw]);
    const float Du = d[iu] * dett - (tri->pu - o[iu]) * det;
    const float Dv = d[iv] * dett - (tri->pv - o[iv]) * det;
    const float detu = tri->e1v * Du - tri->e1u * Dv;
    const float detv = tri->e0u * Dv - tri->e0v * Du;
    const float tmpdet0 = det - detu - detv;
    if ((tmpdet0 > -ORC_HIT_EPS && detu > -ORC_HIT_EPS && detv > -ORC_HIT_EPS) ||
        (tmpdet0 < ORC_HIT_EPS && detu < ORC_HIT_EPS && detv < ORC_HIT_EPS)) {
        const float rdet = 1.0f / det;
        const float t = dett * rdet;
        const float u = detu * rdet;
        const float v = detv * rdet;
        if (t > 0 && (t < h->t || (t == h->t && h->prim >= 0 && i < h->prim))) {
            h->prim = i;
            h->t = t;
            h->u = u;
            h->v = v;
        }
    }
}

/* safe_invert, src/Ray/internal/CoreRef.cpp:272-294 */
static float safe_inv(float v) {
    float r = 1.0f / v;
    if (v <= ORC_FLT_EPS && v >= 0) r = 3.402823466e+38F;
    else if (v >= -ORC_FLT_EPS && v < 0) r = -3.402823466e+38F;
    return r;
}

/* bbox_test, src/Ray/internal/CoreRef.cpp:64-86: the instance-box test of the
 * reference's macro traversal (Traverse_MacroTree_WithStack_ClosestHit,
 * CoreRef.cpp:1133-1222), done with safe_invert'ed directions. */
static int ref_bbox_test(const float *o, const float *d, float t, const float *box) {
    const float inv_d[3] = {safe_inv(d[0]), safe_inv(d[1]), safe_inv(d[2])};
    float lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = inv_d[k] * (box[k] - o[k]);
        hi[k] = inv_d[k] * (box[3 + k] - o[k]);
        if (lo[k] > hi[k]) { const float tmp = lo[k]; lo[k] = hi[k]; hi[k] = tmp; }
    }
    float tmin = lo[0] > lo[1] ? lo[0] : lo[1];
    if (lo[2] > tmin) tmin = lo[2];
    float tmax = hi[0] < hi[1] ? hi[0] : hi[1];
    if (hi[2] < tmax) tmax = hi[2];
    tmax *= 1.00000024f;
    return tmin <= tmax && tmin <= t && tmax > 0;
}

typedef struct {
    const orc_tri *tris;
    int64_t ntris;
    const float *rays;
    orc_hit *hits;
    int64_t begin, end;
    const orc_bvh *bvh;
    const float *world_box;
} work_t;

static void *brute_worker(void *arg) {
    work_t *w = (work_t *)arg;
    for (int64_t r = w->begin; r < w->end; r++) {
        const float *ray = w->rays + 8 * r;
        orc_hit h = {-1, ray[3], 0.0f, 0.0f};
        if (!w->world_box || ref_bbox_test(ray, ray + 4, ray[3], w->world_box))
            for (int64_t i = 0; i < w->ntris; i++) intersect_tri(ray, ray + 4, &w->tris[i], (int32_t)i, &h);
        w->hits[r] = h;
    }
    return NULL;
}

static void run_parallel(void *(*fn)(void *), work_t proto, int64_t n, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    work_t w[256];
    const int64_t chunk = (n + nthreads - 1) / nthreads;
    int started = 0;
    for (int t = 0; t < nthreads; t++) {
        w[t] = proto;
        w[t].begin = t * chunk;
        w[t].end = (t + 1) * chunk < n ? (t + 1) * chunk : n;
        if (w[t].begin >= w[t].end) break;
        if (pthread_create(&th[t], NULL, fn, &w[t]) != 0) { fn(&w[t]); continue; }
        started = t + 1;
    }
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
}

void orc_closest_hit_brute(const orc_tri *tris, int64_t ntris, const float *rays, int64_t nrays, orc_hit *hits, int nthreads,
                           const float *world_box) {
    work_t proto = {tris, ntris, rays, hits, 0, 0, NULL, world_box};
    run_parallel(brute_worker, proto, nrays, nthreads);
}

/* ------------------------------------------------------------ oracle BVH */
/* A plain median-split binary BVH. Its boxes are widened outward so that the
 * traversal never culls a triangle that the brute-force loop would accept;
 * the hit it returns is therefore the brute-force one. */

typedef struct {
    float bmin[3], bmax[3];
    int32_t left, right; /* internal: children; leaf: left = first, right = -count */
} onode;

struct orc_bvh {
    onode *nodes;
    int64_t nnodes;
    uint32_t *prims;
};

static const float *g_cent; /* centroid array for the partition below */

static void swap_u32(uint32_t *a, uint32_t *b) { uint32_t t = *a; *a = *b; *b = t; }

/* quickselect so that prims[lo..mid) <= prims[mid] <= prims[mid..hi) on axis */
static void nth_element_axis(uint32_t *p, int64_t lo, int64_t hi, int64_t mid, int axis) {
    while (hi - lo > 1) {
        const float pivot = g_cent[3 * p[lo + (hi - lo) / 2] + axis];
        int64_t i = lo, j = hi - 1;
        while (i <= j) {
            while (g_cent[3 * p[i] + axis] < pivot) i++;
            while (g_cent[3 * p[j] + axis] > pivot) j--;
            if (i <= j) { swap_u32(&p[i], &p[j]); i++; j--; }
        }
        if (mid <= j) hi = j + 1;
        else if (mid >= i) lo = i;
        else return;
    }
}

static float widen_lo(float v) { return v - (fabsf(v) * 1e-5f + 1e-20f); }
static float widen_hi(float v) { return v + (fabsf(v) * 1e-5f + 1e-20f); }

orc_bvh *orc_bvh_build(const float *aabbs, int64_t n) {
    orc_bvh *b = (orc_bvh *)calloc(1, sizeof(orc_bvh));
    b->prims = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    b->nodes = (onode *)malloc(sizeof(onode) * (size_t)(2 * n + 1));
    float *cent = (float *)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) {
        b->prims[i] = (uint32_t)i;
        for (int k = 0; k < 3; k++) cent[3 * i + k] = 0.5f * (aabbs[6 * i + k] + aabbs[6 * i + 3 + k]);
    }
    g_cent = cent;
    typedef struct { int64_t node, lo, hi; } item;
    item *stack = (item *)malloc(sizeof(item) * 256);
    int sp = 0;
    b->nnodes = 1;
    stack[sp++] = (item){0, 0, n};
    while (sp) {
        item it = stack[--sp];
        onode *nd = &b->nodes[it.node];
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = it.lo; i < it.hi; i++) {
            const uint32_t p = b->prims[i];
            for (int k = 0; k < 3; k++) {
                mn[k] = fminf(mn[k], aabbs[6 * p + k]);
                mx[k] = fmaxf(mx[k], aabbs[6 * p + 3 + k]);
                cmn[k] = fminf(cmn[k], cent[3 * p + k]);
                cmx[k] = fmaxf(cmx[k], cent[3 * p + k]);
            }
        }
        for (int k = 0; k < 3; k++) {
            nd->bmin[k] = widen_lo(mn[k]);
            nd->bmax[k] = widen_hi(mx[k]);
        }
        const int64_t cnt = it.hi - it.lo;
        if (cnt <= 4 || sp >= 250) {
            nd->left = (int32_t)it.lo;
            nd->right = (int32_t)-cnt;
            continue;
        }
        int axis = 0;
        float ext = cmx[0] - cmn[0];
        for (int k = 1; k < 3; k++)
            if (cmx[k] - cmn[k] > ext) { ext = cmx[k] - cmn[k]; axis = k; }
        const int64_t mid = it.lo + cnt / 2;
        nth_element_axis(b->prims, it.lo, it.hi, mid, axis);
        nd->left = (int32_t)b->nnodes;
        nd->right = (int32_t)(b->nnodes + 1);
        b->nnodes += 2;
        stack[sp++] = (item){nd->right, mid, it.hi};
        stack[sp++] = (item){nd->left, it.lo, mid};
    }
    free(stack);
    free(cent);
    return b;
}

void orc_bvh_free(orc_bvh *b) {
    if (!b) return;
    free(b->nodes);
    free(b->prims);
    free(b);
}

static int box_hit(const onode *nd, const float *o, const float *inv_d, float tmax_ray) {
    float tmin = 0.0f, tmax = INFINITY;
    for (int k = 0; k < 3; k++) {
        const float a = (nd->bmin[k] - o[k]) * inv_d[k];
        const float c = (nd->bmax[k] - o[k]) * inv_d[k];
        const float lo = fminf(a, c), hi = fmaxf(a, c); /* NaN-dropping: unbounded */
        tmin = fmaxf(tmin, lo);
        tmax = fminf(tmax, hi);
    }
    return tmin <= tmax * 1.0001f && tmin <= tmax_ray * 1.0001f;
}

static void *bvh_worker(void *arg) {
    work_t *w = (work_t *)arg;
    const orc_bvh *b = w->bvh;
    int32_t stack[512];
    for (int64_t r = w->begin; r < w->end; r++) {
        const float *ray = w->rays + 8 * r;
        const float *o = ray, *d = ray + 4;
        const float inv_d[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
        orc_hit h = {-1, ray[3], 0.0f, 0.0f};
        int sp = 0;
        if (b->nnodes > 0 && b->nodes[0].right != 0 && (!w->world_box || ref_bbox_test(o, d, ray[3], w->world_box))) stack[sp++] = 0;
        while (sp) {
            const onode *nd = &b->nodes[stack[--sp]];
            if (!box_hit(nd, o, inv_d, h.t)) continue;
            if (nd->right <= 0) {
                for (int32_t i = 0; i < -nd->right; i++) {
                    const uint32_t p = b->prims[nd->left + i];
                    intersect_tri(o, d, &w->tris[p], (int32_t)p, &h);
                }
            } else if (sp < 510) {
                stack[sp++] = nd->right;
                stack[sp++] = nd->left;
            }
        }
        w->hits[r] = h;
    }
    return NULL;
}

void orc_closest_hit_bvh(const orc_bvh *b, const orc_tri *tris, const float *rays, int64_t nrays, orc_hit *hits, int nthreads,
                         const float *world_box) {
    work_t proto = {tris, 0, rays, hits, 0, 0, b, world_box};
    run_parallel(bvh_worker, proto, nrays, nthreads);
}

/* ------------------------------------------------------------ ray hashing */

/* Tables of src/Ray/internal/Core.cpp:106-150. The two Morton tables spread
 * the bits of their index (bit k to bit 2k, resp. 3k); the two angle tables
 * are data and have to be reproduced as they are. */
static const int8_t omega_table[33] = {15, 14, 13, 12, 12, 11, 11, 11, 10, 10, 9, 9, 9, 8, 8, 8, 8,
                                       7,  7,  7,  6,  6,  6,  5,  5,  4,  4, 4, 3, 3, 2, 1, 0};
static const int8_t phi_table[17][17] = {
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

static uint32_t spread_bits(uint32_t v, int stride) {
    uint32_t r = 0;
    for (int k = 0; k < 8; k++)
        if (v & (1u << k)) r |= 1u << (k * stride);
    return r;
}

void orc_ray_hash(const float *rays, int64_t nrays, const float root_min[3], const float cell_size[3], uint32_t *keys) {
    /* get_ray_hash, src/Ray/internal/CoreRef.cpp:316-333 */
    for (int64_t i = 0; i < nrays; i++) {
        const float *o = rays + 8 * i, *d = rays + 8 * i + 4;
        const int x = clampi(f2i_x86((o[0] - root_min[0]) / cell_size[0]), 0, 255);
        const int y = clampi(f2i_x86((o[1] - root_min[1]) / cell_size[1]), 0, 255);
        const int z = clampi(f2i_x86((o[2] - root_min[2]) / cell_size[2]), 0, 255);
        const uint32_t mx = spread_bits((uint32_t)x, 3), my = spread_bits((uint32_t)y, 3), mz = spread_bits((uint32_t)z, 3);
        const int oi = clampi(f2i_x86((1.0f + d[2]) / 0.0625f), 0, 32);
        const int pi_y = clampi(f2i_x86((1.0f + d[1]) / 0.125f), 0, 16);
        const int pi_x = clampi(f2i_x86((1.0f + d[0]) / 0.125f), 0, 16);
        const uint32_t om = spread_bits((uint32_t)omega_table[oi], 2);
        const uint32_t pm = spread_bits((uint32_t)phi_table[pi_y][pi_x], 2);
        keys[i] = (om << 25) | (pm << 24) | (my << 2) | (mz << 1) | mx;
    }
}

void orc_sort_perm(const uint32_t *keys, int64_t n, uint32_t *perm) {
    /* stable LSD radix sort, 8-bit digits (the order SortRays_CPU produces,
     * src/Ray/internal/CoreRef.cpp:335-357, 615-657) */
    uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) perm[i] = (uint32_t)i;
    uint32_t *src = perm, *dst = tmp;
    for (int shift = 0; shift < 32; shift += 8) {
        int64_t count[257];
        memset(count, 0, sizeof(count));
        for (int64_t i = 0; i < n; i++) count[((keys[src[i]] >> shift) & 0xFF) + 1]++;
        for (int b = 0; b < 256; b++) count[b + 1] += count[b];
        for (int64_t i = 0; i < n; i++) dst[count[(keys[src[i]] >> shift) & 0xFF]++] = src[i];
        uint32_t *t = src; src = dst; dst = t;
    }
    /* four passes: the result is back in perm */
    free(tmp);
}

/* ------------------------------------------------------------ camera / raygen */

static float len3(const float *v) {
    float t = 0.0f;
    t += v[0] * v[0];
    t += v[1] * v[1];
    t += v[2] * v[2];
    return sqrtf(t);
}

static void cross3(const float *a, const float *b, float *r) { /* Core.cpp:15-19 */
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

void orc_construct_camera(int filter, const float origin[3], const float fwd[3], const float up[3], float fov, float gamma,
                          float focus_distance, float focus_factor, orc_camera *cam) {
    /* ConstructCamera, src/Ray/internal/Core.cpp:856-886 (Persp) */
    float u[3] = {up[0], up[1], up[2]};
    float l2 = 0.0f;
    l2 += u[0] * u[0];
    l2 += u[1] * u[1];
    l2 += u[2] * u[2];
    if (l2 < ORC_FLT_EPS) {
        if (fabsf(fwd[1]) >= 0.999f) { u[0] = 1.0f; u[1] = 0.0f; u[2] = 0.0f; }
        else { u[0] = 0.0f; u[1] = 1.0f; u[2] = 0.0f; }
    }
    float s[3];
    cross3(fwd, u, s);
    const float ls = len3(s);
    s[0] /= ls; s[1] /= ls; s[2] /= ls;
    cross3(s, fwd, u);
    cam->filter = filter;
    cam->fov = fov;
    cam->gamma = gamma;
    cam->focus_distance = focus_distance;
    cam->focus_factor = focus_factor;
    for (int k = 0; k < 3; k++) {
        cam->origin[k] = origin[k];
        cam->fwd[k] = fwd[k];
        cam->side[k] = s[k];
        cam->up[k] = u[k];
    }
}

static void pix_dir(const orc_camera *cam, float k, float fov_k, int w, int h, float x, float y, const float *origin, float *out) {
    /* get_pix_dir lambda, src/Ray/internal/CoreRef.cpp:433-437 */
    const float p0 = 2 * fov_k * x / (float)w - fov_k;
    const float p1 = 2 * fov_k * (-y) / (float)h + fov_k;
    const float p2 = cam->focus_distance;
    float p[3], v[3];
    const float kp0 = k * p0;
    for (int i = 0; i < 3; i++) p[i] = cam->origin[i] + kp0 * cam->side[i] + p1 * cam->up[i] + p2 * cam->fwd[i];
    for (int i = 0; i < 3; i++) v[i] = p[i] - origin[i];
    const float l = len3(v);
    for (int i = 0; i < 3; i++) out[i] = v[i] / l;
}

void orc_generate_primary_rays(const orc_camera *cam, int iteration, int rx, int ry, int rw, int rh, int w, int h,
                               const float *halton, orc_ray_packet *out) {
    /* GeneratePrimaryRays, src/Ray/internal/CoreRef.cpp:427-505 */
    const float k = (float)w / (float)h;
    const float fov_k = tanf(0.5f * cam->fov * ORC_PI / 180.0f) * cam->focus_distance;
    int64_t i = 0;
    for (int y = ry; y < ry + rh; y++) {
        for (int x = rx; x < rx + rw; x++) {
            orc_ray_packet *r = &out[i++];
            const int index = y * w + x;
            const int hi = (iteration & 255) * 24;
            float _x = (float)x, _y = (float)y;
            const int32_t hv = orc_hash(index);
            const int32_t hv2 = orc_hash(hv);
            if (cam->filter == 1) { /* Tent */
                float rxv = fract_pos(halton[hi + 0] + orc_construct_float((uint32_t)hv));
                if (rxv < 0.5f) rxv = sqrtf(2.0f * rxv) - 1.0f;
                else rxv = 1.0f - sqrtf(2.0f - 2 * rxv);
                float ryv = fract_pos(halton[hi + 1] + orc_construct_float((uint32_t)hv2));
                if (ryv < 0.5f) ryv = sqrtf(2.0f * ryv) - 1.0f;
                else ryv = 1.0f - sqrtf(2.0f - 2.0f * ryv);
                _x += 0.5f + rxv;
                _y += 0.5f + ryv;
            } else {
                _x += fract_pos(halton[hi + 0] + orc_construct_float((uint32_t)hv));
                _y += fract_pos(halton[hi + 1] + orc_construct_float((uint32_t)hv2));
            }
            const float ff1 = cam->focus_factor * (-0.5f + fract_pos(halton[hi + 2] + orc_construct_float((uint32_t)hv)));
            const float ff2 = cam->focus_factor * (-0.5f + fract_pos(halton[hi + 3] + orc_construct_float((uint32_t)hv2)));
            float org[3];
            for (int j = 0; j < 3; j++) org[j] = cam->origin[j] + cam->side[j] * ff1 + cam->up[j] * ff2;
            float d[3], dx[3], dy[3];
            pix_dir(cam, k, fov_k, w, h, _x, _y, org, d);
            pix_dir(cam, k, fov_k, w, h, _x + 1, _y, org, dx);
            pix_dir(cam, k, fov_k, w, h, _x, _y + 1, org, dy);
            for (int j = 0; j < 3; j++) {
                r->o[j] = org[j];
                r->d[j] = d[j];
                r->c[j] = 1.0f;
                r->do_dx[j] = 0.0f;
                r->dd_dx[j] = dx[j] - d[j];
                r->do_dy[j] = 0.0f;
                r->dd_dy[j] = dy[j] - d[j];
            }
            r->xy = (x << 16) | y;
            r->ior = 1.0f;
            r->ray_depth = 0;
        }
    }
}

/* ------------------------------------------------------------ Halton table */

static const int g_primes[24] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89};

/* MT19937 (Matsumoto & Nishimura 1998), the engine std::mt19937 implements. */
typedef struct { uint32_t mt[624]; int idx; } mt19937;

static void mt_seed(mt19937 *g, uint32_t s) {
    g->mt[0] = s;
    for (int i = 1; i < 624; i++) g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

static uint32_t mt_next(mt19937 *g) {
    if (g->idx >= 624) {
        for (int i = 0; i < 624; i++) {
            const uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

void orc_halton_perms(uint16_t *perms) {
    /* ComputeRadicalInversePermutations + Shuffle, src/Ray/internal/Halton.h:7-43,
     * fed by uniform_int_distribution<int>() over mt19937(0)
     * (src/Ray/internal/RendererRef.cpp:11-12). For the full [0, INT_MAX]
     * range, libstdc++'s Lemire downscaling of a 32-bit engine reduces to
     * g() >> 1 (the low product word is below 2^31 only when it is 0, and the
     * rejection threshold is then 0). */
    mt19937 g;
    mt_seed(&g, 0u);
    uint16_t *p = perms;
    for (int i = 0; i < 24; i++) {
        const int count = g_primes[i];
        for (int j = 0; j < count; j++) p[j] = (uint16_t)j;
        for (int j = 0; j < count; j++) {
            const uint32_t thres = (~((uint32_t)count) + 1u) % (uint32_t)count;
            uint32_t other;
            for (;;) {
                const uint32_t r = mt_next(&g) >> 1;
                if (r >= thres) { other = r % (uint32_t)count; break; }
            }
            const uint16_t t = p[j]; p[j] = p[other]; p[other] = t;
        }
        p += count;
    }
}

static float scrambled_radical_inverse(int base, const uint16_t *perm, uint64_t a) {
    /* ScrambledRadicalInverse, src/Ray/internal/Halton.h:61-74 */
    const float inv_base = 1.0f / (float)base;
    uint64_t reversed = 0;
    float inv_base_n = 1.0f;
    while (a) {
        const uint64_t next = a / (uint64_t)base;
        const uint64_t digit = a - next * (uint64_t)base;
        reversed = reversed * (uint64_t)base + perm[digit];
        inv_base_n *= inv_base;
        a = next;
    }
    const float v = inv_base_n * ((float)reversed + inv_base * (float)perm[0] / (1.0f - inv_base));
    const float lim = 1.0f - 1.1920928955078125e-07f;
    return (lim < v) ? lim : v;
}

void orc_halton_table(int iteration, const uint16_t *perms, float *out) {
    /* UpdateHaltonSequence, src/Ray/internal/RendererRef.cpp:327-358 */
    int offs[24];
    int acc = 0;
    for (int k = 0; k < 24; k++) { offs[k] = acc; acc += g_primes[k]; }
    for (int i = 0; i < 256; i++)
        for (int k = 0; k < 24; k++)
            out[i * 24 + k] = scrambled_radical_inverse(g_primes[k], perms + offs[k], (uint64_t)(int64_t)(iteration + i));
}
