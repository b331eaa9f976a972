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

/* ------------------------------------------------ metallic-roughness material
 * CPU restatement of the library's RAY_MAT_PRINCIPLED path (no counterpart in
 * the reference): raydemo_b200/csrc/ggx.cuh and the RAY_MAT_PRINCIPLED branch
 * of shade_hit / shade_surface in raydemo_b200/csrc/render_kernels.cu, written
 * again from the same formulas in the same operation order. cos, sin, acos and
 * pow are evaluated in double and rounded once to float, as on the GPU. */

typedef struct { float x, y, z; } pv3;
static pv3 P3(float x, float y, float z) { pv3 r = {x, y, z}; return r; }
static pv3 padd(pv3 a, pv3 b) { return P3(a.x + b.x, a.y + b.y, a.z + b.z); }
static pv3 psub(pv3 a, pv3 b) { return P3(a.x - b.x, a.y - b.y, a.z - b.z); }
static pv3 pmul(pv3 a, pv3 b) { return P3(a.x * b.x, a.y * b.y, a.z * b.z); }
static pv3 pscale(pv3 a, float s) { return P3(a.x * s, a.y * s, a.z * s); }
static pv3 pdiv(pv3 a, float s) { return P3(a.x / s, a.y / s, a.z / s); }
static float pdot(pv3 a, pv3 b) {
    float r = 0.0f;
    r += a.x * b.x;
    r += a.y * b.y;
    r += a.z * b.z;
    return r;
}
static pv3 pnorm(pv3 a) { return pdiv(a, sqrtf(pdot(a, a))); }
static pv3 pcross(pv3 a, pv3 b) { return P3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static float fmax_s(float a, float b) { return (a < b) ? b : a; }
static float clamp_s(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static float cr_cosf(float x) { return (float)cos((double)x); }
static float cr_sinf(float x) { return (float)sin((double)x); }
static float cr_acosf(float x) { return (float)acos((double)x); }
static float cr_powf(float x, float y) { return (float)pow((double)x, (double)y); }
static float pow5f(float v) { return (v * v) * (v * v) * v; }
static float simd_floorf(float v) { return (float)(int32_t)((uint32_t)f2i_x86(v) - (v < 0.0f ? 1u : 0u)); }

static uint32_t brev32(uint32_t x) {
    uint32_t r = 0;
    for (int i = 0; i < 32; i++) r |= ((x >> i) & 1u) << (31 - i);
    return r;
}
static uint32_t mix32(uint32_t x) { return (uint32_t)orc_hash((int32_t)x); }
static uint32_t nested_scramble(uint32_t x, uint32_t seed) {
    x = brev32(x);
    x += seed;
    x ^= x * 0x9E3779B8u;
    x ^= x * 0x7F4A7C16u;
    x ^= x * 0x94D049BAu;
    x ^= x * 0x2C1B3C6Eu;
    return brev32(x);
}
static uint32_t sobol_dim1(uint32_t i) {
    uint32_t r = 0, v = 0x80000000u;
    for (; i; i >>= 1, v ^= v >> 1)
        if (i & 1u) r ^= v;
    return r;
}
static void sobol2(uint32_t index, uint32_t seed, float *x, float *y) {
    const uint32_t i = nested_scramble(index, seed);
    const uint32_t sx = nested_scramble(brev32(i), mix32(seed ^ 0x5bd1e995u));
    const uint32_t sy = nested_scramble(sobol_dim1(i), mix32(seed ^ 0x1b873593u));
    *x = (float)(sx >> 8) * (1.0f / 16777216.0f);
    *y = (float)(sy >> 8) * (1.0f / 16777216.0f);
}
static uint32_t dim_seed(uint32_t pixel, int bounce, int pair) {
    return mix32(mix32(pixel * 0x2545F491u + 0x68E31DA4u) ^ (uint32_t)(bounce * 8 + pair) * 0x9E3779B1u);
}

typedef struct { pv3 t, b, n; } pframe;
static pframe make_frame(pv3 n) {
    const float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    pframe f;
    f.t = P3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    f.b = P3(b, sign + n.y * n.y * a, -n.y);
    f.n = n;
    return f;
}
static pv3 to_local(const pframe *f, pv3 v) { return P3(pdot(v, f->t), pdot(v, f->b), pdot(v, f->n)); }
static pv3 to_world(const pframe *f, pv3 v) { return padd(padd(pscale(f->t, v.x), pscale(f->b, v.y)), pscale(f->n, v.z)); }

typedef struct { pv3 f0, diffuse; float alpha, p_spec; } pparams;
static pparams make_params(pv3 base, float roughness, float metallic) {
    pparams p;
    p.f0 = P3(0.04f + (base.x - 0.04f) * metallic, 0.04f + (base.y - 0.04f) * metallic, 0.04f + (base.z - 0.04f) * metallic);
    p.diffuse = pscale(base, 1.0f - metallic);
    p.alpha = fmax_s(roughness * roughness, 1.0e-4f);
    p.p_spec = 0.5f + 0.5f * metallic;
    return p;
}
static float smith_lambda(pv3 v, float a) {
    const float t2 = (v.x * v.x + v.y * v.y) / (v.z * v.z);
    return 0.5f * (sqrtf(1.0f + a * a * t2) - 1.0f);
}
static float ggx_d(pv3 h, float a) {
    const float a2 = a * a;
    const float k = h.z * h.z * (a2 - 1.0f) + 1.0f;
    return a2 / (ORC_PI * k * k);
}
#define ORC_INV_PI 0.318309886183790671538f
static void ggx_eval(const pparams *p, pv3 wo, pv3 wi, pv3 *f_cos, float *pdf) {
    *f_cos = P3(0.0f, 0.0f, 0.0f);
    *pdf = 0.0f;
    if (wo.z <= 0.0f || wi.z <= 0.0f) return;
    const pv3 h = pnorm(padd(wo, wi));
    const float d = ggx_d(h, p->alpha);
    const float lo = smith_lambda(wo, p->alpha), li = smith_lambda(wi, p->alpha);
    const float g2 = 1.0f / (1.0f + lo + li);
    const float g1 = 1.0f / (1.0f + lo);
    const float c = 1.0f - fmax_s(pdot(wo, h), 0.0f);
    const float c5 = pow5f(c);
    const pv3 F = P3(p->f0.x + (1.0f - p->f0.x) * c5, p->f0.y + (1.0f - p->f0.y) * c5, p->f0.z + (1.0f - p->f0.z) * c5);
    const float spec = d * g2 / (4.0f * wo.z * wi.z);
    *f_cos = pscale(padd(pscale(F, spec), pscale(p->diffuse, ORC_INV_PI)), wi.z);
    const float pdf_spec = g1 * d / (4.0f * wo.z);
    const float pdf_diff = wi.z * ORC_INV_PI;
    *pdf = p->p_spec * pdf_spec + (1.0f - p->p_spec) * pdf_diff;
}
static int ggx_sample(const pparams *p, pv3 wo, float u1, float u2, float ulobe, pv3 *wi) {
    if (ulobe < p->p_spec) {
        const float a = p->alpha;
        const pv3 vh = pnorm(P3(a * wo.x, a * wo.y, wo.z));
        const float lensq = vh.x * vh.x + vh.y * vh.y;
        const pv3 t1 = lensq > 0.0f ? pdiv(P3(-vh.y, vh.x, 0.0f), sqrtf(lensq)) : P3(1.0f, 0.0f, 0.0f);
        const pv3 t2 = pcross(vh, t1);
        const float r = sqrtf(u1);
        const float phi = 2.0f * ORC_PI * u2;
        const float q1 = r * cr_cosf(phi);
        float q2 = r * cr_sinf(phi);
        const float s = 0.5f * (1.0f + vh.z);
        q2 = (1.0f - s) * sqrtf(1.0f - q1 * q1) + s * q2;
        const pv3 nh = padd(padd(pscale(t1, q1), pscale(t2, q2)), pscale(vh, sqrtf(fmax_s(0.0f, 1.0f - q1 * q1 - q2 * q2))));
        const pv3 h = pnorm(P3(a * nh.x, a * nh.y, fmax_s(0.0f, nh.z)));
        *wi = psub(pscale(h, 2.0f * pdot(wo, h)), wo);
    } else {
        const float r = sqrtf(u1);
        const float phi = 2.0f * ORC_PI * u2;
        *wi = P3(r * cr_cosf(phi), r * cr_sinf(phi), sqrtf(fmax_s(0.0f, 1.0f - u1)));
    }
    return wi->z > 0.0f;
}
static float power_heuristic(float a, float b) { return (a * a) / (a * a + b * b); }

/* the AreaLight record (20 floats) */
typedef struct { float p0[3]; uint32_t type; float u[3], area; float v[3], cos_max; float n[3], pad0; float L[3], pad1; } plight;
#define ORC_LIGHT_QUAD 3u
static int hit_quad(const plight *l, pv3 o, pv3 d, float tmax, float *t) {
    const pv3 n = P3(l->n[0], l->n[1], l->n[2]);
    const float dn = pdot(d, n);
    if (!(dn < 0.0f)) return 0;
    const pv3 p0 = P3(l->p0[0], l->p0[1], l->p0[2]);
    *t = pdot(psub(p0, o), n) / dn;
    if (!(*t > 0.0f && *t < tmax)) return 0;
    const pv3 q = psub(padd(o, pscale(d, *t)), p0);
    const pv3 u = P3(l->u[0], l->u[1], l->u[2]), v = P3(l->v[0], l->v[1], l->v[2]);
    const float s = pdot(q, u) / pdot(u, u), r = pdot(q, v) / pdot(v, v);
    return s >= 0.0f && s <= 1.0f && r >= 0.0f && r <= 1.0f;
}

/* InverseMatrix (src/Ray/internal/Core.cpp:909-949): the cofactor inverse of
 * a column-major 4x4 matrix, every product and difference in the order the
 * reference evaluates them. */
static float mdet2(const float *m, int a, int b, int c, int d) { return m[a] * m[b] - m[c] * m[d]; }
static void inverse4(const float m[16], float o[16]) {
    const float A2323 = mdet2(m, 10, 15, 11, 14), A1323 = mdet2(m, 9, 15, 11, 13), A1223 = mdet2(m, 9, 14, 10, 13);
    const float A0323 = mdet2(m, 8, 15, 11, 12), A0223 = mdet2(m, 8, 14, 10, 12), A0123 = mdet2(m, 8, 13, 9, 12);
    const float A2313 = mdet2(m, 6, 15, 7, 14), A1313 = mdet2(m, 5, 15, 7, 13), A1213 = mdet2(m, 5, 14, 6, 13);
    const float A2312 = mdet2(m, 6, 11, 7, 10), A1312 = mdet2(m, 5, 11, 7, 9), A1212 = mdet2(m, 5, 10, 6, 9);
    const float A0313 = mdet2(m, 4, 15, 7, 12), A0213 = mdet2(m, 4, 14, 6, 12), A0312 = mdet2(m, 4, 11, 7, 8);
    const float A0212 = mdet2(m, 4, 10, 6, 8), A0113 = mdet2(m, 4, 13, 5, 12), A0112 = mdet2(m, 4, 9, 5, 8);
    /* c(a, b, c, p, q, r) = a * p - b * q + c * r */
#define C3(a, b, c, p, q, r) (m[a] * (p) - m[b] * (q) + m[c] * (r))
    const float det = m[0] * C3(5, 6, 7, A2323, A1323, A1223) - m[1] * C3(4, 6, 7, A2323, A0323, A0223) +
                      m[2] * C3(4, 5, 7, A1323, A0323, A0123) - m[3] * C3(4, 5, 6, A1223, A0223, A0123);
    const float k = 1.0f / det;
    o[0] = k * C3(5, 6, 7, A2323, A1323, A1223);
    o[1] = k * -C3(1, 2, 3, A2323, A1323, A1223);
    o[2] = k * C3(1, 2, 3, A2313, A1313, A1213);
    o[3] = k * -C3(1, 2, 3, A2312, A1312, A1212);
    o[4] = k * -C3(4, 6, 7, A2323, A0323, A0223);
    o[5] = k * C3(0, 2, 3, A2323, A0323, A0223);
    o[6] = k * -C3(0, 2, 3, A2313, A0313, A0213);
    o[7] = k * C3(0, 2, 3, A2312, A0312, A0212);
    o[8] = k * C3(4, 5, 7, A1323, A0323, A0123);
    o[9] = k * -C3(0, 1, 3, A1323, A0323, A0123);
    o[10] = k * C3(0, 1, 3, A1313, A0313, A0113);
    o[11] = k * -C3(0, 1, 3, A1312, A0312, A0112);
    o[12] = k * -C3(4, 5, 6, A1223, A0223, A0123);
    o[13] = k * C3(0, 1, 2, A1223, A0223, A0123);
    o[14] = k * -C3(0, 1, 2, A1213, A0213, A0113);
    o[15] = k * C3(0, 1, 2, A1212, A0212, A0112);
#undef C3
}

/* TransformBoundingBox (src/Ray/internal/Core.cpp:888-907): the box of the
 * transformed corners, per output axis from the translation plus the smaller
 * and larger of each input axis' two products. */
static void transform_box(const float bmin[3], const float bmax[3], const float x[16], float out[6]) {
    for (int j = 0; j < 3; j++) {
        float lo = x[12 + j], hi = x[12 + j];
        for (int i = 0; i < 3; i++) {
            const float a = x[4 * i + j] * bmin[i], b = x[4 * i + j] * bmax[i];
            lo += a < b ? a : b;
            hi += a < b ? b : a;
        }
        out[j] = lo;
        out[3 + j] = hi;
    }
}

/* TransformNormal (CoreRef.cpp:1625-1629) with the inverse transform */
static pv3 xform_normal(const float *inv, pv3 n) {
    return P3(inv[0] * n.x + inv[1] * n.y + inv[2] * n.z, inv[4] * n.x + inv[5] * n.y + inv[6] * n.z,
              inv[8] * n.x + inv[9] * n.y + inv[10] * n.z);
}

/* ExtractPlaneNormal (src/Ray/internal/Core.cpp:216-228): the stored plane
 * coefficients scaled by their length (the reference's own scaling) */
static pv3 plane_normal(const orc_tri *tri) {
    float n[3];
    const int iw = tri->ci & 3;
    const int iu = iw == 0 ? 1 : 0, iv = iw == 2 ? 1 : 2;
    n[iw] = 1.0f;
    n[iu] = tri->nu;
    n[iv] = tri->nv;
    float l = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (tri->ci & 8) l = -l;
    return P3(n[0] * l, n[1] * l, n[2] * l);
}

typedef struct {
    const orc_principled_scene *sc;
    orc_bvh **bvh; /* per mesh */
    float *inv;    /* 16 floats per instance */
    float *wbox;   /* 6 floats per instance */
} pscene;

/* Closest hit over the instances in order (Traverse_MacroTree_WithStack_ClosestHit,
 * CoreRef.cpp:1133-1222): the instance box test with the current t, the ray
 * taken to object space by TransformRay (CoreRef.cpp:1605-1617), then the
 * mesh's triangles; hit.prim is the global triangle index, *obj the instance. */
static orc_hit trace_scene(const pscene *ps, pv3 po, pv3 pd, float tmax, int *obj) {
    const orc_principled_scene *sc = ps->sc;
    const float o[3] = {po.x, po.y, po.z}, d[3] = {pd.x, pd.y, pd.z};
    orc_hit h = {-1, tmax, 0.0f, 0.0f};
    *obj = -1;
    int32_t stack[512];
    for (int m = 0; m < sc->ninst; m++) {
        const int mesh = sc->inst_mesh[m];
        const int64_t first = sc->mesh_tris[2 * mesh], cnt = sc->mesh_tris[2 * mesh + 1];
        if (cnt == 0 || !ref_bbox_test(o, d, h.t, ps->wbox + 6 * m)) continue;
        const float *x = ps->inv + 16 * m;
        const float lo[3] = {x[0] * o[0] + x[4] * o[1] + x[8] * o[2] + x[12], x[1] * o[0] + x[5] * o[1] + x[9] * o[2] + x[13],
                             x[2] * o[0] + x[6] * o[1] + x[10] * o[2] + x[14]};
        const float ld[3] = {x[0] * d[0] + x[4] * d[1] + x[8] * d[2], x[1] * d[0] + x[5] * d[1] + x[9] * d[2],
                             x[2] * d[0] + x[6] * d[1] + x[10] * d[2]};
        const float inv_d[3] = {1.0f / ld[0], 1.0f / ld[1], 1.0f / ld[2]};
        const orc_bvh *b = ps->bvh[mesh];
        const int32_t before = h.prim;
        int sp = 0;
        if (b->nnodes > 0 && b->nodes[0].right != 0) stack[sp++] = 0;
        while (sp) {
            const onode *nd = &b->nodes[stack[--sp]];
            if (!box_hit(nd, lo, inv_d, h.t)) continue;
            if (nd->right <= 0) {
                for (int32_t i = 0; i < -nd->right; i++) {
                    const int64_t p = first + b->prims[nd->left + i];
                    intersect_tri(lo, ld, &sc->tris[p], (int32_t)p, &h);
                }
            } else if (sp < 510) {
                stack[sp++] = nd->right;
                stack[sp++] = nd->left;
            }
        }
        if (h.prim != before) *obj = m;
    }
    return h;
}

/* ComputeVisibility (CoreRef.cpp:1813-1896) for scenes whose surfaces are
 * all solid: blocked by any hit closer than p2. */
static float visibility(const pscene *ps, pv3 p1, pv3 p2) {
    pv3 dir = psub(p2, p1);
    const float dist = sqrtf(pdot(dir, dir));
    dir = pdiv(dir, dist);
    if (!(dist > ORC_HIT_EPS)) return 1.0f;
    int obj;
    return trace_scene(ps, p1, dir, dist, &obj).prim >= 0 ? 0.0f : 1.0f;
}

static pv3 sample_plain(const orc_principled_scene *sc, int tex, float u, float v) {
    if (tex < 0 || tex >= sc->ntex) return P3(1.0f, 1.0f, 1.0f);
    const int32_t *ti = sc->tex_info + 4 * tex;
    const uint32_t *px = sc->texels + ti[0];
    const int w = ti[1], h = ti[2];
    float fu = u - floorf(u), fv = v - floorf(v);
    if (!(fu >= 0.0f && fu < 1.0f)) fu = 0.0f;
    if (!(fv >= 0.0f && fv < 1.0f)) fv = 0.0f;
    const float x = fu * (float)w - 0.5f, y = fv * (float)h - 0.5f;
    const float x0 = floorf(x), y0 = floorf(y);
    const float kx = x - x0, ky = y - y0;
    const int ix = (int)x0, iy = (int)y0;
    const int xa = (ix + w) % w, xb = (ix + 1) % w, ya = (iy + h) % h, yb = (iy + 1) % h;
    const uint32_t p00 = px[ya * w + xa], p01 = px[ya * w + xb], p10 = px[yb * w + xa], p11 = px[yb * w + xb];
    float c[3];
    for (int k = 0; k < 3; k++) {
        const float a00 = (float)((p00 >> (8 * k)) & 0xFFu), a01 = (float)((p01 >> (8 * k)) & 0xFFu);
        const float a10 = (float)((p10 >> (8 * k)) & 0xFFu), a11 = (float)((p11 >> (8 * k)) & 0xFFu);
        const float top = a00 * (1.0f - kx) + a01 * kx, bot = a10 * (1.0f - kx) + a11 * kx;
        c[k] = (top * (1.0f - ky) + bot * ky) * (1.0f / 255.0f);
    }
    if (ti[3]) { /* srgb_to_rgb, CoreRef.cpp:377-389 */
        for (int k = 0; k < 3; k++) c[k] = c[k] > 0.04045f ? cr_powf((c[k] + 0.055f) / 1.055f, 2.4f) : c[k] / 12.92f;
    }
    return P3(c[0], c[1], c[2]);
}

/* the differentiable albedo at (u, v): bilinear, wrap-around, texel centres at (i + 0.5) / w */
static pv3 sample_param(const orc_principled_scene *sc, float u, float v) {
    const int w = sc->diff_aw, h = sc->diff_ah;
    float fu = u - floorf(u), fv = v - floorf(v);
    if (!(fu >= 0.0f && fu < 1.0f)) fu = 0.0f;
    if (!(fv >= 0.0f && fv < 1.0f)) fv = 0.0f;
    const float x = fu * (float)w - 0.5f, y = fv * (float)h - 0.5f;
    const float x0 = floorf(x), y0 = floorf(y);
    const float kx = x - x0, ky = y - y0;
    const int ix = (int)x0, iy = (int)y0;
    const int xa = (ix + w) % w, xb = (ix + 1) % w, ya = (iy + h) % h, yb = (iy + 1) % h;
    const float *t = sc->diff_albedo;
    float c[3];
    for (int k = 0; k < 3; k++) {
        const float top = t[((size_t)ya * w + xa) * 3 + k] * (1.0f - kx) + t[((size_t)ya * w + xb) * 3 + k] * kx;
        const float bot = t[((size_t)yb * w + xa) * 3 + k] * (1.0f - kx) + t[((size_t)yb * w + xb) * 3 + k] * kx;
        c[k] = top * (1.0f - ky) + bot * ky;
    }
    return P3(c[0], c[1], c[2]);
}

/* the default environment map, one white RGBE texel (exponent 128) at the
 * atlas origin, read by SampleLatlong_RGBE (CoreRef.cpp:1772-1798) */
static float env_white(pv3 dir) {
    const float theta = cr_acosf(clamp_s(dir.y, -1.0f, 1.0f)) / ORC_PI;
    const float r = sqrtf(dir.x * dir.x + dir.z * dir.z);
    float u = 0.5f * cr_acosf(r > ORC_FLT_EPS ? clamp_s(dir.x / r, -1.0f, 1.0f) : 0.0f) / ORC_PI;
    if (dir.z < 0.0f) u = 1.0f - u;
    const float ux = 0.0f + u * 1.0f + 1.0f, uy = 0.0f + theta * 1.0f + 1.0f;
    const float kx = ux - simd_floorf(ux), ky = uy - simd_floorf(uy);
    return (1.0f * kx + 1.0f * (1 - kx)) * ky + (1.0f * kx + 1.0f * (1 - kx)) * (1 - ky);
}

typedef struct {
    pv3 o, d, c;
    float prev_pdf;
    int depth;
} ppath;

#define ORC_HIT_BIAS 0.001f
#define ORC_MAX_DIST 3.402823466e+38F

/* One shading step of the GPU renderer for a path segment: returns its
 * colour in col_out; *emit is set, with the continuation in *next, when the
 * path goes on. The vertex's light sample comes back apart (nee, *nee_valid):
 * the pixel adds it after col_out when its shadow ray is unblocked. */
static void shade_principled(const pscene *ps, const ppath *ray, int pixel, int iteration, int bounce, int max_diff, int max_total,
                             int term_start, float col_out[4], ppath *next, int *emit, float nee[3], int *nee_valid) {
    const orc_principled_scene *sc = ps->sc;
    *emit = 0;
    *nee_valid = 0;
    int obj;
    const orc_hit hit = trace_scene(ps, ray->o, ray->d, ORC_MAX_DIST, &obj);
    const pv3 I = ray->d;
    float cr = 0.0f, cg = 0.0f, cb = 0.0f, ca = 1.0f;
    if (hit.prim < 0) {
        const float e = env_white(I);
        cr = ray->c.x * e * sc->env_col[0];
        cg = ray->c.y * e * sc->env_col[1];
        cb = ray->c.z * e * sc->env_col[2];
    } else {
        const orc_tri *tri = &sc->tris[hit.prim];
        const float *inv = ps->inv + 16 * obj;
        const float t = hit.t, hu = hit.u, hv = hit.v;
        const pv3 P = padd(ray->o, pscale(I, t));
        const float w = 1.0f - hu - hv;
        const float *nn = sc->normals + 9 * (int64_t)hit.prim, *uv = sc->uvs + 6 * (int64_t)hit.prim;
        pv3 N = padd(padd(pscale(P3(nn[0], nn[1], nn[2]), w), pscale(P3(nn[3], nn[4], nn[5]), hu)), pscale(P3(nn[6], nn[7], nn[8]), hv));
        const float uvx = uv[0] * w + uv[2] * hu + uv[4] * hv;
        const float uvy = uv[1] * w + uv[3] * hu + uv[5] * hv;
        pv3 plane_N = xform_normal(inv, plane_normal(tri));
        int mi = sc->mat[2 * (int64_t)hit.prim];
        if (pdot(plane_N, I) > 0.0f) {
            mi = sc->mat[2 * (int64_t)hit.prim + 1];
            plane_N = P3(-plane_N.x, -plane_N.y, -plane_N.z);
            N = P3(-N.x, -N.y, -N.z);
        }
        if (mi < 0 || mi >= sc->nmats) {
            ca = 0.0f;
        } else {
            const float *m = sc->mats + 8 * mi;
            const int diff_depth = ray->depth & 0xff;
            const int total_depth = diff_depth;
            const int cant_terminate = total_depth < term_start;
            const pv3 wo = pnorm(P3(-I.x, -I.y, -I.z));
            pv3 Ns = pnorm(xform_normal(inv, N));
            if (!(pdot(Ns, wo) > 0.0f)) Ns = pnorm(plane_N);
            const pframe fr = make_frame(Ns);
            const pv3 wo_l = to_local(&fr, wo);
            const int slot = (int)m[6];
            const int dparam = slot >= 0 && slot < sc->n_diff_rough && sc->diff_albedo != NULL;
            const pv3 base = pmul(dparam ? sample_param(sc, uvx, uvy) : sample_plain(sc, (int)m[5], uvx, uvy), P3(m[0], m[1], m[2]));
            const pparams prm = make_params(base, dparam ? sc->diff_rough[slot] : m[3], m[4]);
            const int frozen = dparam && sc->diff_rough_sampling != NULL;
            const pparams prm_s = frozen ? make_params(base, sc->diff_rough_sampling[slot], m[4]) : prm;
            const uint32_t sidx = (uint32_t)(iteration - 1);
            const pv3 P_off = padd(P, pscale(plane_N, ORC_HIT_BIAS));
            pv3 col = P3(0.0f, 0.0f, 0.0f);
            if (sc->nlights > 0) { /* next-event estimation from one light picked uniformly */
                float ul, ua, ub, uc;
                sobol2(sidx, dim_seed((uint32_t)pixel, bounce, 2), &ul, &ua);
                sobol2(sidx, dim_seed((uint32_t)pixel, bounce, 3), &ub, &uc);
                const uint32_t nl = (uint32_t)sc->nlights;
                uint32_t k = (uint32_t)(ul * (float)nl);
                if (k >= nl) k = nl - 1;
                const plight *L = (const plight *)(sc->lights + 20 * k);
                const pv3 Lc = P3(L->L[0], L->L[1], L->L[2]);
                if (L->type == ORC_LIGHT_QUAD) {
                    const pv3 p = padd(padd(P3(L->p0[0], L->p0[1], L->p0[2]), pscale(P3(L->u[0], L->u[1], L->u[2]), ub)),
                                       pscale(P3(L->v[0], L->v[1], L->v[2]), uc));
                    const pv3 dv = psub(p, P_off);
                    const float dist2 = pdot(dv, dv);
                    const float dist = sqrtf(dist2);
                    const pv3 wi = pdiv(dv, dist);
                    const float cos_l = -pdot(wi, P3(L->n[0], L->n[1], L->n[2]));
                    if (cos_l > 0.0f) {
                        const float pdf_l = dist2 / (L->area * cos_l) / (float)nl;
                        pv3 f_cos, unused;
                        float pdf_b;
                        ggx_eval(&prm, wo_l, to_local(&fr, wi), &f_cos, &pdf_b);
                        if (frozen) ggx_eval(&prm_s, wo_l, to_local(&fr, wi), &unused, &pdf_b);
                        if (f_cos.x > 0.0f || f_cos.y > 0.0f || f_cos.z > 0.0f) {
                            const pv3 e = pscale(pmul(Lc, f_cos), power_heuristic(pdf_l, pdf_b) / pdf_l);
                            if (visibility(ps, P_off, p) > 0.0f) {
                                nee[0] = ray->c.x * e.x;
                                nee[1] = ray->c.y * e.y;
                                nee[2] = ray->c.z * e.z;
                                *nee_valid = 1;
                            }
                        }
                    }
                } else {
                    const float cos_t = 1.0f - ub * (1.0f - L->cos_max);
                    const float sin_t = sqrtf(fmax_s(0.0f, 1.0f - cos_t * cos_t));
                    const float phi = 2.0f * ORC_PI * uc;
                    const pframe fs = make_frame(P3(L->n[0], L->n[1], L->n[2]));
                    const pv3 wi = to_world(&fs, P3(sin_t * cr_cosf(phi), sin_t * cr_sinf(phi), cos_t));
                    pv3 f_cos;
                    float pdf_b;
                    ggx_eval(&prm, wo_l, to_local(&fr, wi), &f_cos, &pdf_b);
                    if (f_cos.x > 0.0f || f_cos.y > 0.0f || f_cos.z > 0.0f) {
                        const pv3 e = pscale(pmul(Lc, f_cos), (float)nl);
                        if (visibility(ps, P_off, padd(P_off, pscale(wi, 1.0e5f))) > 0.0f) {
                            nee[0] = ray->c.x * e.x;
                            nee[1] = ray->c.y * e.y;
                            nee[2] = ray->c.z * e.z;
                            *nee_valid = 1;
                        }
                    }
                }
            }
            if (diff_depth < max_diff && total_depth < max_total) {
                float u1, u2, ulobe, urr;
                sobol2(sidx, dim_seed((uint32_t)pixel, bounce, 0), &u1, &u2);
                sobol2(sidx, dim_seed((uint32_t)pixel, bounce, 1), &ulobe, &urr);
                pv3 wi_l;
                if (ggx_sample(&prm_s, wo_l, u1, u2, ulobe, &wi_l)) {
                    pv3 f_cos, unused;
                    float pdf;
                    ggx_eval(&prm, wo_l, wi_l, &f_cos, &pdf);
                    if (frozen) ggx_eval(&prm_s, wo_l, wi_l, &unused, &pdf);
                    if (pdf > 0.0f) {
                        const pv3 wi = to_world(&fr, wi_l);
                        next->o = padd(P, pscale(plane_N, pdot(wi, plane_N) > 0.0f ? ORC_HIT_BIAS : -ORC_HIT_BIAS));
                        next->d = wi;
                        next->c = pmul(ray->c, pdiv(f_cos, pdf));
                        next->prev_pdf = pdf;
                        next->depth = ray->depth + 1;
                        /* Russian roulette, CoreRef.cpp:2246-2256 */
                        const float lum = fmax_s(next->c.x, fmax_s(next->c.y, next->c.z));
                        const float q = cant_terminate ? 0.0f : fmax_s(0.05f, 1.0f - lum);
                        if (urr >= q) {
                            next->c = P3(next->c.x / (1.0f - q), next->c.y / (1.0f - q), next->c.z / (1.0f - q));
                            *emit = 1;
                        }
                    }
                }
            }
            cr = ray->c.x * col.x;
            cg = ray->c.y * col.y;
            cb = ray->c.z * col.z;
        }
    }
    /* quad lights the segment passes before its hit, weighted against the
     * light pdf of the vertex that sampled it */
    const float tmax = hit.prim >= 0 ? hit.t : ORC_MAX_DIST;
    for (int k = 0; k < sc->nlights; k++) {
        const plight *L = (const plight *)(sc->lights + 20 * k);
        float tq;
        if (L->type != ORC_LIGHT_QUAD || !hit_quad(L, ray->o, ray->d, tmax, &tq)) continue;
        float wgt = 1.0f;
        if (ray->prev_pdf > 0.0f) {
            const float cos_l = -pdot(ray->d, P3(L->n[0], L->n[1], L->n[2]));
            const float pdf_l = tq * tq / (L->area * cos_l) / (float)sc->nlights;
            wgt = power_heuristic(ray->prev_pdf, pdf_l);
        }
        cr += ray->c.x * L->L[0] * wgt;
        cg += ray->c.y * L->L[1] * wgt;
        cb += ray->c.z * L->L[2] * wgt;
    }
    col_out[0] = cr;
    col_out[1] = cg;
    col_out[2] = cb;
    col_out[3] = ca;
}

typedef struct {
    const pscene *ps;
    const orc_camera *cam;
    const float *halton;
    int w, h, iteration, max_diff, max_total, term_start;
    float *temp;
    int row0, row1;
} prender_work;

static void *prender_worker(void *arg) {
    prender_work *pw = (prender_work *)arg;
    for (int y = pw->row0; y < pw->row1; y++) {
        for (int x = 0; x < pw->w; x++) {
            orc_ray_packet pk;
            orc_generate_primary_rays(pw->cam, pw->iteration, x, y, 1, 1, pw->w, pw->h, pw->halton, &pk);
            ppath ray = {P3(pk.o[0], pk.o[1], pk.o[2]), P3(pk.d[0], pk.d[1], pk.d[2]), P3(pk.c[0], pk.c[1], pk.c[2]), 0.0f, 0};
            const int pixel = y * pw->w + x;
            float c[4], acc[4], nee[3];
            ppath next;
            int emit, nee_valid;
            /* bounce numbering as the renderer's: 2 for camera rays, 3.. after;
             * each vertex adds its colour, then its unblocked light sample */
            shade_principled(pw->ps, &ray, pixel, pw->iteration, 2, pw->max_diff, pw->max_total, pw->term_start, acc, &next, &emit, nee,
                             &nee_valid);
            if (nee_valid)
                for (int k = 0; k < 3; k++) acc[k] += nee[k];
            for (int b = 0; b < pw->max_total && emit; b++) {
                ray = next;
                shade_principled(pw->ps, &ray, pixel, pw->iteration, b + 3, pw->max_diff, pw->max_total, pw->term_start, c, &next, &emit,
                                 nee, &nee_valid);
                acc[0] += c[0];
                acc[1] += c[1];
                acc[2] += c[2];
                if (nee_valid)
                    for (int k = 0; k < 3; k++) acc[k] += nee[k];
            }
            memcpy(pw->temp + 4 * (size_t)pixel, acc, sizeof(acc));
        }
    }
    return NULL;
}

void orc_render_principled(const orc_principled_scene *sc, const orc_camera *cam, int w, int h, int spp, int max_diff_depth,
                           int max_total_depth, int termination_start_depth, float *out, int nthreads, int plain_mean) {
    pscene ps;
    ps.sc = sc;
    ps.bvh = (orc_bvh **)calloc((size_t)(sc->nmeshes > 0 ? sc->nmeshes : 1), sizeof(orc_bvh *));
    ps.inv = (float *)malloc(sizeof(float) * 16 * (size_t)(sc->ninst > 0 ? sc->ninst : 1));
    ps.wbox = (float *)malloc(sizeof(float) * 6 * (size_t)(sc->ninst > 0 ? sc->ninst : 1));
    float *mbox = (float *)malloc(sizeof(float) * 6 * (size_t)(sc->nmeshes > 0 ? sc->nmeshes : 1));
    for (int m = 0; m < sc->nmeshes; m++) {
        const int64_t first = sc->mesh_tris[2 * m], cnt = sc->mesh_tris[2 * m + 1];
        ps.bvh[m] = orc_bvh_build(sc->aabbs + 6 * first, cnt);
        /* the mesh box: the union of its triangles' boxes */
        for (int k = 0; k < 3; k++) {
            mbox[6 * m + k] = INFINITY;
            mbox[6 * m + 3 + k] = -INFINITY;
        }
        for (int64_t i = first; i < first + cnt; i++)
            for (int k = 0; k < 3; k++) {
                mbox[6 * m + k] = fminf(mbox[6 * m + k], sc->aabbs[6 * i + k]);
                mbox[6 * m + 3 + k] = fmaxf(mbox[6 * m + 3 + k], sc->aabbs[6 * i + 3 + k]);
            }
    }
    for (int i = 0; i < sc->ninst; i++) {
        inverse4(sc->inst_xform + 16 * i, ps.inv + 16 * i);
        const float *mb = mbox + 6 * sc->inst_mesh[i];
        transform_box(mb, mb + 3, sc->inst_xform + 16 * i, ps.wbox + 6 * i);
    }
    uint16_t perms[1002];
    orc_halton_perms(perms);
    float *table = (float *)malloc(sizeof(float) * (24 * 256 + 64));
    float *temp = (float *)malloc(sizeof(float) * 4 * (size_t)w * h);
    memset(out, 0, sizeof(float) * 4 * (size_t)w * h);
    if (nthreads < 1) nthreads = 1;
    if (max_total_depth > 10) max_total_depth = 10; /* MAX_BOUNCES, src/Ray/internal/Core.h:53 */
    int base = -1;
    for (int it = 1; it <= spp; it++) {
        /* the sample table of iteration it: from 1 below 256, else from it & ~255 */
        const int b = it < 256 ? 1 : (it & ~255);
        if (b != base) {
            memset(table, 0, sizeof(float) * (24 * 256 + 64));
            orc_halton_table(b, perms, table);
            base = b;
        }
        pthread_t th[64];
        prender_work pw[64];
        const int nt = nthreads > 64 ? 64 : nthreads;
        for (int t = 0; t < nt; t++) {
            pw[t] = (prender_work){&ps,
                                   cam,
                                   table,
                                   w,
                                   h,
                                   it,
                                   max_diff_depth,
                                   max_total_depth,
                                   termination_start_depth,
                                   temp,
                                   (int)((int64_t)h * t / nt),
                                   (int)((int64_t)h * (t + 1) / nt)};
            pthread_create(&th[t], NULL, prender_worker, &pw[t]);
        }
        for (int t = 0; t < nt; t++) pthread_join(th[t], NULL);
        if (plain_mean) { /* the differentiable forward pass: a sum, scaled at the end */
            for (size_t i = 0; i < 4 * (size_t)w * h; i++) out[i] = it == 1 ? temp[i] : out[i] + temp[i];
        } else { /* Framebuffer::MixWith (FramebufferRef.cpp:57-68) */
            const float k = 1.0f / (float)it;
            for (size_t i = 0; i < 4 * (size_t)w * h; i++) out[i] += (temp[i] - out[i]) * k;
        }
    }
    if (plain_mean) {
        const float inv = 1.0f / (float)spp;
        for (size_t i = 0; i < 4 * (size_t)w * h; i++) out[i] = out[i] * inv;
    }
    free(temp);
    free(table);
    for (int m = 0; m < sc->nmeshes; m++) orc_bvh_free(ps.bvh[m]);
    free(mbox);
    free(ps.bvh);
    free(ps.inv);
    free(ps.wbox);
}

int orc_area_light(int type, const float position[3], const float color[3], const float direction[3], float angle,
                   const float edge_u[3], const float edge_v[3], float out[20]) {
    plight a;
    memset(&a, 0, sizeof(a));
    a.type = (uint32_t)type;
    for (int k = 0; k < 3; k++) a.L[k] = color[k];
    if (type == 3) {
        const float *u = edge_u, *v = edge_v;
        const float c[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
        const float area = sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        if (!(area > 0.0f)) return -1;
        for (int k = 0; k < 3; k++) {
            a.p0[k] = position[k];
            a.u[k] = u[k];
            a.v[k] = v[k];
            a.n[k] = c[k] / area;
        }
        a.area = area;
    } else if (type == 4) {
        const float l = sqrtf(direction[0] * direction[0] + direction[1] * direction[1] + direction[2] * direction[2]);
        if (!(l > 0.0f) || !(angle > 0.0f && angle < 180.0f)) return -1;
        for (int k = 0; k < 3; k++) a.n[k] = -direction[k] / l;
        a.cos_max = cosf(0.5f * angle * ORC_PI / 180.0f);
    } else {
        return -1;
    }
    memcpy(out, &a, sizeof(a));
    return 0;
}
