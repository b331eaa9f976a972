// Kernels of the renderer: sample table, primary rays, shading (with shadow
// rays traced in the kernel), and the accumulate/tone pass. One thread per
// ray or pixel; ray counts live on the device so a frame's bounces run back
// to back without a host round trip.
#include "ggx.cuh"
#include "render.cuh"
#include "shade.cuh"
#include "traverse.cuh"

namespace rg {

using namespace shade;
using trav::Best;
using trav::Stack;

namespace {

constexpr int SHADE_BLOCK = 128;
constexpr float PI_F = 3.141592653589793238463f;
constexpr float HIT_BIAS = 0.001f;
constexpr float LIGHT_ATTEN_CUTOFF = 0.001f;

__constant__ int c_primes[HALTON_COUNT] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89};
// sampling_pattern (src/Ray/internal/Core.cpp:152-160): the 8x8 pixel pattern
// of UseCoherentSampling
__constant__ int c_sampling_pattern[64] = {0, 1, 2, 3, 1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2, 1, 2, 3, 0, 2, 1, 0, 3,
                                           3, 0, 1, 2, 0, 3, 2, 1, 2, 3, 0, 1, 1, 0, 3, 2, 0, 1, 2, 3, 0, 3, 2, 1,
                                           3, 2, 1, 0, 3, 2, 1, 0, 1, 0, 3, 2, 2, 1, 0, 3};

// ScrambledRadicalInverse (src/Ray/internal/Halton.h:61-74) for row i, dim k
// of UpdateHaltonSequence (RendererRef.cpp:327-358).
__global__ void k_halton_table(const uint16_t *__restrict__ perms, int base_iteration, float *__restrict__ table) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= HALTON_COUNT * HALTON_SEQ_LEN) return;
    const int i = idx / HALTON_COUNT, k = idx % HALTON_COUNT;
    int off = 0;
    for (int j = 0; j < k; j++) off += c_primes[j];
    const int base = c_primes[k];
    const uint16_t *perm = perms + off;
    const float inv_base = __fdiv_rn(1.0f, (float)base);
    uint64_t a = (uint64_t)(int64_t)(base_iteration + i);
    uint64_t reversed = 0;
    float inv_base_n = 1.0f;
    while (a) {
        const uint64_t next = a / (uint64_t)base;
        const uint64_t digit = a - next * (uint64_t)base;
        reversed = reversed * (uint64_t)base + perm[digit];
        inv_base_n = __fmul_rn(inv_base_n, inv_base);
        a = next;
    }
    const float v = __fmul_rn(inv_base_n, __fadd_rn(__ull2float_rn(reversed), __fdiv_rn(__fmul_rn(inv_base, (float)perm[0]),
                                                                                          __fsub_rn(1.0f, inv_base))));
    const float lim = 1.0f - 1.1920928955078125e-07f;
    table[idx] = (lim < v) ? lim : v;
}

// get_pix_dir of GeneratePrimaryRays (CoreRef.cpp:434-438)
__device__ __forceinline__ V3 pix_dir(const CameraDev &cam, float k, float fov_k, int w, int h, float x, float y, V3 origin) {
    const float px = 2 * fov_k * x / (float)w - fov_k, py = 2 * fov_k * (-y) / (float)h + fov_k, pz = cam.focus_distance;
    const V3 p = v3(cam.origin) + (k * px) * v3(cam.side) + py * v3(cam.up) + pz * v3(cam.fwd);
    return normalize(p - origin);
}

// GeneratePrimaryRays, CoreRef.cpp:427-505, for the pixel (x, y).
__device__ __forceinline__ void gen_primary(const CameraDev &cam, float k, float fov_k, int iteration, int x, int y, int w, int h,
                                            const float *__restrict__ halton, float4 &r0, float4 &r1, RayPayload &p) {
    const int index = y * w + x;
    const int hi = (iteration & (HALTON_SEQ_LEN - 1)) * HALTON_COUNT;
    float fx = (float)x, fy = (float)y;
    const int hash_val = hash_i(index);
    const float o1 = construct_float((uint32_t)hash_val), o2 = construct_float((uint32_t)hash_i(hash_val));
    if (cam.filter == 1) {
        float tx = frac_modf(halton[hi + 0] + o1);
        if (tx < 0.5f) tx = sqrtf(2.0f * tx) - 1.0f;
        else tx = 1.0f - sqrtf(2.0f - 2 * tx);
        float ty = frac_modf(halton[hi + 1] + o2);
        if (ty < 0.5f) ty = sqrtf(2.0f * ty) - 1.0f;
        else ty = 1.0f - sqrtf(2.0f - 2.0f * ty);
        fx += 0.5f + tx;
        fy += 0.5f + ty;
    } else {
        fx += frac_modf(halton[hi + 0] + o1);
        fy += frac_modf(halton[hi + 1] + o2);
    }
    const float ff1 = cam.focus_factor * (-0.5f + frac_modf(halton[hi + 2 + 0] + o1));
    const float ff2 = cam.focus_factor * (-0.5f + frac_modf(halton[hi + 2 + 1] + o2));
    const V3 origin = v3(cam.origin) + v3(cam.side) * ff1 + v3(cam.up) * ff2;
    const V3 d = pix_dir(cam, k, fov_k, w, h, fx, fy, origin);
    const V3 dx = pix_dir(cam, k, fov_k, w, h, fx + 1, fy, origin);
    const V3 dy = pix_dir(cam, k, fov_k, w, h, fx, fy + 1, origin);
    r0 = make_float4(origin.x, origin.y, origin.z, MAX_DIST);
    r1 = make_float4(d.x, d.y, d.z, __int_as_float((x << 16) | y));
    p.c[0] = p.c[1] = p.c[2] = 1.0f;
    p.ior = 1.0f;
    const V3 ddx = dx - d, ddy = dy - d;
    p.do_dx[0] = p.do_dx[1] = p.do_dx[2] = 0.0f;
    p.do_dy[0] = p.do_dy[1] = p.do_dy[2] = 0.0f;
    p.dd_dx[0] = ddx.x; p.dd_dx[1] = ddx.y; p.dd_dx[2] = ddx.z;
    p.dd_dy[0] = ddy.x; p.dd_dy[1] = ddy.y; p.dd_dy[2] = ddy.z;
    p.ray_depth = 0;
    p.pad[0] = p.pad[1] = p.pad[2] = 0;
}

// Closest hit of one ray against the whole scene: the instance loop of
// Traverse_MacroTree_WithStack_ClosestHit (CoreRef.cpp:1133-1222), as the
// trace kernels run it.
__device__ __forceinline__ Best trace_closest_scene(const SceneView &sv, float4 r0, float4 r1, Stack<true> &st, uint32_t &err) {
    Best best;
    best.t = r0.w;
    best.u = best.v = 0.0f;
    best.prim = best.obj = -1;
    const float sx = trav::safe_inv(r1.x), sy = trav::safe_inv(r1.y), sz = trav::safe_inv(r1.z);
    uint32_t nvis = 0, ntri = 0;
    for (uint32_t m = 0; m < sv.n_inst; m++) {
        const InstanceRec *ir = sv.inst + m;
        float bmin[3], bmax[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            bmin[q] = __ldg(&ir->bbox_min[q]);
            bmax[q] = __ldg(&ir->bbox_max[q]);
        }
        if (!trav::ref_bbox_test(r0.x, r0.y, r0.z, sx, sy, sz, best.t, bmin, bmax)) continue;
        trav::trace_mesh<false>(trav::mesh_of(sv, ir, (int)m), trav::transform_ray(ir, r0, r1), best, st, err, nvis, ntri);
    }
    return best;
}

// Shadow ray against the whole scene: the instance loop of
// Traverse_MacroTree_WithStack_AnyHit (CoreRef.cpp:1224-1368).
__device__ __forceinline__ Best trace_any(const SceneView &sv, V3 o, V3 d, float tmax, Stack<true> &st, uint32_t &err) {
    Best best;
    best.t = tmax;
    best.u = best.v = 0.0f;
    best.prim = best.obj = -1;
    const float sx = trav::safe_inv(d.x), sy = trav::safe_inv(d.y), sz = trav::safe_inv(d.z);
    const float4 r0 = make_float4(o.x, o.y, o.z, tmax), r1 = make_float4(d.x, d.y, d.z, 0.0f);
    for (uint32_t m = 0; m < sv.n_inst; m++) {
        const InstanceRec *ir = sv.inst + m;
        float bmin[3], bmax[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            bmin[q] = __ldg(&ir->bbox_min[q]);
            bmax[q] = __ldg(&ir->bbox_max[q]);
        }
        if (!trav::ref_bbox_test(o.x, o.y, o.z, sx, sy, sz, best.t, bmin, bmax)) continue;
        if (trav::trace_mesh_any(trav::mesh_of(sv, ir, (int)m), trav::transform_ray(ir, r0, r1), best, st, err)) break;
    }
    return best;
}

__device__ __forceinline__ void load_vertex(const RenderScene &sc, uint32_t vi, VertexRec &v) {
    const float4 *src = reinterpret_cast<const float4 *>(sc.vertices + vi);
    float4 *dst = reinterpret_cast<float4 *>(&v);
#pragma unroll
    for (int q = 0; q < 4; q++) dst[q] = __ldg(src + q);
}

__device__ __forceinline__ TriRec load_tri(const RenderScene &sc, uint32_t prim) {
    const float4 *tp = reinterpret_cast<const float4 *>(sc.tris + prim);
    const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
    TriRec t;
    t.nu = a.x; t.nv = a.y; t.np = a.z; t.pu = a.w;
    t.pv = b.x; t.ci = __float_as_int(b.y); t.e0u = b.z; t.e0v = b.w;
    t.e1u = c.x; t.e1v = c.y; t.mi = __float_as_uint(c.z); t.back_mi = __float_as_uint(c.w);
    return t;
}

constexpr uint32_t SHADE_ERR_BAD_INDEX = 8u;   // a material/texture/instance index out of range
constexpr uint32_t SHADE_ERR_MIX_LOOP = 16u;    // mix materials nested beyond the bound
constexpr uint32_t SHADE_ERR_SHADOW_LOOP = 32u; // more transparent layers than the bound
constexpr int MAX_MIX_NESTING = 32;
constexpr int MAX_SHADOW_LAYERS = 256;

// ComputeVisibility, CoreRef.cpp:1800-1896
__device__ float compute_visibility(const RenderScene &sc, V3 p1, V3 p2, const float *halton, int hi, int rand_hash2, Stack<true> &st,
                                    uint32_t &err, uint32_t &nshadow) {
    V3 dir = p2 - p1;
    float dist = length(dir);
    dir = dir / dist;
    V3 o = p1;
    float visibility = 1.0f;
    int layers = 0;
    while (dist > HIT_EPS) {
        if (++layers > MAX_SHADOW_LAYERS) {
            err |= SHADE_ERR_SHADOW_LOOP;
            break;
        }
        const Best sh = trace_any(sc.sv, o, dir, dist, st, err);
        nshadow++;
        if (sh.prim < 0) break;
        if ((uint32_t)sh.prim >= sc.n_tris || (uint32_t)sh.obj >= sc.sv.n_inst) {
            err |= SHADE_ERR_BAD_INDEX;
            break;
        }
        const TriRec tri = load_tri(sc, (uint32_t)sh.prim);
        if (tri.ci & TRI_SOLID_BIT) {
            visibility = 0;
            break;
        }
        uint32_t mi = tri.mi;
        const float *inv = sc.sv.inst[sh.obj].inv_xform;
        VertexRec v1, v2, v3v;
        load_vertex(sc, sc.vtx_indices[(uint32_t)sh.prim * 3 + 0], v1);
        load_vertex(sc, sc.vtx_indices[(uint32_t)sh.prim * 3 + 1], v2);
        load_vertex(sc, sc.vtx_indices[(uint32_t)sh.prim * 3 + 2], v3v);
        const V3 I = dir;
        const float w = 1.0f - sh.u - sh.v;
        const float uvx = v1.t[0][0] * w + v2.t[0][0] * sh.u + v3v.t[0][0] * sh.v;
        const float uvy = v1.t[0][1] * w + v2.t[0][1] * sh.u + v3v.t[0][1] * sh.v;
        V3 pn = transform_normal(plane_normal(tri), inv);
        bool skip = false;
        const bool is_backfacing = dot(pn, I) < 0.0f;
        if (is_backfacing) {
            if (tri.back_mi == RAY_INVALID_INDEX) skip = true;
            else {
                mi = tri.back_mi;
                pn = -pn;
            }
        }
        if (!skip) {
            const int sh_rand_hash = hash_i(rand_hash2);
            const float sh_rand_offset = construct_float((uint32_t)sh_rand_hash);
            float sh_r = frac_modf(halton[hi] + sh_rand_offset);
            int nest = 0;
            bool bad = false;
            while (true) {
                if (mi >= sc.n_materials) {
                    bad = true;
                    err |= SHADE_ERR_BAD_INDEX;
                    break;
                }
                const MaterialRec &mat = sc.materials[mi];
                if (mat.type != (uint32_t)RAY_MAT_MIX) break;
                if (++nest > MAX_MIX_NESTING) {
                    bad = true;
                    err |= SHADE_ERR_MIX_LOOP;
                    break;
                }
                const float mix_val = sample_bilinear(sc, mat.textures[1], uvx, uvy, 0).x * mat.roughness_or_strength;
                if (sh_r > mix_val) {
                    mi = mat.textures[2];
                    sh_r = (sh_r - mix_val) / (1.0f - mix_val);
                } else {
                    mi = mat.textures[3];
                    sh_r = sh_r / mix_val;
                }
            }
            if (bad || sc.materials[mi].type != (uint32_t)RAY_MAT_TRANSPARENT) {
                visibility = 0;
                break;
            }
        }
        const float t = sh.t + HIT_BIAS;
        o.x += dir.x * t;
        o.y += dir.y * t;
        o.z += dir.z * t;
        dist -= t;
    }
    return visibility;
}

// AcumulateLightContribution, CoreRef.cpp:1898-1933
// dcol (may be null): also adds the contribution's derivative by sigma.
__device__ __forceinline__ void accumulate_light(const RenderScene &sc, const LightRec &l, V3 I, V3 P, V3 N, V3 B, V3 plane_N, float sigma,
                                                 const float *halton, int hi, int rand_hash2, float rand_offset, float rand_offset2, V3 &col,
                                                 Stack<true> &st, uint32_t &err, uint32_t &nshadow, V3 *dcol = nullptr) {
    const V3 lpos = v3(l.pos);
    V3 L = P - lpos;
    const float distance = length(L);
    const float d = fmax_std(distance - l.radius, 0.0f);
    L = L / distance;
    const float z = frac_modf(halton[hi + 0] + rand_offset);
    const float dir = sqrtf(z);
    const float phi = 2 * PI_F * frac_modf(halton[hi + 1] + rand_offset2);
    const float cos_phi = cr_cos(phi), sin_phi = cr_sin(phi);
    const V3 TT = cross(L, B);
    const V3 BB = cross(L, TT);
    const V3 V = (dir * sin_phi) * BB + sqrtf(1.0f - dir) * L + (dir * cos_phi) * TT;
    L = normalize(lpos + V * l.radius - P);
    const float denom = d / l.radius + 1.0f;
    float atten = 1.0f / (denom * denom);
    atten = (atten - LIGHT_ATTEN_CUTOFF / l.brightness) / (1.0f - LIGHT_ATTEN_CUTOFF);
    atten = fmax_std(atten, 0.0f);
    const float dot1 = fmax_std(dot(L, N), 0.0f);
    const float dot2 = dot(L, v3(l.dir));
    if (dot1 > FLT_EPS_ && dot2 > l.spot && (l.brightness * atten) > FLT_EPS_) {
        const float visibility = compute_visibility(sc, P + HIT_BIAS * plane_N, lpos, halton, hi, rand_hash2, st, err, nshadow);
        if (dcol) {
            float d_sigma = 0.0f;
            const float on = brdf_oren_nayar_d(L, I, N, B, sigma, d_sigma);
            col = col + v3(l.col) * dot1 * visibility * atten * on;
            *dcol = *dcol + v3(l.col) * dot1 * visibility * atten * d_sigma;
        } else {
            col = col + v3(l.col) * dot1 * visibility * atten * brdf_oren_nayar(L, I, N, B, sigma);
        }
    }
}

struct NewRay {
    float4 r0, r1;
    RayPayload p;
};

// The shadow ray of the segment p1 -> p2 as ComputeVisibility forms it
// (direction p2 - p1 over its length, tmax the length); a segment of length
// HIT_EPS or less (which is visible without a trace) gets tmax 0.
__device__ __forceinline__ void shadow_ray(V3 p1, V3 p2, float4 &r0, float4 &r1) {
    V3 dir = p2 - p1;
    const float dist = length(dir);
    dir = dir / dist;
    if (dist > HIT_EPS) {
        r0 = make_float4(p1.x, p1.y, p1.z, dist);
        r1 = make_float4(dir.x, dir.y, dir.z, 0.0f);
    } else {
        r0 = make_float4(p1.x, p1.y, p1.z, 0.0f);
        r1 = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    }
}

// A RAY_MAT_PRINCIPLED vertex's light sample, traced after the shading: the
// segment o -> p2 and the colour it adds to the pixel when nothing blocks it
// (the path weight times the estimator). The pixel's sum takes the shading's
// colour first and this one after it, in every kernel and in the oracle.
struct ShadowReq {
    V3 o, p2, contrib;
    bool valid;
};

// What the adjoint needs of a RAY_MAT_PRINCIPLED vertex whose parameters are
// differentiable: the parameters as read, the local outgoing direction, the
// light sample's local direction and Le times its estimator scale, and the
// continuation's local direction.
struct VertexGrad {
    bool valid, light, cont;
    uint32_t slot;
    float u, v, rough;
    V3 main_color, wo_l, wl_l, le_s, wi_l;
    ggx::Params prm;
    float metallic;
    // a RAY_MAT_DIFFUSE vertex (diffuse set): its texture colour (the albedo
    // before main_color), the direct light it adds before the albedo and that
    // light's derivative by the roughness, whether the albedo multiplies them
    // (not on the camera rays of a lighting-only pass), and the continuation
    // weight's d(Oren-Nayar)/d(roughness) over Oren-Nayar
    bool diffuse, albedo_on;
    V3 tex, direct, d_direct;
    float cont_g;
};

// Russian roulette and emission of a continuation ray (CoreRef.cpp:2246-2256)
__device__ __forceinline__ bool roulette(NewRay &r, bool cant_terminate, float p) {
    const float lum = fmax_std(r.p.c[0], fmax_std(r.p.c[1], r.p.c[2]));
    const float q = cant_terminate ? 0.0f : fmax_std(0.05f, 1.0f - lum);
    if (p >= q) {
        r.p.c[0] /= 1.0f - q;
        r.p.c[1] /= 1.0f - q;
        r.p.c[2] /= 1.0f - q;
        return true;
    }
    return false;
}

__device__ __forceinline__ void set3(float *dst, V3 v) {
    dst[0] = v.x;
    dst[1] = v.y;
    dst[2] = v.z;
}

// ShadeSurface, CoreRef.cpp:2055-2391. Returns the pixel contribution;
// fills nr and sets emit when the path continues, and sr with a
// RAY_MAT_PRINCIPLED vertex's light sample. REF_LIGHTS: the scene may have
// the reference's point/spot/directional lights (their shadow rays are traced
// here); without, the kernel carries no traversal code.
template <bool REF_LIGHTS, bool PONLY = false>
__device__ F4 shade_hit(const RenderScene &sc, const PassInfo &pi, int rand_index, const float *halton, float4 hit, int obj,
                        float4 r0, float4 r1, const RayPayload &ray, NewRay &nr, bool &emit, ShadowReq &sr, Stack<true> &st,
                        uint32_t &err, uint32_t &nshadow, VertexGrad *vg = nullptr) {
    emit = false;
    sr.valid = false;
    if (vg) vg->valid = vg->diffuse = false;
    const int prim = __float_as_int(hit.x);
    const V3 I = v3(r1.x, r1.y, r1.z);
    const uint32_t xy = __float_as_uint(r1.w);
    if (prim < 0) {
        F4 env = {0.0f, 0.0f, 0.0f, 0.0f};
        if (!(pi.flags & PASS_NO_BACKGROUND) || pi.bounce > 2) {
            env = sample_latlong_rgbe(sc, sc.env_map, I);
            if (sc.env_clamp > FLT_EPS_) {
                const float c = sc.env_clamp;
                env.x = env.x < c ? env.x : c;
                env.y = env.y < c ? env.y : c;
                env.z = env.z < c ? env.z : c;
                env.w = env.w < c ? env.w : c;
            }
            env.w = 1.0f;
        }
        return F4{ray.c[0] * env.x * sc.env_col[0], ray.c[1] * env.y * sc.env_col[1], ray.c[2] * env.z * sc.env_col[2], env.w};
    }
    if ((uint32_t)prim >= sc.n_tris || (uint32_t)obj >= sc.sv.n_inst) {
        err |= SHADE_ERR_BAD_INDEX;
        return F4{0.0f, 0.0f, 0.0f, 0.0f};
    }
    const float t = hit.y, hu = hit.z, hv = hit.w;
    const V3 P = v3(r0.x, r0.y, r0.z) + t * I;
    const TriRec tri = load_tri(sc, (uint32_t)prim);
    uint32_t mi = tri.mi;
    const float *inv = sc.sv.inst[obj].inv_xform;
    VertexRec v1, v2, v3v;
    load_vertex(sc, sc.vtx_indices[(uint32_t)prim * 3 + 0], v1);
    load_vertex(sc, sc.vtx_indices[(uint32_t)prim * 3 + 1], v2);
    load_vertex(sc, sc.vtx_indices[(uint32_t)prim * 3 + 2], v3v);

    const float w = 1.0f - hu - hv;
    V3 N = v3(v1.n) * w + v3(v2.n) * hu + v3(v3v.n) * hv;
    const float uvx = v1.t[0][0] * w + v2.t[0][0] * hu + v3v.t[0][0] * hv;
    const float uvy = v1.t[0][1] * w + v2.t[0][1] * hu + v3v.t[0][1] * hv;

    V3 plane_N = transform_normal(plane_normal(tri), inv);
    const bool is_backfacing = dot(plane_N, I) > 0.0f;
    if (is_backfacing) {
        if (tri.back_mi == RAY_INVALID_INDEX) return F4{0.0f, 0.0f, 0.0f, 0.0f};
        mi = tri.back_mi;
        plane_N = -plane_N;
        N = -N;
    }

    Derivs der;
    compute_derivatives(I, t, v3(ray.do_dx), v3(ray.do_dy), v3(ray.dd_dx), v3(ray.dd_dy), v1, v2, v3v, plane_N, der);

    const int rand_hash = hash_i(rand_index), rand_hash2 = hash_i(rand_hash), rand_hash3 = hash_i(rand_hash2);
    const float rand_offset = construct_float((uint32_t)rand_hash), rand_offset2 = construct_float((uint32_t)rand_hash2),
                rand_offset3 = construct_float((uint32_t)rand_hash3);
    const int hi = (pi.iteration & (HALTON_SEQ_LEN - 1)) * HALTON_COUNT + pi.bounce * 2;

    float mix_rand = frac_modf(halton[hi] + rand_offset);
    int nest = 0;
    while (true) {
        if (mi >= sc.n_materials) {
            err |= SHADE_ERR_BAD_INDEX;
            return F4{0.0f, 0.0f, 0.0f, 0.0f};
        }
        const MaterialRec &mat = sc.materials[mi];
        if (PONLY || mat.type != (uint32_t)RAY_MAT_MIX) break;
        if (++nest > MAX_MIX_NESTING) {
            err |= SHADE_ERR_MIX_LOOP;
            return F4{0.0f, 0.0f, 0.0f, 0.0f};
        }
        float mix_val = sample_bilinear(sc, mat.textures[1], uvx, uvy, 0).x * mat.roughness_or_strength;
        const float mix_ior = is_backfacing ? mat.ext_ior : mat.int_ior;
        float R0 = (ray.ior - mix_ior) / (ray.ior + mix_ior);
        R0 *= R0;
        float RR;
        if (ray.ior > mix_ior) {
            const float eta = ray.ior / mix_ior;
            const float cosi = -dot(I, N);
            const float cost2 = 1.0f - eta * eta * (1.0f - cosi * cosi);
            if (cost2 >= 0.0f) {
                const float m = eta * cosi - sqrtf(cost2);
                const V3 V = eta * I + m * N;
                RR = R0 + (1.0f - R0) * pow5(1.0f + dot(V, N));
            } else {
                RR = 1.0f;
            }
        } else {
            RR = R0 + (1.0f - R0) * pow5(1.0f + dot(I, N));
        }
        mix_val *= clampf_ref(RR, 0.0f, 1.0f);
        if (mix_rand > mix_val) {
            mi = mat.textures[2];
            mix_rand = (mix_rand - mix_val) / (1.0f - mix_val);
        } else {
            mi = mat.textures[3];
            mix_rand = mix_rand / mix_val;
        }
    }
    const MaterialRec &mat = sc.materials[mi];
    const V3 N_vertex = N; // interpolated vertex normal (flipped on a back face), before the normal map

    // the reference's materials: normal map and main texture (RAY_MAT_PRINCIPLED reads neither)
    V3 B = v3(0.0f, 0.0f, 0.0f), T = v3(0.0f, 0.0f, 0.0f), alb = v3(0.0f, 0.0f, 0.0f);
    float sigma_d = mat.roughness_or_strength; // the diffuse material's Oren-Nayar roughness
    if (!PONLY && mat.type != (uint32_t)RAY_MAT_PRINCIPLED) {
        B = v3(v1.b) * w + v3(v2.b) * hu + v3(v3v.b) * hv;
        T = cross(B, N);
        F4 nm = sample_bilinear(sc, mat.textures[0], uvx, uvy, 0);
        nm.x = nm.x * 2.0f - 1.0f;
        nm.y = nm.y * 2.0f - 1.0f;
        nm.z = nm.z * 2.0f - 1.0f;
        N = nm.x * B + nm.z * N + nm.y * T;
        N = transform_normal(N, inv);
        B = transform_normal(B, inv);
        T = transform_normal(T, inv);

        const uint32_t main_tex = mat.textures[1];
        const float albedo_lod = texture_lod(sc, main_tex, der.duv_dx[0], der.duv_dx[1], der.duv_dy[0], der.duv_dy[1]);
        F4 albedo = sample_bilinear(sc, main_tex, uvx, uvy, f2i_x86(albedo_lod));
        if (main_tex < sc.n_textures && (sc.textures[main_tex].width & 0x8000u)) albedo = srgb_to_rgb(albedo);
        // a differentiable diffuse material: main colour and roughness from its slot
        const uint32_t dslot = mat.type == (uint32_t)RAY_MAT_DIFFUSE ? mat.textures[2] : RAY_INVALID_INDEX;
        const bool dparam = dslot < sc.n_diff_rough && sc.diff_rough;
        const V3 mc = (dparam && sc.diff_color) ? v3(sc.diff_color[3 * dslot], sc.diff_color[3 * dslot + 1], sc.diff_color[3 * dslot + 2])
                                                : v3(mat.main_color);
        if (dparam) sigma_d = sc.diff_rough[dslot];
        if (vg && dparam) {
            vg->diffuse = true;
            vg->slot = dslot;
            vg->tex = v3(albedo.x, albedo.y, albedo.z);
            vg->main_color = mc;
            vg->direct = vg->d_direct = v3(0.0f, 0.0f, 0.0f);
            vg->cont = false;
            vg->cont_g = 0.0f;
        }
        albedo.x *= mc.x;
        albedo.y *= mc.y;
        albedo.z *= mc.z;
        alb = v3(albedo.x, albedo.y, albedo.z);
    }

    V3 col = v3(0.0f, 0.0f, 0.0f);
    const int diff_depth = ray.ray_depth & 0xff, gloss_depth = (ray.ray_depth >> 8) & 0xff, refr_depth = (ray.ray_depth >> 16) & 0xff,
              transp_depth = (ray.ray_depth >> 24) & 0xff;
    const int total_depth = diff_depth + gloss_depth + refr_depth + transp_depth;
    const bool cant_terminate = total_depth < pi.termination_start_depth;
    const bool consider_albedo = !(pi.flags & PASS_LIGHTING_ONLY) || pi.bounce > 2;

    nr.r1.w = __uint_as_float(xy);
    nr.p.ior = ray.ior;
    nr.p.pad[0] = nr.p.pad[1] = nr.p.pad[2] = 0;
    const float dot_I_pN = dot(I, plane_N);

    if (!PONLY && mat.type == (uint32_t)RAY_MAT_DIFFUSE) {
        const bool dgrad = vg && vg->diffuse;
        if (dgrad) vg->albedo_on = consider_albedo;
        if (!(pi.flags & PASS_SKIP_DIRECT) || pi.bounce > 2) {
            if (REF_LIGHTS)
                for (uint32_t li = 0; li < sc.n_lights; li++)
                    accumulate_light(sc, sc.lights[li], I, P, N, B, plane_N, sigma_d, halton, hi, rand_hash2, rand_offset, rand_offset2, col, st,
                                     err, nshadow, dgrad ? &vg->d_direct : nullptr);
            if (dgrad) vg->direct = col;
            if (consider_albedo) col = col * alb;
        }
        if (diff_depth < pi.max_diff_depth && total_depth < pi.max_total_depth) {
            const float u1 = frac_modf(halton[hi + 0] + rand_offset);
            const float u2 = frac_modf(halton[hi + 1] + rand_offset2);
            const float phi = 2 * PI_F * u2;
            const float cos_phi = cr_cos(phi), sin_phi = cr_sin(phi);
            V3 V;
            float weight = 1.0f;
            if ((pi.flags & PASS_OUTPUT_SH) && pi.bounce <= 2) {
                const float dir = sqrtf(1.0f - u1 * u1);
                V = (dir * sin_phi) * B + u1 * N + (dir * cos_phi) * T;
                weight = 2 * u1;
            } else {
                const float dir = sqrtf(u1);
                V = (dir * sin_phi) * B + sqrtf(1.0f - u1) * N + (dir * cos_phi) * T;
            }
            if (dgrad) {
                float d_sigma = 0.0f;
                const float on = brdf_oren_nayar_d(V, I, N, B, sigma_d, d_sigma);
                weight *= on;
                vg->cont_g = on > 0.0f ? d_sigma / on : 0.0f;
            } else {
                weight *= brdf_oren_nayar(V, I, N, B, sigma_d);
            }
            nr.p.ray_depth = ray.ray_depth + 0x00000001;
            const V3 o = P + HIT_BIAS * plane_N;
            nr.r0 = make_float4(o.x, o.y, o.z, MAX_DIST);
            nr.r1.x = V.x; nr.r1.y = V.y; nr.r1.z = V.z;
            nr.p.c[0] = ray.c[0] * weight;
            nr.p.c[1] = ray.c[1] * weight;
            nr.p.c[2] = ray.c[2] * weight;
            if (consider_albedo) {
                nr.p.c[0] *= alb.x;
                nr.p.c[1] *= alb.y;
                nr.p.c[2] *= alb.z;
            }
            set3(nr.p.do_dx, der.do_dx);
            set3(nr.p.do_dy, der.do_dy);
            set3(nr.p.dd_dx, der.dd_dx - 2 * (dot_I_pN * der.dndx + der.ddn_dx * plane_N));
            set3(nr.p.dd_dy, der.dd_dy - 2 * (dot_I_pN * der.dndy + der.ddn_dy * plane_N));
            emit = roulette(nr, cant_terminate, frac_modf(halton[hi + 0] + rand_offset3));
            if (dgrad) vg->cont = emit;
        }
    } else if (!PONLY && mat.type == (uint32_t)RAY_MAT_GLOSSY) {
        if (gloss_depth < pi.max_glossy_depth && total_depth < pi.max_total_depth) {
            V3 V = reflect(I, N);
            const float rough = mat.roughness_or_strength;
            const float h = 1.0f - cr_cos(0.5f * PI_F * rough * rough);
            const float z = h * frac_modf(halton[hi + 0] + rand_offset);
            const float dir = sqrtf(z);
            const float phi = 2 * PI_F * frac_modf(halton[hi + 1] + rand_offset2);
            const float cos_phi = cr_cos(phi), sin_phi = cr_sin(phi);
            const V3 TT = cross(V, B);
            const V3 BB = cross(V, TT);
            if (dot(V, plane_N) > 0) {
                V = (dir * sin_phi) * BB + sqrtf(1.0f - dir) * V + (dir * cos_phi) * TT;
            } else {
                V = (-dir * sin_phi) * BB + sqrtf(1.0f - dir) * V - (dir * cos_phi) * TT;
            }
            nr.p.ray_depth = ray.ray_depth + 0x00000100;
            const V3 o = P + HIT_BIAS * plane_N;
            nr.r0 = make_float4(o.x, o.y, o.z, MAX_DIST);
            nr.r1.x = V.x; nr.r1.y = V.y; nr.r1.z = V.z;
            nr.p.c[0] = ray.c[0];
            nr.p.c[1] = ray.c[1];
            nr.p.c[2] = ray.c[2];
            if (consider_albedo) {
                nr.p.c[0] *= alb.x;
                nr.p.c[1] *= alb.y;
                nr.p.c[2] *= alb.z;
            }
            set3(nr.p.do_dx, der.do_dx);
            set3(nr.p.do_dy, der.do_dy);
            set3(nr.p.dd_dx, der.dd_dx - 2 * (dot_I_pN * der.dndx + der.ddn_dx * plane_N));
            set3(nr.p.dd_dy, der.dd_dy - 2 * (dot_I_pN * der.dndy + der.ddn_dy * plane_N));
            emit = roulette(nr, cant_terminate, frac_modf(halton[hi + 0] + rand_offset3));
        }
    } else if (!PONLY && mat.type == (uint32_t)RAY_MAT_REFRACTIVE) {
        if (refr_depth < pi.max_refr_depth && total_depth < pi.max_total_depth) {
            const float ior = is_backfacing ? mat.ext_ior : mat.int_ior;
            const float eta = ray.ior / ior;
            const float cosi = -dot(I, N);
            const float cost2 = 1.0f - eta * eta * (1.0f - cosi * cosi);
            if (cost2 < 0) return F4{0.0f, 0.0f, 0.0f, 1.0f};
            const float m = eta * cosi - sqrtf(cost2);
            V3 V = eta * I + m * N;
            const float z = 1.0f - halton[hi + 0] * mat.roughness_or_strength;
            const float temp = sqrtf(1.0f - z * z);
            const int hj = (int)(((uint32_t)(hash_i(hi) + pi.iteration) & (HALTON_SEQ_LEN - 1)) * HALTON_COUNT) + pi.bounce * 2;
            const float phi = halton[hj + 0] * 2 * PI_F;
            const float cos_phi = cr_cos(phi), sin_phi = cr_sin(phi);
            const V3 TT = normalize(cross(V, B));
            const V3 BB = normalize(cross(V, TT));
            V = (temp * sin_phi) * BB + z * V + (temp * cos_phi) * TT;
            const float kk = (eta - eta * eta * dot(I, plane_N) / dot(V, plane_N));
            const float dmdx = kk * der.ddn_dx, dmdy = kk * der.ddn_dy;
            nr.p.ior = ior;
            nr.p.ray_depth = ray.ray_depth + 0x00010000;
            const V3 o = P + HIT_BIAS * I;
            nr.r0 = make_float4(o.x, o.y, o.z, MAX_DIST);
            nr.r1.x = V.x; nr.r1.y = V.y; nr.r1.z = V.z;
            nr.p.c[0] = ray.c[0] * z;
            nr.p.c[1] = ray.c[1] * z;
            nr.p.c[2] = ray.c[2] * z;
            set3(nr.p.do_dx, der.do_dx);
            set3(nr.p.do_dy, der.do_dy);
            set3(nr.p.dd_dx, eta * der.dd_dx - (m * der.dndx + dmdx * plane_N));
            set3(nr.p.dd_dy, eta * der.dd_dy - (m * der.dndy + dmdy * plane_N));
            emit = roulette(nr, cant_terminate, frac_modf(halton[hi + 0] + rand_offset3));
        }
    } else if (PONLY || mat.type == (uint32_t)RAY_MAT_PRINCIPLED) {
        // metallic-roughness material: next-event estimation + a sampled continuation ray
        const V3 wo = normalize(-I);
        V3 Ns = normalize(transform_normal(N_vertex, inv));
        if (!(dot(Ns, wo) > 0.0f)) Ns = normalize(plane_N); // shading normal facing away: the face normal
        const ggx::Frame fr = ggx::make_frame(Ns);
        const V3 wo_l = ggx::to_local(fr, wo);
        // the differentiable parameters where the material has a slot
        const uint32_t slot = mat.textures[2];
        const bool dparam = slot < sc.n_diff_rough && sc.diff_albedo != nullptr;
        const V3 base = (dparam ? ggx::sample_param(sc, uvx, uvy) : ggx::sample_plain(sc, mat.textures[1], uvx, uvy)) * v3(mat.main_color);
        const float rough = dparam ? __ldg(sc.diff_rough + slot) : mat.roughness_or_strength;
        const ggx::Params prm = ggx::make_params(base, rough, mat.metallic);
        // sampling, pdfs and MIS weights: the same parameters unless frozen ones are given
        const bool frozen = dparam && sc.diff_rough_sampling != nullptr;
        const ggx::Params prm_s = frozen ? ggx::make_params(base, __ldg(sc.diff_rough_sampling + slot), mat.metallic) : prm;
        if (vg && dparam) {
            vg->valid = true;
            vg->light = vg->cont = false;
            vg->slot = slot;
            vg->u = uvx;
            vg->v = uvy;
            vg->rough = rough;
            vg->main_color = v3(mat.main_color);
            vg->wo_l = wo_l;
            vg->prm = prm;
            vg->metallic = mat.metallic;
        }
        const uint32_t sidx = (uint32_t)(pi.iteration - 1);
        const V3 P_off = P + HIT_BIAS * plane_N;
        if ((!(pi.flags & PASS_SKIP_DIRECT) || pi.bounce > 2) && sc.n_area_lights > 0) {
            float ul, ua, ub, uc;
            ggx::sobol2(sidx, ggx::dim_seed((uint32_t)rand_index, pi.bounce, 2), ul, ua);
            ggx::sobol2(sidx, ggx::dim_seed((uint32_t)rand_index, pi.bounce, 3), ub, uc);
            const uint32_t nl = sc.n_area_lights;
            uint32_t k = (uint32_t)(ul * (float)nl);
            if (k >= nl) k = nl - 1;
            const AreaLight L = sc.area_lights[k];
            if (L.type == (uint32_t)RAY_LIGHT_QUAD) {
                const V3 p = v3(L.p0) + v3(L.u) * ub + v3(L.v) * uc;
                const V3 dv = p - P_off;
                const float dist2 = dot(dv, dv);
                const float dist = sqrtf(dist2);
                const V3 wi = dv / dist;
                const float cos_l = -dot(wi, v3(L.n));
                if (cos_l > 0.0f) {
                    const float pdf_l = dist2 / (L.area * cos_l) / (float)nl;
                    V3 f_cos;
                    float pdf_b;
                    ggx::eval(prm, wo_l, ggx::to_local(fr, wi), f_cos, pdf_b);
                    if (frozen) {
                        V3 unused;
                        ggx::eval(prm_s, wo_l, ggx::to_local(fr, wi), unused, pdf_b);
                    }
                    if (f_cos.x > 0.0f || f_cos.y > 0.0f || f_cos.z > 0.0f) {
                        const float scale = ggx::power_heuristic(pdf_l, pdf_b) / pdf_l;
                        const V3 e = v3(L.L) * f_cos * scale;
                        sr.o = P_off;
                        sr.p2 = p;
                        sr.contrib = v3(ray.c[0] * e.x, ray.c[1] * e.y, ray.c[2] * e.z);
                        sr.valid = true;
                        if (vg && vg->valid) {
                            vg->light = true;
                            vg->wl_l = ggx::to_local(fr, wi);
                            vg->le_s = v3(L.L) * scale;
                        }
                    }
                }
            } else {
                const float cos_t = 1.0f - ub * (1.0f - L.cos_max);
                const float sin_t = sqrtf(fmax_std(0.0f, 1.0f - cos_t * cos_t));
                const float phi = 2.0f * PI_F * uc;
                const ggx::Frame fs = ggx::make_frame(v3(L.n));
                const V3 wi = ggx::to_world(fs, v3(sin_t * cr_cos(phi), sin_t * cr_sin(phi), cos_t));
                V3 f_cos;
                float pdf_b;
                ggx::eval(prm, wo_l, ggx::to_local(fr, wi), f_cos, pdf_b);
                if (f_cos.x > 0.0f || f_cos.y > 0.0f || f_cos.z > 0.0f) {
                    const V3 e = v3(L.L) * f_cos * (float)nl;
                    sr.o = P_off;
                    sr.p2 = P_off + wi * 1.0e5f;
                    sr.contrib = v3(ray.c[0] * e.x, ray.c[1] * e.y, ray.c[2] * e.z);
                    sr.valid = true;
                    if (vg && vg->valid) {
                        vg->light = true;
                        vg->wl_l = ggx::to_local(fr, wi);
                        vg->le_s = v3(L.L) * (float)nl;
                    }
                }
            }
        }
        if (diff_depth < pi.max_diff_depth && total_depth < pi.max_total_depth) {
            float u1, u2, ulobe, urr;
            ggx::sobol2(sidx, ggx::dim_seed((uint32_t)rand_index, pi.bounce, 0), u1, u2);
            ggx::sobol2(sidx, ggx::dim_seed((uint32_t)rand_index, pi.bounce, 1), ulobe, urr);
            V3 wi_l;
            if (ggx::sample(prm_s, wo_l, u1, u2, ulobe, wi_l)) {
                V3 f_cos;
                float pdf;
                ggx::eval(prm, wo_l, wi_l, f_cos, pdf);
                if (frozen) {
                    V3 unused;
                    ggx::eval(prm_s, wo_l, wi_l, unused, pdf);
                }
                if (pdf > 0.0f) {
                    const V3 wi = ggx::to_world(fr, wi_l);
                    const V3 o = P + (dot(wi, plane_N) > 0.0f ? HIT_BIAS : -HIT_BIAS) * plane_N;
                    nr.p.ray_depth = ray.ray_depth + 0x00000001;
                    nr.r0 = make_float4(o.x, o.y, o.z, MAX_DIST);
                    nr.r1.x = wi.x; nr.r1.y = wi.y; nr.r1.z = wi.z;
                    const V3 wgt = f_cos / pdf;
                    nr.p.c[0] = ray.c[0] * wgt.x;
                    nr.p.c[1] = ray.c[1] * wgt.y;
                    nr.p.c[2] = ray.c[2] * wgt.z;
                    set3(nr.p.do_dx, der.do_dx);
                    set3(nr.p.do_dy, der.do_dy);
                    set3(nr.p.dd_dx, der.dd_dx - 2 * (dot_I_pN * der.dndx + der.ddn_dx * plane_N));
                    set3(nr.p.dd_dy, der.dd_dy - 2 * (dot_I_pN * der.dndy + der.ddn_dy * plane_N));
                    nr.p.pad[0] = __float_as_uint(pdf); // for the MIS weight where this ray meets a quad light
                    emit = roulette(nr, cant_terminate, urr);
                    if (vg && vg->valid) {
                        vg->cont = emit;
                        vg->wi_l = wi_l;
                    }
                }
            }
        }
    } else if (mat.type == (uint32_t)RAY_MAT_EMISSIVE) {
        col = mat.roughness_or_strength * alb;
    } else if (mat.type == (uint32_t)RAY_MAT_TRANSPARENT) {
        if (transp_depth < pi.max_transp_depth && total_depth < pi.max_total_depth) {
            nr.p.ray_depth = ray.ray_depth + 0x01000000;
            const V3 o = P + HIT_BIAS * I;
            nr.r0 = make_float4(o.x, o.y, o.z, MAX_DIST);
            nr.r1.x = I.x; nr.r1.y = I.y; nr.r1.z = I.z;
            for (int q = 0; q < 3; q++) {
                nr.p.c[q] = ray.c[q];
                nr.p.do_dx[q] = ray.do_dx[q];
                nr.p.do_dy[q] = ray.do_dy[q];
                nr.p.dd_dx[q] = ray.dd_dx[q];
                nr.p.dd_dy[q] = ray.dd_dy[q];
            }
            emit = roulette(nr, cant_terminate, frac_modf(halton[hi + 0] + rand_offset3));
        }
    }
    return F4{ray.c[0] * col.x, ray.c[1] * col.y, ray.c[2] * col.z, 1.0f};
}

// shade_hit plus the emission of the quad lights the ray passes on its way to
// the hit: weight 1 for rays whose last vertex did not sample quad lights
// (pdf 0 in the payload), else the power heuristic against the light pdf that
// next-event estimation at that vertex used.
template <bool REF_LIGHTS, bool PONLY = false>
__device__ __forceinline__ F4 shade_surface(const RenderScene &sc, const PassInfo &pi, int rand_index, const float *halton, float4 hit,
                                            int obj, float4 r0, float4 r1, const RayPayload &ray, NewRay &nr, bool &emit, ShadowReq &sr,
                                            Stack<true> &st, uint32_t &err, uint32_t &nshadow, VertexGrad *vg = nullptr) {
    F4 c = shade_hit<REF_LIGHTS, PONLY>(sc, pi, rand_index, halton, hit, obj, r0, r1, ray, nr, emit, sr, st, err, nshadow, vg);
    if (sc.n_area_lights == 0) return c;
    const V3 o = v3(r0.x, r0.y, r0.z), d = v3(r1.x, r1.y, r1.z);
    const float tmax = __float_as_int(hit.x) >= 0 ? hit.y : MAX_DIST;
    const float prev_pdf = __uint_as_float(ray.pad[0]);
    for (uint32_t k = 0; k < sc.n_area_lights; k++) {
        const AreaLight &L = sc.area_lights[k];
        float tq;
        if (L.type != (uint32_t)RAY_LIGHT_QUAD || !ggx::hit_quad(L, o, d, tmax, tq)) continue;
        float w = 1.0f;
        if (prev_pdf > 0.0f) { // a unit direction sampled by RAY_MAT_PRINCIPLED
            const float cos_l = -dot(d, v3(L.n));
            const float pdf_l = tq * tq / (L.area * cos_l) / (float)sc.n_area_lights;
            w = ggx::power_heuristic(prev_pdf, pdf_l);
        }
        c.x += ray.c[0] * L.L[0] * w;
        c.y += ray.c[1] * L.L[1] * w;
        c.z += ray.c[2] * L.L[2] * w;
    }
    return c;
}

// Framebuffer::MixWith, ComputeSHData, MixWith_SH (FramebufferRef.cpp:57-101)
// and the tone step of RenderScene (RendererRef.cpp:301-324).
// p: the pixel's sample; s (may be null): its SH sample data, rewritten in place.
__device__ __forceinline__ void resolve_pixel(float4 p, float4 *__restrict__ clean, float4 *__restrict__ fin, SHData *s,
                                              SHData *__restrict__ clean_sh, size_t idx, float k, int srgb, float gamma, int clamp) {
    float4 c = clean[idx];
    c.x += (p.x - c.x) * k;
    c.y += (p.y - c.y) * k;
    c.z += (p.z - c.z) * k;
    c.w += (p.w - c.w) * k;
    clean[idx] = c;
    if (s) {
        const float inv_weight = s->coeff_g[0] > FLT_EPS_ ? (2.0f * PI_F / s->coeff_g[0]) : 0.0f;
        const float pr = p.x * inv_weight, pg = p.y * inv_weight, pb = p.z * inv_weight;
        for (int j = 0; j < 4; j++) {
            s->coeff_g[j] = s->coeff_r[j] * pg;
            s->coeff_b[j] = s->coeff_r[j] * pb;
            s->coeff_r[j] = s->coeff_r[j] * pr;
        }
        SHData o = clean_sh[idx];
        for (int j = 0; j < 4; j++) {
            o.coeff_r[j] += (s->coeff_r[j] - o.coeff_r[j]) * k;
            o.coeff_g[j] += (s->coeff_g[j] - o.coeff_g[j]) * k;
            o.coeff_b[j] += (s->coeff_b[j] - o.coeff_b[j]) * k;
        }
        clean_sh[idx] = o;
    }
    float v[4] = {c.x, c.y, c.z, c.w};
    if (srgb) {
        for (int q = 0; q < 3; q++) {
            if (v[q] > 0.0031308f) v[q] = cr_pow(1.055f * v[q], (1.0f / 2.4f)) - 0.055f;
            else v[q] = 12.92f * v[q];
        }
    }
    if (gamma != 1.0f) {
        const float g = 1.0f / gamma;
        for (int q = 0; q < 4; q++) v[q] = cr_pow(v[q], g);
    }
    if (clamp) {
        for (int q = 0; q < 4; q++) {
            const float t = v[q] < 1.0f ? v[q] : 1.0f; // minps(v, 1)
            v[q] = 0.0f > t ? 0.0f : t;               // maxps(0, t)
        }
    }
    fin[idx] = make_float4(v[0], v[1], v[2], v[3]);
}

// Job of a global ray or pixel index: the jobs cover consecutive ranges from pixel_base.
__device__ __forceinline__ int job_of(const FrameJob *__restrict__ jobs, int n_jobs, uint32_t p) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].pixel_base <= p) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Primary rays of every job, one thread per pixel: job-major, row-major in
// each job's rect. ray_job[i] records the job of ray i.
__global__ void k_raygen_jobs(const FrameJob *__restrict__ jobs, int n_jobs, uint32_t total, int sample, float4 *__restrict__ rays,
                              RayPayload *__restrict__ pay, uint32_t *__restrict__ ray_job, uint32_t *__restrict__ count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *count = total;
    if (i >= total) return;
    const int j = job_of(jobs, n_jobs, i);
    const FrameJob &J = jobs[j];
    const uint32_t li = i - J.pixel_base;
    const int x = J.rx + (int)(li % (uint32_t)J.rw), y = J.ry + (int)(li / (uint32_t)J.rw);
    ray_job[i] = (uint32_t)j;
    if (J.geo.on) {
        // k_geo_rays writes this pixel's ray and hit; where the trace runs for
        // other jobs of the launch, this ray (tmax 0) hits nothing
        rays[2ull * i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        rays[2ull * i + 1] = make_float4(0.0f, 0.0f, 1.0f, __int_as_float((x << 16) | y));
        return;
    }
    float4 r0, r1;
    RayPayload p;
    gen_primary(J.cam, J.k, J.fov_k, J.pi.iteration + sample, x, y, J.w, J.h, J.halton, r0, r1, p);
    rays[2ull * i] = r0;
    rays[2ull * i + 1] = r1;
    pay[i] = p;
}

// ---- Geo (lightmap) cameras: SampleMeshInTextureSpace, CoreRef.cpp:507-603.
// The reference rasterises the mesh's triangles in order into the rect, a
// texel taking the first triangle whose UV-space triangle holds the texel's
// jittered sample point. Here k_geo_cover runs one warp per triangle over the
// texels of its box and keeps the smallest covering triangle per texel
// (atomicMin: the same winner as the first in order), then k_geo_rays
// recomputes the winner's barycentrics per texel and writes the camera ray
// and its hit, the arithmetic as in the reference (contraction off).

// A triangle in texel space: corners t, edges d01 = t0 - t1, d12 = t1 - t2,
// d20 = t2 - t0, signed area, and its box clipped to the rect.
struct GeoTri {
    float t0x, t0y, t1x, t1y, t2x, t2y;
    float d01x, d01y, d12x, d12y, d20x, d20y;
    float area;
    int x0, y0, x1, y1;
};

// The per-triangle part (CoreRef.cpp:530-562); false where the triangle
// samples no texel: its box misses the rect or its area is below FLT_EPS
// (triangles wound clockwise in texel space included).
__device__ __forceinline__ bool geo_setup(const FrameJob &J, uint32_t tri, GeoTri &g) {
    const RenderScene &sc = J.sc;
    const uint32_t uv = J.geo.uv;
    const float sw = (float)J.w, sh = (float)J.h;
    float tx[3], ty[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const VertexRec &v = sc.vertices[sc.vtx_indices[tri * 3u + k]];
        tx[k] = __ldg(&v.t[uv][0]) * sw;
        ty[k] = (1.0f - __ldg(&v.t[uv][1])) * sh;
    }
    g.t0x = tx[0]; g.t0y = ty[0];
    g.t1x = tx[1]; g.t1y = ty[1];
    g.t2x = tx[2]; g.t2y = ty[2];
    float bminx = tx[0], bminy = ty[0], bmaxx = tx[0], bmaxy = ty[0];
#pragma unroll
    for (int k = 1; k < 3; k++) {
        bminx = tx[k] < bminx ? tx[k] : bminx;
        bminy = ty[k] < bminy ? ty[k] : bminy;
        bmaxx = bmaxx < tx[k] ? tx[k] : bmaxx;
        bmaxy = bmaxy < ty[k] ? ty[k] : bmaxy;
    }
    // the box's lower corner truncated, its upper corner rounded half away from zero
    int x0 = (int)bminx, y0 = (int)bminy;
    int x1 = (int)roundf(bmaxx), y1 = (int)roundf(bmaxy);
    const int rx1 = J.rx + J.rw - 1, ry1 = J.ry + J.rh - 1;
    if (x1 < J.rx || y1 < J.ry || x0 > rx1 || y0 > ry1) return false;
    g.x0 = x0 > J.rx ? x0 : J.rx;
    g.y0 = y0 > J.ry ? y0 : J.ry;
    g.x1 = x1 < rx1 ? x1 : rx1;
    g.y1 = y1 < ry1 ? y1 : ry1;
    if (g.x1 < g.x0 || g.y1 < g.y0) return false;
    g.d01x = g.t0x - g.t1x; g.d01y = g.t0y - g.t1y;
    g.d12x = g.t1x - g.t2x; g.d12y = g.t1y - g.t2y;
    g.d20x = g.t2x - g.t0x; g.d20y = g.t2y - g.t0y;
    g.area = g.d01x * g.d20y - g.d20x * g.d01y;
    return g.area >= FLT_EPS_;
}

// Texel (x, y)'s jittered sample point against the triangle (CoreRef.cpp:573-585):
// the unnormalised barycentrics and whether all are >= -FLT_EPS.
__device__ __forceinline__ bool geo_cover(const FrameJob &J, const GeoTri &g, int x, int y, int hi, float &u, float &v, float &w) {
    const int index = y * J.w + x;
    const int hash_val = hash_i(index);
    const float sx = (float)x + frac_modf(__ldg(J.halton + hi + 0) + construct_float((uint32_t)hash_val));
    const float sy = (float)y + frac_modf(__ldg(J.halton + hi + 1) + construct_float((uint32_t)hash_i(hash_val)));
    u = g.d01x * (sy - g.t0y) - g.d01y * (sx - g.t0x);
    v = g.d12x * (sy - g.t1y) - g.d12y * (sx - g.t1x);
    w = g.d20x * (sy - g.t2y) - g.d20y * (sx - g.t2x);
    return u >= -FLT_EPS_ && v >= -FLT_EPS_ && w >= -FLT_EPS_;
}

constexpr int GEO_BLOCK = 256;

// One warp per triangle of job blockIdx.y's mesh; best (one per ray of the
// launch, all ones beforehand) takes the smallest covering triangle.
__global__ void __launch_bounds__(GEO_BLOCK) k_geo_cover(const FrameJob *__restrict__ jobs, int sample, uint32_t *__restrict__ best) {
    const FrameJob &J = jobs[blockIdx.y];
    if (!J.geo.on) return;
    const uint32_t t = (blockIdx.x * GEO_BLOCK + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (t >= J.geo.ntri) return;
    const uint32_t tri = J.geo.tri0 + t;
    GeoTri g;
    if (!geo_setup(J, tri, g)) return;
    const int hi = ((J.pi.iteration + sample) & (HALTON_SEQ_LEN - 1)) * HALTON_COUNT;
    const uint32_t nx = (uint32_t)(g.x1 - g.x0 + 1), n = nx * (uint32_t)(g.y1 - g.y0 + 1);
    for (uint32_t k = lane; k < n; k += 32u) {
        const int x = g.x0 + (int)(k % nx), y = g.y0 + (int)(k / nx);
        float u, v, w;
        if (geo_cover(J, g, x, y, hi, u, v, w))
            atomicMin(best + J.pixel_base + (uint32_t)(y - J.ry) * (uint32_t)J.rw + (uint32_t)(x - J.rx), tri);
    }
}

// The camera ray and hit of every texel of the Geo jobs (CoreRef.cpp:510-521,
// 587-600): a covered texel's surface point p and normal n (interpolated,
// transformed, not normalised) give the ray o = p + n, d = -n and the hit
// (triangle, instance, t = 1, u = w, v = u); an uncovered texel is a miss
// along d = 0. Both with colour 1 and zero differentials.
__global__ void k_geo_rays(const FrameJob *__restrict__ jobs, int n_jobs, uint32_t total, int sample, const uint32_t *__restrict__ best,
                           float4 *__restrict__ rays, RayPayload *__restrict__ pay, float4 *__restrict__ hits, int32_t *__restrict__ obj) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const FrameJob &J = jobs[job_of(jobs, n_jobs, i)];
    if (!J.geo.on) return;
    const uint32_t li = i - J.pixel_base;
    const int x = J.rx + (int)(li % (uint32_t)J.rw), y = J.ry + (int)(li / (uint32_t)J.rw);
    const uint32_t tri = best[i];
    float4 r0 = make_float4(0.0f, 0.0f, 0.0f, MAX_DIST), r1 = make_float4(0.0f, 0.0f, 0.0f, __int_as_float((x << 16) | y));
    float4 hit = make_float4(__int_as_float(-1), MAX_DIST, 0.0f, 0.0f);
    int32_t ob = -1;
    GeoTri g;
    if (tri != 0xffffffffu && geo_setup(J, tri, g)) {
        const int hi = ((J.pi.iteration + sample) & (HALTON_SEQ_LEN - 1)) * HALTON_COUNT;
        float u, v, w;
        geo_cover(J, g, x, y, hi, u, v, w);
        const float inv_area = 1.0f / g.area;
        u *= inv_area;
        v *= inv_area;
        w *= inv_area;
        VertexRec a, b, c;
        load_vertex(J.sc, J.sc.vtx_indices[tri * 3u + 0], a);
        load_vertex(J.sc, J.sc.vtx_indices[tri * 3u + 1], b);
        load_vertex(J.sc, J.sc.vtx_indices[tri * 3u + 2], c);
        float pl[3], nl[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            pl[q] = a.p[q] * v + b.p[q] * w + c.p[q] * u;
            nl[q] = a.n[q] * v + b.n[q] * w + c.n[q] * u;
        }
        const float *xf = J.geo.xf; // TransformPoint, CoreRef.cpp:1619-1623
        float p[3];
#pragma unroll
        for (int q = 0; q < 3; q++) p[q] = xf[4 * q + 0] * pl[0] + xf[4 * q + 1] * pl[1] + xf[4 * q + 2] * pl[2] + xf[4 * q + 3];
        const V3 n = transform_normal(V3{nl[0], nl[1], nl[2]}, J.geo.inv);
        r0 = make_float4(p[0] + n.x, p[1] + n.y, p[2] + n.z, MAX_DIST);
        r1.x = -n.x;
        r1.y = -n.y;
        r1.z = -n.z;
        hit = make_float4(__uint_as_float(tri), 1.0f, w, u);
        ob = (int32_t)J.geo.obj;
    }
    rays[2ull * i] = r0;
    rays[2ull * i + 1] = r1;
    RayPayload pl;
    pl.c[0] = pl.c[1] = pl.c[2] = 1.0f;
    pl.ior = 1.0f;
#pragma unroll
    for (int q = 0; q < 3; q++) pl.do_dx[q] = pl.dd_dx[q] = pl.do_dy[q] = pl.dd_dy[q] = 0.0f;
    pl.ray_depth = 0;
    pl.pad[0] = pl.pad[1] = pl.pad[2] = 0;
    pay[i] = pl;
    hits[i] = hit;
    obj[i] = ob;
}

// Shading of *in_count rays of any jobs (bounce: pass_info_t::bounce, 2 for
// primary rays). PRIMARY: SetPixel into the job's sample buffer, else AddPixel
// with alpha 0. A continuation ray is appended where the path goes on and its
// job traces another bounce. PONLY: every material of every job's scene is
// RAY_MAT_PRINCIPLED (and no scene has the reference's lights), so the
// kernel carries none of the other materials' code.
template <bool PRIMARY, bool REF_LIGHTS, bool PONLY = false>
__global__ void __launch_bounds__(SHADE_BLOCK, REF_LIGHTS ? 3 : 4) k_shade_jobs(const FrameJob *__restrict__ jobs, int sample, int bounce,
                                                            const float4 *__restrict__ rays, const RayPayload *__restrict__ pay,
                                                            const uint32_t *__restrict__ ray_job, const float4 *__restrict__ hits,
                                                            const int32_t *__restrict__ obj, const uint32_t *__restrict__ in_count,
                                                            uint32_t max_rays, float4 *__restrict__ out_rays, RayPayload *__restrict__ out_pay,
                                                            uint32_t *__restrict__ out_job, uint32_t *__restrict__ out_count,
                                                            ShadowQueue shadow, uint32_t *__restrict__ err_out,
                                                            unsigned long long *__restrict__ ray_stats) {
    __shared__ uint2 s_stack[REF_LIGHTS ? trav::SMEM_STACK * SHADE_BLOCK : 1];
    Stack<true> st;
    st.smem = s_stack + threadIdx.x;
    st.sp = 0;
    uint32_t err = 0, nshadow = 0;
    const uint32_t n = min(*in_count, max_rays);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * SHADE_BLOCK; base < n; base += gridDim.x * SHADE_BLOCK) {
        const uint32_t i = base + threadIdx.x;
        bool append = false;
        uint32_t j = 0;
        NewRay nr;
        ShadowReq sr;
        sr.valid = false;
        uint32_t sr_index = 0, sr_rand = 0;
        if (i < n) {
            j = ray_job[i];
            const FrameJob &J = jobs[j];
            const float4 r0 = rays[2ull * i], r1 = rays[2ull * i + 1];
            const RayPayload p = pay[i];
            const uint32_t xy = __float_as_uint(r1.w);
            const int x = (int)(xy >> 16), y = (int)(xy & 0xffffu);
            const int index = y * J.w + x;
            PassInfo pi = J.pi;
            pi.iteration += sample;
            pi.bounce = bounce;
            const int rand_index = (pi.flags & PASS_COHERENT) ? c_sampling_pattern[(y % 8) * 8 + (x % 8)] : index;
            bool emit = false;
            const F4 c = shade_surface<REF_LIGHTS, PONLY>(J.sc, pi, rand_index, J.halton, hits[i], obj[i], r0, r1, p, nr, emit, sr, st, err,
                                                          nshadow);
            sr_index = (uint32_t)index;
            sr_rand = (uint32_t)rand_index;
            append = emit && bounce - 2 < J.bounces;
            if (PRIMARY) {
                J.temp[index] = make_float4(c.x, c.y, c.z, c.w);
                if (J.temp_sh) {
                    // ResetSampleData + SetSampleDir/SetSampleWeight (FramebufferRef.h:69-88)
                    SHData &s = J.temp_sh[index];
                    s.coeff_g[0] = 0.0f;
                    if (emit) {
                        const float SH_Y0 = 0.282094806f, SH_Y1 = 0.488602519f;
                        s.coeff_r[0] = SH_Y0;
                        s.coeff_r[1] = SH_Y1 * nr.r1.y;
                        s.coeff_r[2] = SH_Y1 * nr.r1.z;
                        s.coeff_r[3] = SH_Y1 * nr.r1.x;
                        s.coeff_g[0] = nr.p.c[0];
                    }
                }
            } else {
                float4 acc = J.temp[index];
                acc.x += c.x;
                acc.y += c.y;
                acc.z += c.z;
                acc.w += 0.0f;
                J.temp[index] = acc;
            }
        }
        // warp-aggregated append of the light samples
        const uint32_t ms = __ballot_sync(0xffffffffu, sr.valid);
        if (ms) {
            uint32_t slot = 0;
            const uint32_t leader = __ffs(ms) - 1;
            if (lane == leader) slot = atomicAdd(shadow.count, (uint32_t)__popc(ms));
            slot = __shfl_sync(0xffffffffu, slot, leader) + __popc(ms & ((1u << lane) - 1u));
            if (sr.valid && slot < max_rays) {
                ShadowRec rec;
                rec.o[0] = sr.o.x; rec.o[1] = sr.o.y; rec.o[2] = sr.o.z;
                rec.p2[0] = sr.p2.x; rec.p2[1] = sr.p2.y; rec.p2[2] = sr.p2.z;
                rec.c[0] = sr.contrib.x; rec.c[1] = sr.contrib.y; rec.c[2] = sr.contrib.z;
                rec.index = sr_index;
                rec.job = j;
                rec.rand_index = sr_rand;
                static_cast<ShadowRec *>(shadow.recs)[slot] = rec;
                float4 q0, q1;
                shadow_ray(sr.o, sr.p2, q0, q1);
                shadow.rays[2ull * slot] = q0;
                shadow.rays[2ull * slot + 1] = q1;
                shadow.job[slot] = j;
            }
        }
        // warp-aggregated append of the continuation rays
        const uint32_t m = __ballot_sync(0xffffffffu, append);
        if (m) {
            uint32_t slot = 0;
            const uint32_t leader = __ffs(m) - 1;
            if (lane == leader) slot = atomicAdd(out_count, (uint32_t)__popc(m));
            slot = __shfl_sync(0xffffffffu, slot, leader) + __popc(m & ((1u << lane) - 1u));
            if (append && slot < max_rays) {
                out_rays[2ull * slot] = nr.r0;
                out_rays[2ull * slot + 1] = nr.r1;
                out_pay[slot] = nr.p;
                out_job[slot] = j;
            }
        }
    }
    if (err) atomicOr(err_out, err);
    // rays shaded (each was traced once) and shadow-ray segments traced
    if (ray_stats) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&ray_stats[0], (unsigned long long)n);
        const uint32_t ws = __reduce_add_sync(0xffffffffu, nshadow);
        if (lane == 0 && ws) atomicAdd(&ray_stats[1], (unsigned long long)ws);
    }
}

// Whether the light sample of record i is unblocked, from its shadow ray's
// any-hit result: a miss is; a solid first hit is not; a first hit on a
// non-solid triangle takes ComputeVisibility's walk through the transparent
// layers (CoreRef.cpp:1813-1896), which decides it as the reference does.
__device__ __forceinline__ bool sample_visible(const FrameJob &J, int iteration, int bounce, const float *o, const float *p2,
                                               uint32_t rand_index, float4 hit, Stack<true> &st, uint32_t &err, uint32_t &nshadow) {
    nshadow++;
    const int prim = __float_as_int(hit.x);
    if (prim < 0) return true;
    if ((uint32_t)prim >= J.sc.n_tris) {
        err |= SHADE_ERR_BAD_INDEX;
        return false;
    }
    if (load_tri(J.sc, (uint32_t)prim).ci & TRI_SOLID_BIT) return false;
    const int hi = (iteration & (HALTON_SEQ_LEN - 1)) * HALTON_COUNT + bounce * 2;
    const int rand_hash2 = hash_i(hash_i((int)rand_index));
    return compute_visibility(J.sc, v3(o), v3(p2), J.halton, hi, rand_hash2, st, err, nshadow) > 0.0f;
}

// Adds the colour of each unblocked light sample to its pixel, after the
// colour the shading added (the order the path kernel and the oracle keep).
__global__ void __launch_bounds__(SHADE_BLOCK) k_shadow_apply(const FrameJob *__restrict__ jobs, int sample, int bounce, ShadowQueue q,
                                                              const float4 *__restrict__ hits, uint32_t max_recs,
                                                              uint32_t *__restrict__ err_out, unsigned long long *__restrict__ ray_stats) {
    __shared__ uint2 s_stack[trav::SMEM_STACK * SHADE_BLOCK];
    Stack<true> st;
    st.smem = s_stack + threadIdx.x;
    st.sp = 0;
    uint32_t err = 0, nshadow = 0;
    const uint32_t n = min(*q.count, max_recs);
    const ShadowRec *recs = static_cast<const ShadowRec *>(q.recs);
    for (uint32_t i = blockIdx.x * SHADE_BLOCK + threadIdx.x; i < n; i += gridDim.x * SHADE_BLOCK) {
        const ShadowRec rec = recs[i];
        const FrameJob &J = jobs[rec.job];
        if (sample_visible(J, J.pi.iteration + sample, bounce, rec.o, rec.p2, rec.rand_index, hits[i], st, err, nshadow)) {
            float4 acc = J.temp[rec.index];
            acc.x += rec.c[0];
            acc.y += rec.c[1];
            acc.z += rec.c[2];
            J.temp[rec.index] = acc;
        }
    }
    if (err) atomicOr(err_out, err);
    if (ray_stats) {
        const uint32_t ws = __reduce_add_sync(0xffffffffu, nshadow);
        if ((threadIdx.x & 31u) == 0 && ws) atomicAdd(&ray_stats[1], (unsigned long long)ws);
    }
}

// Accumulation and tone of every job's rect, one thread per pixel.
__global__ void k_resolve_jobs(const FrameJob *__restrict__ jobs, int n_jobs, uint32_t total, int sample) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const FrameJob &J = jobs[job_of(jobs, n_jobs, i)];
    const uint32_t li = i - J.pixel_base;
    const int x = J.rx + (int)(li % (uint32_t)J.rw), y = J.ry + (int)(li / (uint32_t)J.rw);
    const size_t idx = (size_t)y * J.w + x;
    const float mix_k = 1.0f / (J.pi.iteration + sample); // RendererRef.cpp:293
    if (J.temp_sh) {
        SHData s = J.temp_sh[idx];
        resolve_pixel(J.temp[idx], J.clean, J.fin, &s, J.clean_sh, idx, mix_k, J.srgb, J.gamma, J.clamp);
        J.temp_sh[idx] = s;
    } else {
        resolve_pixel(J.temp[idx], J.clean, J.fin, nullptr, nullptr, idx, mix_k, J.srgb, J.gamma, J.clamp);
    }
}

// The path kernel: one thread follows one pixel's path through ray
// generation, every bounce (closest hit, shading, shadow rays) and the
// accumulation, with the same arithmetic as the wavefront kernels, so both
// give the same image. Warps take 32 pixels at a time from *work across all
// jobs of the launch.
__device__ __forceinline__ void render_path(const FrameJob &J, uint32_t i, int iteration, Stack<true> &st, uint32_t &err,
                                            uint32_t &nshadow, uint32_t &nrays) {
    const int x = J.rx + (int)(i % (uint32_t)J.rw), y = J.ry + (int)(i / (uint32_t)J.rw);
    const int index = y * J.w + x;
    float4 r0, r1;
    RayPayload pay;
    gen_primary(J.cam, J.k, J.fov_k, iteration, x, y, J.w, J.h, J.halton, r0, r1, pay);
    const int rand_index = (J.pi.flags & PASS_COHERENT) ? c_sampling_pattern[(y % 8) * 8 + (x % 8)] : index;
    PassInfo pi = J.pi;
    pi.iteration = iteration;
    pi.bounce = 2;
    Best b = trace_closest_scene(J.sc.sv, r0, r1, st, err);
    nrays++;
    NewRay nr;
    bool emit = false;
    ShadowReq sr;
    const int rand_hash2 = hash_i(hash_i(rand_index));
    F4 c = shade_surface<true>(J.sc, pi, rand_index, J.halton,
                               make_float4(__int_as_float(b.prim), b.t, b.prim >= 0 ? b.u : 0.0f, b.prim >= 0 ? b.v : 0.0f), b.obj, r0, r1, pay,
                               nr, emit, sr, st, err, nshadow);
    float4 acc = make_float4(c.x, c.y, c.z, c.w);
    // a light sample adds after the shading's colour, as k_shadow_apply does
    if (sr.valid && compute_visibility(J.sc, sr.o, sr.p2, J.halton, (iteration & (HALTON_SEQ_LEN - 1)) * HALTON_COUNT + pi.bounce * 2,
                                       rand_hash2, st, err, nshadow) > 0.0f) {
        acc.x += sr.contrib.x;
        acc.y += sr.contrib.y;
        acc.z += sr.contrib.z;
    }
    SHData s;
    if (J.temp_sh) {
        // ResetSampleData + SetSampleDir/SetSampleWeight (FramebufferRef.h:69-88)
        s = J.temp_sh[index];
        s.coeff_g[0] = 0.0f;
        if (emit) {
            const float SH_Y0 = 0.282094806f, SH_Y1 = 0.488602519f;
            s.coeff_r[0] = SH_Y0;
            s.coeff_r[1] = SH_Y1 * nr.r1.y;
            s.coeff_r[2] = SH_Y1 * nr.r1.z;
            s.coeff_r[3] = SH_Y1 * nr.r1.x;
            s.coeff_g[0] = nr.p.c[0];
        }
    }
    for (int bounce = 0; bounce < J.bounces && emit; bounce++) {
        r0 = nr.r0;
        r1 = nr.r1;
        pay = nr.p;
        b = trace_closest_scene(J.sc.sv, r0, r1, st, err);
        nrays++;
        pi.bounce = bounce + 3;
        c = shade_surface<true>(J.sc, pi, rand_index, J.halton,
                                make_float4(__int_as_float(b.prim), b.t, b.prim >= 0 ? b.u : 0.0f, b.prim >= 0 ? b.v : 0.0f), b.obj, r0, r1,
                                pay, nr, emit, sr, st, err, nshadow);
        acc.x += c.x;
        acc.y += c.y;
        acc.z += c.z;
        acc.w += 0.0f;
        if (sr.valid && compute_visibility(J.sc, sr.o, sr.p2, J.halton, (iteration & (HALTON_SEQ_LEN - 1)) * HALTON_COUNT + pi.bounce * 2,
                                           rand_hash2, st, err, nshadow) > 0.0f) {
            acc.x += sr.contrib.x;
            acc.y += sr.contrib.y;
            acc.z += sr.contrib.z;
        }
    }
    J.temp[index] = acc;
    const float mix_k = 1.0f / iteration; // RendererRef.cpp:293
    if (J.temp_sh) {
        resolve_pixel(acc, J.clean, J.fin, &s, J.clean_sh, (size_t)index, mix_k, J.srgb, J.gamma, J.clamp);
        J.temp_sh[index] = s;
    } else {
        resolve_pixel(acc, J.clean, J.fin, nullptr, nullptr, (size_t)index, mix_k, J.srgb, J.gamma, J.clamp);
    }
}

__global__ void __launch_bounds__(SHADE_BLOCK) k_render_paths(const FrameJob *__restrict__ jobs, int n_jobs, uint32_t total,
                                                              uint32_t *__restrict__ work, uint32_t *__restrict__ err_out,
                                                              unsigned long long *__restrict__ ray_stats) {
    __shared__ uint2 s_stack[trav::SMEM_STACK * SHADE_BLOCK];
    Stack<true> st;
    st.smem = s_stack + threadIdx.x;
    st.sp = 0;
    uint32_t err = 0, nshadow = 0, nrays = 0;
    const uint32_t lane = threadIdx.x & 31u;
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(work, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        const uint32_t p = base + lane;
        if (p < total) {
            int lo = 0, hi = n_jobs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (jobs[mid].pixel_base <= p) lo = mid;
                else hi = mid - 1;
            }
            const FrameJob &J = jobs[lo];
            for (int k = 0; k < J.samples; k++) render_path(J, p - J.pixel_base, J.pi.iteration + k, st, err, nshadow, nrays);
        }
    }
    if (err) atomicOr(err_out, err);
    if (ray_stats) {
        const uint32_t wr = __reduce_add_sync(0xffffffffu, nrays), ws = __reduce_add_sync(0xffffffffu, nshadow);
        if (lane == 0 && wr) atomicAdd(&ray_stats[0], (unsigned long long)wr);
        if (lane == 0 && ws) atomicAdd(&ray_stats[1], (unsigned long long)ws);
    }
}

__global__ void k_fill(float4 *buf, size_t n, float4 v) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) buf[i] = v;
}

__global__ void k_fill_sh(SHData *buf, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        SHData z;
        for (int j = 0; j < 4; j++) z.coeff_r[j] = z.coeff_g[j] = z.coeff_b[j] = 0.0f;
        buf[i] = z;
    }
}

// ---- the path-replay adjoint
//
// Path replay backpropagation (Vicini, Speierer and Jakob 2021) with detached
// sampling: each sample's path is traced again with the same random numbers
// and shaded by the same code as the forward pass; at a vertex with
// differentiable parameters the gradient of the pixel's loss takes
//   * the light sample: d_image . beta . Le . s . d(f cos)/dp, when its shadow
//     ray is unblocked (beta: the path weight, s: its estimator scale);
//   * the continuation: d_image . R . (d(f cos)/dp) / (f cos) per channel,
//     with R = (the sample's radiance) - (what the path summed through this
//     vertex), the radiance that arrived through the continuation. The sum is
//     kept in the order the forward pass summed it, so R is exact up to the
//     one subtraction. It is settled when the continuation ray is shaded (or,
//     the path having ended, never: R = 0).
// Sampling pdfs and MIS weights are held constant (detached), which keeps the
// estimator of the gradient of the expected image unbiased.

// d alpha / d roughness of make_params (alpha = max(r^2, 1e-4)).
__device__ __forceinline__ float dalpha_drough(float r) { return r * r > 1.0e-4f ? 2.0f * r : 0.0f; }

__device__ __forceinline__ void scatter_albedo(const RenderScene &sc, float *grad, float u, float v, float g0, float g1, float g2) {
    if (g0 == 0.0f && g1 == 0.0f && g2 == 0.0f) return;
    const ggx::Bilinear b = ggx::bilinear_at(sc.diff_aw, sc.diff_ah, u, v);
    const float w[4] = {(1.0f - b.kx) * (1.0f - b.ky), b.kx * (1.0f - b.ky), (1.0f - b.kx) * b.ky, b.kx * b.ky};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (w[k] == 0.0f) continue;
        float *t = grad + ((size_t)b.iy[k >> 1] * sc.diff_aw + b.ix[k & 1]) * 3;
        atomicAdd(t + 0, g0 * w[k]);
        atomicAdd(t + 1, g1 * w[k]);
        atomicAdd(t + 2, g2 * w[k]);
    }
}

__device__ __forceinline__ float safe_ratio(float a, float b) { return b != 0.0f ? a / b : 0.0f; }

__device__ __forceinline__ void flush_slots(float *s_gr, float *grad_rough, uint32_t n_slots) {
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n_slots; k += blockDim.x)
        if (s_gr[k] != 0.0f) atomicAdd(grad_rough + k, s_gr[k]);
}

// REF_LIGHTS: the scene has the reference's point/spot/directional lights
// (the replayed shading traces their shadow rays again, as the forward did).
template <bool PRIMARY, bool REF_LIGHTS, bool PONLY = false>
__global__ void __launch_bounds__(SHADE_BLOCK, 3) k_adjoint_shade(const FrameJob *__restrict__ jobs, int bounce,
                                                                  const float4 *__restrict__ rays, const RayPayload *__restrict__ pay,
                                                                  const uint32_t *__restrict__ ray_job, const AdjState *__restrict__ adj_in,
                                                                  const float4 *__restrict__ hits, const int32_t *__restrict__ obj,
                                                                  const uint32_t *__restrict__ in_count, uint32_t max_rays,
                                                                  float4 *__restrict__ out_rays, RayPayload *__restrict__ out_pay,
                                                                  uint32_t *__restrict__ out_job, AdjState *__restrict__ adj_out,
                                                                  uint32_t *__restrict__ out_count, ShadowQueue shadow, AdjArgs args,
                                                                  uint32_t *__restrict__ err_out) {
    __shared__ float s_gr[ADJ_MAX_SLOTS];
    __shared__ float s_gc[3 * ADJ_MAX_SLOTS]; // the diffuse slots' colour gradients
    __shared__ uint2 s_stack[REF_LIGHTS ? trav::SMEM_STACK * SHADE_BLOCK : 1];
    for (int k = threadIdx.x; k < ADJ_MAX_SLOTS; k += blockDim.x) s_gr[k] = 0.0f;
    for (int k = threadIdx.x; k < 3 * ADJ_MAX_SLOTS; k += blockDim.x) s_gc[k] = 0.0f;
    __syncthreads();
    Stack<true> st;
    st.smem = s_stack + (REF_LIGHTS ? threadIdx.x : 0);
    st.sp = 0;
    uint32_t err = 0, nshadow = 0;
    const uint32_t n = min(*in_count, max_rays);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n_slots = jobs[0].sc.n_diff_rough < (uint32_t)ADJ_MAX_SLOTS ? jobs[0].sc.n_diff_rough : (uint32_t)ADJ_MAX_SLOTS;
    for (uint32_t base = blockIdx.x * SHADE_BLOCK; base < n; base += gridDim.x * SHADE_BLOCK) {
        const uint32_t i = base + threadIdx.x;
        bool append = false, light = false;
        uint32_t j = 0;
        NewRay nr;
        ShadowReq sr;
        sr.valid = false;
        AdjState out;
        AdjShadowRec rec;
        if (i < n) {
            j = ray_job[i];
            const FrameJob &J = jobs[j];
            const RenderScene &sc = J.sc;
            const float4 r0 = rays[2ull * i], r1 = rays[2ull * i + 1];
            const RayPayload p = pay[i];
            const uint32_t xy = __float_as_uint(r1.w);
            const int x = (int)(xy >> 16), y = (int)(xy & 0xffffu);
            const int index = y * J.w + x;
            const size_t px = (size_t)j * ((size_t)J.w * J.h) + (size_t)index;
            const float d0 = args.d_image[3ull * index + 0] * args.inv_spp, d1 = args.d_image[3ull * index + 1] * args.inv_spp,
                        d2 = args.d_image[3ull * index + 2] * args.inv_spp;
            float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
            if (!PRIMARY) {
                const AdjState in = adj_in[i];
                a0 = in.a[0];
                a1 = in.a[1];
                a2 = in.a[2];
                const uint32_t in_slot = in.slot & ~ADJ_DIFFUSE_SLOT;
                if (in.slot != RAY_INVALID_INDEX && in_slot < n_slots) { // the previous vertex's continuation: R = radiance - sum so far
                    const float R0 = args.sample_rgb[3 * px + 0] - a0, R1 = args.sample_rgb[3 * px + 1] - a1,
                                R2 = args.sample_rgb[3 * px + 2] - a2;
                    if (in.slot & ADJ_DIFFUSE_SLOT) { // a diffuse slot's main colour
                        const float g0 = d0 * R0 * in.ga[0], g1 = d1 * R1 * in.ga[1], g2 = d2 * R2 * in.ga[2];
                        if (g0 != 0.0f) atomicAdd(&s_gc[3 * in_slot + 0], g0);
                        if (g1 != 0.0f) atomicAdd(&s_gc[3 * in_slot + 1], g1);
                        if (g2 != 0.0f) atomicAdd(&s_gc[3 * in_slot + 2], g2);
                    } else {
                        scatter_albedo(sc, args.grad_albedo, in.u, in.v, d0 * R0 * in.ga[0], d1 * R1 * in.ga[1], d2 * R2 * in.ga[2]);
                    }
                    const float g = d0 * R0 * in.gr[0] + d1 * R1 * in.gr[1] + d2 * R2 * in.gr[2];
                    if (g != 0.0f) atomicAdd(&s_gr[in_slot], g);
                }
            }
            PassInfo pi = J.pi;
            pi.bounce = bounce;
            const int rand_index = (pi.flags & PASS_COHERENT) ? c_sampling_pattern[(y % 8) * 8 + (x % 8)] : index;
            bool emit = false;
            VertexGrad vg;
            const F4 c = shade_surface<REF_LIGHTS, PONLY>(sc, pi, rand_index, J.halton, hits[i], obj[i], r0, r1, p, nr, emit, sr, st, err,
                                                          nshadow, &vg);
            // the sum as the sample buffer takes it (SetPixel on camera rays, AddPixel after)
            if (PRIMARY) {
                a0 = c.x;
                a1 = c.y;
                a2 = c.z;
            } else {
                a0 += c.x;
                a1 += c.y;
                a2 += c.z;
            }
            append = emit && bounce - 2 < J.bounces;
            out.a[0] = a0;
            out.a[1] = a1;
            out.a[2] = a2;
            out.slot = RAY_INVALID_INDEX;
            out.u = out.v = 0.0f;
            out.ga[0] = out.ga[1] = out.ga[2] = out.gr[0] = out.gr[1] = out.gr[2] = 0.0f;
            const bool dv = vg.valid && vg.slot < n_slots;
            const float dadr = dv ? dalpha_drough(vg.rough) : 0.0f;
            if (append && dv && vg.cont) {
                V3 f, dfb, dfa;
                ggx::eval_grad(vg.prm, vg.metallic, vg.wo_l, vg.wi_l, f, dfb, dfa);
                out.slot = vg.slot;
                out.u = vg.u;
                out.v = vg.v;
                out.ga[0] = safe_ratio(dfb.x, f.x) * vg.main_color.x;
                out.ga[1] = safe_ratio(dfb.y, f.y) * vg.main_color.y;
                out.ga[2] = safe_ratio(dfb.z, f.z) * vg.main_color.z;
                out.gr[0] = safe_ratio(dfa.x, f.x) * dadr;
                out.gr[1] = safe_ratio(dfa.y, f.y) * dadr;
                out.gr[2] = safe_ratio(dfa.z, f.z) * dadr;
            }
            if (vg.diffuse && vg.slot < n_slots) {
                // a diffuse vertex: the direct light it added (ray.c x direct x albedo) ...
                const float pc0 = d0 * p.c[0], pc1 = d1 * p.c[1], pc2 = d2 * p.c[2];
                const V3 alb = vg.albedo_on ? v3(vg.tex.x * vg.main_color.x, vg.tex.y * vg.main_color.y, vg.tex.z * vg.main_color.z)
                                            : v3(1.0f, 1.0f, 1.0f);
                if (vg.albedo_on) {
                    const float g0 = pc0 * vg.direct.x * vg.tex.x, g1 = pc1 * vg.direct.y * vg.tex.y, g2 = pc2 * vg.direct.z * vg.tex.z;
                    if (g0 != 0.0f) atomicAdd(&s_gc[3 * vg.slot + 0], g0);
                    if (g1 != 0.0f) atomicAdd(&s_gc[3 * vg.slot + 1], g1);
                    if (g2 != 0.0f) atomicAdd(&s_gc[3 * vg.slot + 2], g2);
                }
                const float gs = pc0 * vg.d_direct.x * alb.x + pc1 * vg.d_direct.y * alb.y + pc2 * vg.d_direct.z * alb.z;
                if (gs != 0.0f) atomicAdd(&s_gr[vg.slot], gs);
                // ... and its continuation, settled at the next vertex: weight = Oren-Nayar x albedo
                if (append && vg.cont) {
                    out.slot = vg.slot | ADJ_DIFFUSE_SLOT;
                    out.ga[0] = vg.albedo_on && vg.main_color.x != 0.0f ? 1.0f / vg.main_color.x : 0.0f;
                    out.ga[1] = vg.albedo_on && vg.main_color.y != 0.0f ? 1.0f / vg.main_color.y : 0.0f;
                    out.ga[2] = vg.albedo_on && vg.main_color.z != 0.0f ? 1.0f / vg.main_color.z : 0.0f;
                    out.gr[0] = out.gr[1] = out.gr[2] = vg.cont_g;
                }
            }
            if (sr.valid) {
                light = true;
                rec.o[0] = sr.o.x; rec.o[1] = sr.o.y; rec.o[2] = sr.o.z;
                rec.p2[0] = sr.p2.x; rec.p2[1] = sr.p2.y; rec.p2[2] = sr.p2.z;
                rec.nee[0] = sr.contrib.x; rec.nee[1] = sr.contrib.y; rec.nee[2] = sr.contrib.z;
                rec.ga[0] = rec.ga[1] = rec.ga[2] = rec.gr = 0.0f;
                rec.u = vg.u;
                rec.v = vg.v;
                rec.slot = RAY_INVALID_INDEX;
                if (dv && vg.light) {
                    V3 f, dfb, dfa;
                    ggx::eval_grad(vg.prm, vg.metallic, vg.wo_l, vg.wl_l, f, dfb, dfa);
                    // d(beta . Le . s . f cos) with d_image folded in
                    const float k0 = d0 * p.c[0] * vg.le_s.x, k1 = d1 * p.c[1] * vg.le_s.y, k2 = d2 * p.c[2] * vg.le_s.z;
                    rec.ga[0] = k0 * dfb.x * vg.main_color.x;
                    rec.ga[1] = k1 * dfb.y * vg.main_color.y;
                    rec.ga[2] = k2 * dfb.z * vg.main_color.z;
                    rec.gr = (k0 * dfa.x + k1 * dfa.y + k2 * dfa.z) * dadr;
                    rec.slot = vg.slot;
                }
                rec.job = j;
                rec.rand_index = (uint32_t)rand_index;
                rec.index = (uint32_t)index;
            }
        }
        // continuation rays first (their slots go into the light samples)
        uint32_t cont = RAY_INVALID_INDEX;
        const uint32_t m = __ballot_sync(0xffffffffu, append);
        if (m) {
            uint32_t slot = 0;
            const uint32_t leader = __ffs(m) - 1;
            if (lane == leader) slot = atomicAdd(out_count, (uint32_t)__popc(m));
            slot = __shfl_sync(0xffffffffu, slot, leader) + __popc(m & ((1u << lane) - 1u));
            if (append && slot < max_rays) {
                out_rays[2ull * slot] = nr.r0;
                out_rays[2ull * slot + 1] = nr.r1;
                out_pay[slot] = nr.p;
                out_job[slot] = j;
                adj_out[slot] = out;
                cont = slot;
            }
        }
        const uint32_t ml = __ballot_sync(0xffffffffu, light);
        if (ml) {
            uint32_t slot = 0;
            const uint32_t leader = __ffs(ml) - 1;
            if (lane == leader) slot = atomicAdd(shadow.count, (uint32_t)__popc(ml));
            slot = __shfl_sync(0xffffffffu, slot, leader) + __popc(ml & ((1u << lane) - 1u));
            if (light && slot < max_rays) {
                rec.cont = cont;
                static_cast<AdjShadowRec *>(shadow.recs)[slot] = rec;
                float4 q0, q1;
                shadow_ray(v3(rec.o), v3(rec.p2), q0, q1);
                shadow.rays[2ull * slot] = q0;
                shadow.rays[2ull * slot + 1] = q1;
                shadow.job[slot] = j;
            }
        }
    }
    if (err) atomicOr(err_out, err);
    flush_slots(s_gr, args.grad_rough, n_slots);
    if (args.grad_color)
        for (uint32_t k = threadIdx.x; k < 3 * n_slots; k += blockDim.x)
            if (s_gc[k] != 0.0f) atomicAdd(args.grad_color + k, s_gc[k]);
}

__global__ void __launch_bounds__(SHADE_BLOCK) k_adjoint_shadow_apply(const FrameJob *__restrict__ jobs, int bounce, ShadowQueue q,
                                                                      const float4 *__restrict__ hits, uint32_t max_recs,
                                                                      AdjState *__restrict__ adj_cont, AdjArgs args,
                                                                      uint32_t *__restrict__ err_out) {
    __shared__ float s_gr[ADJ_MAX_SLOTS];
    __shared__ uint2 s_stack[trav::SMEM_STACK * SHADE_BLOCK];
    for (int k = threadIdx.x; k < ADJ_MAX_SLOTS; k += blockDim.x) s_gr[k] = 0.0f;
    __syncthreads();
    Stack<true> st;
    st.smem = s_stack + threadIdx.x;
    st.sp = 0;
    uint32_t err = 0, nshadow = 0;
    const uint32_t n = min(*q.count, max_recs);
    const uint32_t n_slots = jobs[0].sc.n_diff_rough < (uint32_t)ADJ_MAX_SLOTS ? jobs[0].sc.n_diff_rough : (uint32_t)ADJ_MAX_SLOTS;
    const AdjShadowRec *recs = static_cast<const AdjShadowRec *>(q.recs);
    for (uint32_t i = blockIdx.x * SHADE_BLOCK + threadIdx.x; i < n; i += gridDim.x * SHADE_BLOCK) {
        const AdjShadowRec rec = recs[i];
        const FrameJob &J = jobs[rec.job];
        if (sample_visible(J, J.pi.iteration, bounce, rec.o, rec.p2, rec.rand_index, hits[i], st, err, nshadow)) {
            if (rec.slot < n_slots) {
                scatter_albedo(J.sc, args.grad_albedo, rec.u, rec.v, rec.ga[0], rec.ga[1], rec.ga[2]);
                if (rec.gr != 0.0f) atomicAdd(&s_gr[rec.slot], rec.gr);
            }
            if (rec.cont != RAY_INVALID_INDEX) { // the sum goes on with the light sample, as in the forward pass
                AdjState &a = adj_cont[rec.cont];
                a.a[0] += rec.nee[0];
                a.a[1] += rec.nee[1];
                a.a[2] += rec.nee[2];
            }
        }
    }
    if (err) atomicOr(err_out, err);
    flush_slots(s_gr, args.grad_rough, n_slots);
}

// image = (sum over samples of the sample buffers) / n, and each sample's RGB.
__global__ void k_diff_collect(const FrameJob *__restrict__ jobs, int n_jobs, uint32_t n_pix, float *__restrict__ image,
                               float *__restrict__ sample_rgb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pix) return;
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
    for (int k = 0; k < n_jobs; k++) {
        const float4 t = jobs[k].temp[i];
        float *o = sample_rgb + 3 * ((size_t)k * n_pix + i);
        o[0] = t.x;
        o[1] = t.y;
        o[2] = t.z;
        if (k == 0) {
            s0 = t.x;
            s1 = t.y;
            s2 = t.z;
        } else {
            s0 += t.x;
            s1 += t.y;
            s2 += t.z;
        }
    }
    const float inv = 1.0f / (float)n_jobs;
    image[3ull * i + 0] = s0 * inv;
    image[3ull * i + 1] = s1 * inv;
    image[3ull * i + 2] = s2 * inv;
}

} // namespace

cudaError_t launch_halton_table(const uint16_t *perms, int base_iteration, float *table, cudaStream_t st) {
    k_halton_table<<<(HALTON_COUNT * HALTON_SEQ_LEN + 255) / 256, 256, 0, st>>>(perms, base_iteration, table);
    return cudaGetLastError();
}

cudaError_t launch_raygen_jobs(const FrameJob *jobs, int n_jobs, uint32_t total, int sample, float4 *rays, RayPayload *pay,
                               uint32_t *ray_job, uint32_t *count, cudaStream_t st) {
    if (total == 0) return cudaSuccess;
    k_raygen_jobs<<<(total + 255) / 256, 256, 0, st>>>(jobs, n_jobs, total, sample, rays, pay, ray_job, count);
    return cudaGetLastError();
}

cudaError_t launch_geo_cover(const FrameJob *jobs, int n_jobs, uint32_t max_tris, int sample, uint32_t *best, cudaStream_t st) {
    if (max_tris == 0 || n_jobs == 0) return cudaSuccess;
    const uint64_t threads = (uint64_t)max_tris * 32u;
    k_geo_cover<<<dim3((unsigned)((threads + GEO_BLOCK - 1) / GEO_BLOCK), (unsigned)n_jobs), GEO_BLOCK, 0, st>>>(jobs, sample, best);
    return cudaGetLastError();
}

cudaError_t launch_geo_rays(const FrameJob *jobs, int n_jobs, uint32_t total, int sample, const uint32_t *best, float4 *rays, RayPayload *pay,
                            float4 *hits, int32_t *obj, cudaStream_t st) {
    if (total == 0) return cudaSuccess;
    k_geo_rays<<<(total + 255) / 256, 256, 0, st>>>(jobs, n_jobs, total, sample, best, rays, pay, hits, obj);
    return cudaGetLastError();
}

// Resident blocks of a kernel on this device (one multiple of the SM count).
template <typename K>
static int resident_blocks(K kernel, int fallback_per_sm) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SHADE_BLOCK, 0);
    return (sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : fallback_per_sm);
}

cudaError_t launch_shade_jobs(const FrameJob *jobs, int sample, int bounce, const float4 *rays, const RayPayload *pay, const uint32_t *ray_job,
                              const float4 *hits, const int32_t *obj, const uint32_t *in_count, uint32_t max_rays, float4 *out_rays,
                              RayPayload *out_pay, uint32_t *out_job, uint32_t *out_count, const ShadowQueue &shadow, bool ref_lights,
                              bool principled_only, uint32_t *err, unsigned long long *ray_stats, cudaStream_t st) {
    const bool ponly = principled_only && !ref_lights;
    static int resident[3] = {0, 0, 0};
    int &res = resident[ref_lights ? 1 : (ponly ? 2 : 0)];
    if (res == 0)
        res = ref_lights ? resident_blocks(k_shade_jobs<false, true>, 4)
                         : (ponly ? resident_blocks(k_shade_jobs<false, false, true>, 4) : resident_blocks(k_shade_jobs<false, false>, 4));
    const uint32_t need = (max_rays + SHADE_BLOCK - 1) / SHADE_BLOCK;
    const uint32_t blocks = need < (uint32_t)res ? (need > 0 ? need : 1) : (uint32_t)res;
#define RG_SHADE(P, R, O)                                                                                                                  \
    k_shade_jobs<P, R, O><<<blocks, SHADE_BLOCK, 0, st>>>(jobs, sample, bounce, rays, pay, ray_job, hits, obj, in_count, max_rays, out_rays, \
                                                          out_pay, out_job, out_count, shadow, err, ray_stats)
    if (bounce == 2) {
        if (ref_lights) RG_SHADE(true, true, false);
        else if (ponly) RG_SHADE(true, false, true);
        else RG_SHADE(true, false, false);
    } else {
        if (ref_lights) RG_SHADE(false, true, false);
        else if (ponly) RG_SHADE(false, false, true);
        else RG_SHADE(false, false, false);
    }
#undef RG_SHADE
    return cudaGetLastError();
}

cudaError_t launch_shadow_apply(const FrameJob *jobs, int sample, int bounce, const ShadowQueue &shadow, const float4 *hits, uint32_t max_recs,
                                uint32_t *err, unsigned long long *ray_stats, cudaStream_t st) {
    static int resident = 0;
    if (resident == 0) resident = resident_blocks(k_shadow_apply, 4);
    if (max_recs == 0) return cudaSuccess;
    const uint32_t need = (max_recs + SHADE_BLOCK - 1) / SHADE_BLOCK;
    const uint32_t blocks = need < (uint32_t)resident ? need : (uint32_t)resident;
    k_shadow_apply<<<blocks, SHADE_BLOCK, 0, st>>>(jobs, sample, bounce, shadow, hits, max_recs, err, ray_stats);
    return cudaGetLastError();
}

cudaError_t launch_resolve_jobs(const FrameJob *jobs, int n_jobs, uint32_t total, int sample, cudaStream_t st) {
    if (total == 0) return cudaSuccess;
    k_resolve_jobs<<<(total + 255) / 256, 256, 0, st>>>(jobs, n_jobs, total, sample);
    return cudaGetLastError();
}

cudaError_t launch_render_paths(const FrameJob *jobs, int n_jobs, uint32_t total_pixels, uint32_t *work, uint32_t *err,
                                unsigned long long *ray_stats, cudaStream_t st) {
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render_paths, SHADE_BLOCK, 0);
        blocks = (sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 2);
    }
    if (total_pixels == 0 || n_jobs <= 0) return cudaSuccess;
    const uint32_t need = (total_pixels + SHADE_BLOCK - 1) / SHADE_BLOCK;
    const uint32_t grid = need < (uint32_t)blocks ? need : (uint32_t)blocks;
    k_render_paths<<<grid, SHADE_BLOCK, 0, st>>>(jobs, n_jobs, total_pixels, work, err, ray_stats);
    return cudaGetLastError();
}

cudaError_t launch_diff_collect(const FrameJob *jobs, int n_jobs, uint32_t n_pix, float *image, float *sample_rgb, cudaStream_t st) {
    if (n_pix == 0 || n_jobs <= 0) return cudaSuccess;
    k_diff_collect<<<(n_pix + 255) / 256, 256, 0, st>>>(jobs, n_jobs, n_pix, image, sample_rgb);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_shade(const FrameJob *jobs, int bounce, const float4 *rays, const RayPayload *pay, const uint32_t *ray_job,
                                 const AdjState *adj_in, const float4 *hits, const int32_t *obj, const uint32_t *in_count, uint32_t max_rays,
                                 float4 *out_rays, RayPayload *out_pay, uint32_t *out_job, AdjState *adj_out, uint32_t *out_count,
                                 const ShadowQueue &shadow, const AdjArgs &args, uint32_t *err, cudaStream_t st, bool ref_lights,
                                 bool principled_only) {
    const bool ponly = principled_only && !ref_lights;
    static int resident[3] = {0, 0, 0};
    if (resident[0] == 0) resident[0] = resident_blocks(k_adjoint_shade<false, false>, 3);
    if (resident[1] == 0) resident[1] = resident_blocks(k_adjoint_shade<false, true>, 3);
    if (resident[2] == 0) resident[2] = resident_blocks(k_adjoint_shade<false, false, true>, 3);
    const int res = resident[ref_lights ? 1 : (ponly ? 2 : 0)];
    const uint32_t need = (max_rays + SHADE_BLOCK - 1) / SHADE_BLOCK;
    const uint32_t blocks = need < (uint32_t)res ? (need > 0 ? need : 1) : (uint32_t)res;
#define RG_ADJ(P, L, O)                                                                                                                 \
    k_adjoint_shade<P, L, O><<<blocks, SHADE_BLOCK, 0, st>>>(jobs, bounce, rays, pay, ray_job, adj_in, hits, obj, in_count, max_rays,       \
                                                             out_rays, out_pay, out_job, adj_out, out_count, shadow, args, err)
    if (bounce == 2) {
        if (ref_lights) RG_ADJ(true, true, false);
        else if (ponly) RG_ADJ(true, false, true);
        else RG_ADJ(true, false, false);
    } else {
        if (ref_lights) RG_ADJ(false, true, false);
        else if (ponly) RG_ADJ(false, false, true);
        else RG_ADJ(false, false, false);
    }
#undef RG_ADJ
    return cudaGetLastError();
}

cudaError_t launch_adjoint_shadow_apply(const FrameJob *jobs, int bounce, const ShadowQueue &shadow, const float4 *hits, uint32_t max_recs,
                                        AdjState *adj_cont, const AdjArgs &args, uint32_t *err, cudaStream_t st) {
    static int resident = 0;
    if (resident == 0) resident = resident_blocks(k_adjoint_shadow_apply, 3);
    if (max_recs == 0) return cudaSuccess;
    const uint32_t need = (max_recs + SHADE_BLOCK - 1) / SHADE_BLOCK;
    const uint32_t blocks = need < (uint32_t)resident ? need : (uint32_t)resident;
    k_adjoint_shadow_apply<<<blocks, SHADE_BLOCK, 0, st>>>(jobs, bounce, shadow, hits, max_recs, adj_cont, args, err);
    return cudaGetLastError();
}

cudaError_t launch_fill(float4 *buf, size_t n, float4 v, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_fill<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(buf, n, v);
    return cudaGetLastError();
}

cudaError_t launch_fill_sh(SHData *buf, size_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_fill_sh<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(buf, n);
    return cudaGetLastError();
}

} // namespace rg
