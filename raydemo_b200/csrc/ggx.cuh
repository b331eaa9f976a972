// RAY_MAT_PRINCIPLED: a metallic-roughness material (Lambert + GGX) with its
// sampler, next-event estimation from quad and sun lights, and multiple
// importance sampling. There is no counterpart in the reference; the CPU
// restatement the tests compare against is orc_render_principled in
// oracle/ray_oracle.c, written from the same formulas in the same order.
//
// Published methods used: the GGX / Trowbridge-Reitz distribution with the
// height-correlated Smith shadowing term (Heitz 2014, "Understanding the
// Masking-Shadowing Function"), sampling of the distribution of visible
// normals (Heitz 2018, "Sampling the GGX Distribution of Visible Normals"),
// Schlick's Fresnel approximation, the branchless orthonormal basis of Duff
// et al. 2017, Veach's power heuristic, and a padded 2D Sobol sequence with
// hash-based Owen scrambling (Burley 2020): the first two Sobol dimensions
// (bit reversal and the Pascal-matrix dimension), each index and coordinate
// scrambled by a nested uniform permutation built from even multiplications
// (each bit depends only on the bits below it), per pixel and dimension pair.
#pragma once

#include "shade.cuh"

namespace rg {
namespace ggx {

using namespace shade;

constexpr float PI_G = 3.141592653589793238463f;
constexpr float INV_PI_G = 0.318309886183790671538f;

// ---- sampler
__device__ __forceinline__ uint32_t mix32(uint32_t x) { return (uint32_t)hash_i((int)x); }

// A nested uniform scramble of the bits of x (most significant first).
__device__ __forceinline__ uint32_t nested_scramble(uint32_t x, uint32_t seed) {
    x = __brev(x);
    x += seed;
    x ^= x * 0x9E3779B8u;
    x ^= x * 0x7F4A7C16u;
    x ^= x * 0x94D049BAu;
    x ^= x * 0x2C1B3C6Eu;
    return __brev(x);
}

// Second Sobol dimension: generator matrix = Pascal's triangle mod 2.
__device__ __forceinline__ uint32_t sobol_dim1(uint32_t i) {
    uint32_t r = 0, v = 0x80000000u;
    for (; i; i >>= 1, v ^= v >> 1)
        if (i & 1u) r ^= v;
    return r;
}

// Sample `index` of the scrambled 2D sequence of a (pixel, dimension pair) seed, in [0, 1)^2.
__device__ __forceinline__ void sobol2(uint32_t index, uint32_t seed, float &x, float &y) {
    const uint32_t i = nested_scramble(index, seed);
    const uint32_t sx = nested_scramble(__brev(i), mix32(seed ^ 0x5bd1e995u));
    const uint32_t sy = nested_scramble(sobol_dim1(i), mix32(seed ^ 0x1b873593u));
    x = (float)(sx >> 8) * (1.0f / 16777216.0f);
    y = (float)(sy >> 8) * (1.0f / 16777216.0f);
}

// Seed of dimension pair `pair` at bounce `bounce` of pixel `pixel`.
__device__ __forceinline__ uint32_t dim_seed(uint32_t pixel, int bounce, int pair) {
    return mix32(mix32(pixel * 0x2545F491u + 0x68E31DA4u) ^ (uint32_t)(bounce * 8 + pair) * 0x9E3779B1u);
}

// ---- material
struct Frame {
    V3 t, b, n;
};
// Duff et al. 2017: an orthonormal basis around a unit vector.
__device__ __forceinline__ Frame make_frame(V3 n) {
    const float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (sign + n.z);
    const float b = n.x * n.y * a;
    Frame f;
    f.t = v3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    f.b = v3(b, sign + n.y * n.y * a, -n.y);
    f.n = n;
    return f;
}
__device__ __forceinline__ V3 to_local(const Frame &f, V3 v) { return v3(dot(v, f.t), dot(v, f.b), dot(v, f.n)); }
__device__ __forceinline__ V3 to_world(const Frame &f, V3 v) { return f.t * v.x + f.b * v.y + f.n * v.z; }

struct Params {
    V3 f0, diffuse;  // specular reflectance at normal incidence, diffuse albedo
    float alpha;     // roughness^2
    float p_spec;    // probability of sampling the specular lobe
};

__device__ __forceinline__ Params make_params(V3 base, float roughness, float metallic) {
    Params p;
    p.f0 = v3(0.04f + (base.x - 0.04f) * metallic, 0.04f + (base.y - 0.04f) * metallic, 0.04f + (base.z - 0.04f) * metallic);
    p.diffuse = base * (1.0f - metallic);
    p.alpha = fmax_std(roughness * roughness, 1.0e-4f);
    p.p_spec = 0.5f + 0.5f * metallic;
    return p;
}

// Smith Lambda of direction v (local frame) for the GGX distribution.
__device__ __forceinline__ float smith_lambda(V3 v, float a) {
    const float t2 = (v.x * v.x + v.y * v.y) / (v.z * v.z);
    return 0.5f * (sqrtf(1.0f + a * a * t2) - 1.0f);
}

__device__ __forceinline__ float ggx_d(V3 h, float a) {
    const float a2 = a * a;
    const float k = h.z * h.z * (a2 - 1.0f) + 1.0f;
    return a2 / (PI_G * k * k);
}

// f(wo, wi) * cos(wi) and the pdf (solid angle) of sampling wi, local frame.
__device__ __forceinline__ void eval(const Params &p, V3 wo, V3 wi, V3 &f_cos, float &pdf) {
    f_cos = v3(0.0f, 0.0f, 0.0f);
    pdf = 0.0f;
    if (wo.z <= 0.0f || wi.z <= 0.0f) return;
    const V3 h = normalize(wo + wi);
    const float d = ggx_d(h, p.alpha);
    const float lo = smith_lambda(wo, p.alpha), li = smith_lambda(wi, p.alpha);
    const float g2 = 1.0f / (1.0f + lo + li);
    const float g1 = 1.0f / (1.0f + lo);
    const float c = 1.0f - fmax_std(dot(wo, h), 0.0f);
    const float c5 = pow5(c);
    const V3 F = v3(p.f0.x + (1.0f - p.f0.x) * c5, p.f0.y + (1.0f - p.f0.y) * c5, p.f0.z + (1.0f - p.f0.z) * c5);
    const float spec = d * g2 / (4.0f * wo.z * wi.z);
    f_cos = (F * spec + p.diffuse * INV_PI_G) * wi.z;
    const float pdf_spec = g1 * d / (4.0f * wo.z);
    const float pdf_diff = wi.z * INV_PI_G;
    pdf = p.p_spec * pdf_spec + (1.0f - p.p_spec) * pdf_diff;
}

// Samples wi (local frame) from the lobe mixture. False: no valid direction.
__device__ __forceinline__ bool sample(const Params &p, V3 wo, float u1, float u2, float ulobe, V3 &wi) {
    if (ulobe < p.p_spec) {
        // visible normals (Heitz 2018)
        const float a = p.alpha;
        const V3 vh = normalize(v3(a * wo.x, a * wo.y, wo.z));
        const float lensq = vh.x * vh.x + vh.y * vh.y;
        const V3 t1 = lensq > 0.0f ? v3(-vh.y, vh.x, 0.0f) / sqrtf(lensq) : v3(1.0f, 0.0f, 0.0f);
        const V3 t2 = cross(vh, t1);
        const float r = sqrtf(u1);
        const float phi = 2.0f * PI_G * u2;
        const float q1 = r * cr_cos(phi);
        float q2 = r * cr_sin(phi);
        const float s = 0.5f * (1.0f + vh.z);
        q2 = (1.0f - s) * sqrtf(1.0f - q1 * q1) + s * q2;
        const V3 nh = t1 * q1 + t2 * q2 + vh * sqrtf(fmax_std(0.0f, 1.0f - q1 * q1 - q2 * q2));
        const V3 h = normalize(v3(a * nh.x, a * nh.y, fmax_std(0.0f, nh.z)));
        wi = h * (2.0f * dot(wo, h)) - wo;
    } else {
        const float r = sqrtf(u1);
        const float phi = 2.0f * PI_G * u2;
        wi = v3(r * cr_cos(phi), r * cr_sin(phi), sqrtf(fmax_std(0.0f, 1.0f - u1)));
    }
    return wi.z > 0.0f;
}

__device__ __forceinline__ float power_heuristic(float a, float b) { return (a * a) / (a * a + b * b); }

// Bilinear texture read at level 0 with wrap-around addressing (the base
// colour of RAY_MAT_PRINCIPLED): texel centres at (i + 0.5) / w. No texture
// (RAY_INVALID_INDEX, the only index past the last texture add_material lets
// through for this material) reads as white.
__device__ __forceinline__ V3 sample_plain(const RenderScene &sc, uint32_t tex, float u, float v) {
    if (tex >= sc.n_textures) return v3(1.0f, 1.0f, 1.0f);
    const TexDev &t = sc.textures[tex];
    const TexLevel lv = t.lv[0];
    const int w = (int)(t.width & 0x7FFFu), h = (int)t.height;
    float fu = u - floorf(u), fv = v - floorf(v);
    if (!(fu >= 0.0f && fu < 1.0f)) fu = 0.0f; // NaN or the rounding of a tiny negative u
    if (!(fv >= 0.0f && fv < 1.0f)) fv = 0.0f;
    const float x = fu * (float)w - 0.5f, y = fv * (float)h - 0.5f;
    const float x0 = floorf(x), y0 = floorf(y);
    const float kx = x - x0, ky = y - y0;
    // block coordinates: the level's texel (i, j) is at (i + 1, j + 1), with wrapped borders
    const int bx = (int)x0 + 1, by = (int)y0 + 1;
    const uint32_t *b = sc.texels + lv.off;
    const uint32_t p00 = __ldg(b + (uint32_t)by * lv.pitch + (uint32_t)bx), p01 = __ldg(b + (uint32_t)by * lv.pitch + (uint32_t)bx + 1u);
    const uint32_t p10 = __ldg(b + (uint32_t)(by + 1) * lv.pitch + (uint32_t)bx), p11 = __ldg(b + (uint32_t)(by + 1) * lv.pitch + (uint32_t)bx + 1u);
    float c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float a00 = (float)((p00 >> (8 * k)) & 0xFFu), a01 = (float)((p01 >> (8 * k)) & 0xFFu);
        const float a10 = (float)((p10 >> (8 * k)) & 0xFFu), a11 = (float)((p11 >> (8 * k)) & 0xFFu);
        const float top = a00 * (1.0f - kx) + a01 * kx, bot = a10 * (1.0f - kx) + a11 * kx;
        c[k] = (top * (1.0f - ky) + bot * ky) * (1.0f / 255.0f);
    }
    V3 r = v3(c[0], c[1], c[2]);
    if (t.width & 0x8000u) {
        const F4 s = srgb_to_rgb(F4{r.x, r.y, r.z, 1.0f});
        r = v3(s.x, s.y, s.z);
    }
    return r;
}

// The four texels and bilinear weights of a wrap-around read of a w x h
// texture at (u, v), texel centres at (i + 0.5) / w: texel k = iy[k >> 1] * w
// + ix[k & 1], weight wt[k].
struct Bilinear {
    uint32_t ix[2], iy[2];
    float kx, ky;
};
__device__ __forceinline__ Bilinear bilinear_at(uint32_t w, uint32_t h, float u, float v) {
    float fu = u - floorf(u), fv = v - floorf(v);
    if (!(fu >= 0.0f && fu < 1.0f)) fu = 0.0f;
    if (!(fv >= 0.0f && fv < 1.0f)) fv = 0.0f;
    const float x = fu * (float)w - 0.5f, y = fv * (float)h - 0.5f;
    const float x0 = floorf(x), y0 = floorf(y);
    Bilinear b;
    b.kx = x - x0;
    b.ky = y - y0;
    const int ix = (int)x0, iy = (int)y0; // -1 .. w - 1
    b.ix[0] = (uint32_t)((ix + (int)w) % (int)w);
    b.ix[1] = (uint32_t)((ix + 1) % (int)w);
    b.iy[0] = (uint32_t)((iy + (int)h) % (int)h);
    b.iy[1] = (uint32_t)((iy + 1) % (int)h);
    return b;
}

// The differentiable albedo (float RGB, h x w x 3) at (u, v).
__device__ __forceinline__ V3 sample_param(const RenderScene &sc, float u, float v) {
    const Bilinear b = bilinear_at(sc.diff_aw, sc.diff_ah, u, v);
    const float *t = sc.diff_albedo;
    const size_t i00 = ((size_t)b.iy[0] * sc.diff_aw + b.ix[0]) * 3, i01 = ((size_t)b.iy[0] * sc.diff_aw + b.ix[1]) * 3;
    const size_t i10 = ((size_t)b.iy[1] * sc.diff_aw + b.ix[0]) * 3, i11 = ((size_t)b.iy[1] * sc.diff_aw + b.ix[1]) * 3;
    float c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float top = __ldg(t + i00 + k) * (1.0f - b.kx) + __ldg(t + i01 + k) * b.kx;
        const float bot = __ldg(t + i10 + k) * (1.0f - b.kx) + __ldg(t + i11 + k) * b.kx;
        c[k] = top * (1.0f - b.ky) + bot * b.ky;
    }
    return v3(c[0], c[1], c[2]);
}

// f * cos of eval() with its derivatives: per channel with respect to the
// base colour (the same channel) and with respect to alpha. Zero where eval
// is zero.
__device__ __forceinline__ void eval_grad(const Params &p, float metallic, V3 wo, V3 wi, V3 &f_cos, V3 &df_dbase, V3 &df_dalpha) {
    f_cos = df_dbase = df_dalpha = v3(0.0f, 0.0f, 0.0f);
    if (wo.z <= 0.0f || wi.z <= 0.0f) return;
    const V3 h = normalize(wo + wi);
    const float a = p.alpha, a2 = a * a;
    const float k = h.z * h.z * (a2 - 1.0f) + 1.0f;
    const float d = a2 / (PI_G * k * k);
    const float dd_da = 2.0f * a * (k - 2.0f * a2 * h.z * h.z) / (PI_G * k * k * k);
    const float to = (wo.x * wo.x + wo.y * wo.y) / (wo.z * wo.z), ti = (wi.x * wi.x + wi.y * wi.y) / (wi.z * wi.z);
    const float so = sqrtf(1.0f + a2 * to), si = sqrtf(1.0f + a2 * ti);
    const float g2 = 1.0f / (1.0f + 0.5f * (so - 1.0f) + 0.5f * (si - 1.0f));
    const float dg2_da = -g2 * g2 * (0.5f * a * to / so + 0.5f * a * ti / si);
    const float c5 = pow5(1.0f - fmax_std(dot(wo, h), 0.0f));
    const float spec = d * g2 / (4.0f * wo.z * wi.z);
    const float dspec = (dd_da * g2 + d * dg2_da) / (4.0f * wo.z * wi.z);
    const float fb = (metallic * (1.0f - c5) * spec + (1.0f - metallic) * INV_PI_G) * wi.z;
    const float f0[3] = {p.f0.x, p.f0.y, p.f0.z}, dif[3] = {p.diffuse.x, p.diffuse.y, p.diffuse.z};
    float fc[3], fa[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float F = f0[c] + (1.0f - f0[c]) * c5;
        fc[c] = (F * spec + dif[c] * INV_PI_G) * wi.z;
        fa[c] = F * dspec * wi.z;
    }
    f_cos = v3(fc[0], fc[1], fc[2]);
    df_dbase = v3(fb, fb, fb);
    df_dalpha = v3(fa[0], fa[1], fa[2]);
}

// Ray against a quad light (front side only); t in (0, tmax) on a hit.
__device__ __forceinline__ bool hit_quad(const AreaLight &l, V3 o, V3 d, float tmax, float &t) {
    const V3 n = v3(l.n);
    const float dn = dot(d, n);
    if (!(dn < 0.0f)) return false;
    t = dot(v3(l.p0) - o, n) / dn;
    if (!(t > 0.0f && t < tmax)) return false;
    const V3 q = o + d * t - v3(l.p0);
    const V3 u = v3(l.u), v = v3(l.v);
    const float s = dot(q, u) / dot(u, u), r = dot(q, v) / dot(v, v);
    return s >= 0.0f && s <= 1.0f && r >= 0.0f && r <= 1.0f;
}

} // namespace ggx
} // namespace rg
