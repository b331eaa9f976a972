// Device-side shading of the path tracer: the arithmetic of the reference's
// Ref backend (src/Ray/internal/CoreRef.cpp), restated operation by operation
// in FP32 without contraction (the library is built with --fmad=false), so
// that a hit shades to the same bits as on the CPU wherever the reference
// uses only +, -, *, / and sqrt. cos/sin/acos/pow/tan are evaluated in FP64
// and rounded once to FP32: the correctly rounded value, which libm's float
// functions return for all but a small fraction of arguments.
#pragma once

#include "common.cuh"
#include "render.cuh"

namespace rg {
namespace shade {

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 v3(const float *p) { return V3{p[0], p[1], p[2]}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
// simd_vec dot/length2 accumulate from 0 in component order (simd_vec.h:559-563, 325-329)
__device__ __forceinline__ float dot(V3 a, V3 b) {
    float r = 0.0f;
    r += a.x * b.x;
    r += a.y * b.y;
    r += a.z * b.z;
    return r;
}
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 normalize(V3 a) { return a / length(a); }
// cross, CoreRef.cpp:301-303
__device__ __forceinline__ V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// reflect, CoreRef.cpp:305-307: I - 2 * dot(N, I) * N
__device__ __forceinline__ V3 reflect(V3 i, V3 n) { return i - (2.0f * dot(n, i)) * n; }

__device__ __forceinline__ float fmax_std(float a, float b) { return (a < b) ? b : a; } // std::max
__device__ __forceinline__ float fmin_std(float a, float b) { return (b < a) ? b : a; } // std::min
__device__ __forceinline__ float clampf_ref(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float pow5(float v) { return (v * v) * (v * v) * v; }

// Transcendentals: FP64 evaluation rounded once to FP32.
__device__ __forceinline__ float cr_cos(float x) { return __double2float_rn(cos((double)x)); }
__device__ __forceinline__ float cr_sin(float x) { return __double2float_rn(sin((double)x)); }
__device__ __forceinline__ float cr_acos(float x) { return __double2float_rn(acos((double)x)); }
__device__ __forceinline__ float cr_pow(float x, float y) { return __double2float_rn(pow((double)x, (double)y)); }

// std::modf's fractional part: x - trunc(x) is exact for finite x.
__device__ __forceinline__ float frac_modf(float x) { return x - truncf(x); }

// x86 cvttss2si: NaN or out of range gives INT_MIN.
__device__ __forceinline__ int f2i_x86(float f) {
    if (f != f || f >= 2147483648.0f || f < -2147483648.0f) return (int)0x80000000u;
    return __float2int_rz(f);
}
// simd_vec floor: (float)((int)v - (v < 0)), simd_vec.h:408-412 (floor(-1) is -2)
__device__ __forceinline__ float simd_floor(float v) {
    return (float)(int)((uint32_t)f2i_x86(v) - (v < 0.0f ? 1u : 0u));
}

// hash, CoreRef.cpp:263-269
__device__ __forceinline__ int hash_i(int x) {
    uint32_t r = (uint32_t)x;
    r = ((r >> 16) ^ r) * 0x45d9f3bu;
    r = ((r >> 16) ^ r) * 0x45d9f3bu;
    r = (r >> 16) ^ r;
    return (int)r;
}
// construct_float, CoreRef.cpp:359-368
__device__ __forceinline__ float construct_float(uint32_t m) {
    m &= 0x007FFFFFu;
    m |= 0x3F800000u;
    return __uint_as_float(m) - 1.0f;
}
// to_norm_float, Core.h:249-252
__device__ __forceinline__ float to_norm_float(uint32_t v) {
    const uint32_t val = 0x3f800000u + v * 0x8080u + (v + 1u) / 2u;
    return __uint_as_float(val) - 1.0f;
}
// fast_log2, CoreRef.cpp:391-400
__device__ __forceinline__ float fast_log2(float val) {
    int32_t x = __float_as_int(val);
    float log_2 = (float)(((x >> 23) & 255) - 128);
    x &= ~(255 << 23);
    x += 127 << 23;
    const float v = __int_as_float(x);
    log_2 += ((-0.34484843f) * v + 2.02466578f) * v - 0.67487759f;
    return log_2;
}

// ---- textures. A texture level is stored as its own block of
// (w + 2) x (h + 2) RGBA8 texels with the reference's 1-texel wrap border
// (TextureAtlasTiled::Allocate, TextureAtlasRef.cpp:131-169). Coordinates are
// computed exactly as against the reference's 8192-texel atlas, at the
// position the reference's splitter gives the level, and the block is then
// addressed relative to that position.
constexpr float ATLAS_SIZE = 8192.0f;

__device__ __forceinline__ uint32_t texel(const uint32_t *texels, const TexLevel &lv, int ax, int ay) {
    int x = ax - (int)lv.px, y = ay - (int)lv.py;
    // outside the block only for NaN coordinates or the latlong edge case
    x = x < 0 ? 0 : (x >= (int)lv.pitch ? (int)lv.pitch - 1 : x);
    y = y < 0 ? 0 : (y >= (int)lv.rows ? (int)lv.rows - 1 : y);
    return __ldg(texels + lv.off + (uint32_t)y * lv.pitch + (uint32_t)x);
}

struct F4 {
    float x, y, z, w;
};

// SampleBilinear(atlas, t, uvs, lod), CoreRef.cpp:1652-1678, with TransformUV (:1631-1638)
__device__ __forceinline__ F4 sample_bilinear(const RenderScene &sc, uint32_t tex, float u, float v, int lod) {
    if (tex >= sc.n_textures) return F4{0.0f, 0.0f, 0.0f, 0.0f};
    const TexDev &t = sc.textures[tex];
    lod = lod < 0 ? 0 : (lod > 13 ? 13 : lod);
    const TexLevel lv = t.lv[lod];
    const float posx = (float)lv.px, posy = (float)lv.py;
    const float sizex = (float)((t.width & 0x7FFFu) >> lod), sizey = (float)(t.height >> lod);
    const float fu = u - simd_floor(u), fv = v - simd_floor(v);
    float rx = posx + fu * sizex + 1.0f, ry = posy + fv * sizey + 1.0f;
    rx /= ATLAS_SIZE;
    ry /= ATLAS_SIZE;
    const float ux = rx * ATLAS_SIZE - 0.5f, uy = ry * ATLAS_SIZE - 0.5f;
    const int ix = f2i_x86(ux), iy = f2i_x86(uy);
    const uint32_t p00 = texel(sc.texels, lv, ix + 0, iy + 0), p01 = texel(sc.texels, lv, ix + 1, iy + 0);
    const uint32_t p10 = texel(sc.texels, lv, ix + 0, iy + 1), p11 = texel(sc.texels, lv, ix + 1, iy + 1);
    const float kx = ux - floorf(ux), ky = uy - floorf(uy);
    float c0[4], c1[4], out[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float a00 = (float)((p00 >> (8 * c)) & 0xFFu), a01 = (float)((p01 >> (8 * c)) & 0xFFu);
        const float a10 = (float)((p10 >> (8 * c)) & 0xFFu), a11 = (float)((p11 >> (8 * c)) & 0xFFu);
        c0[c] = a01 * kx + a00 * (1 - kx);
        c1[c] = a11 * kx + a10 * (1 - kx);
        out[c] = (c1[c] * ky + c0[c] * (1.0f - ky)) * (1.0f / 255.0f);
    }
    return F4{out[0], out[1], out[2], out[3]};
}

// rgbe_to_rgb, CoreRef.cpp:370-375 (exp2 of an integer is exact)
__device__ __forceinline__ F4 rgbe_to_rgb(uint32_t p) {
    const float f = ldexpf(1.0f, (int)(p >> 24) - 128);
    return F4{to_norm_float(p & 0xFFu) * f, to_norm_float((p >> 8) & 0xFFu) * f, to_norm_float((p >> 16) & 0xFFu) * f, 1.0f};
}

// SampleLatlong_RGBE, CoreRef.cpp:1772-1798
__device__ __forceinline__ F4 sample_latlong_rgbe(const RenderScene &sc, uint32_t tex, V3 dir) {
    if (tex >= sc.n_textures) return F4{0.0f, 0.0f, 0.0f, 0.0f};
    const TexDev &t = sc.textures[tex];
    const float PI = 3.141592653589793238463f;
    const float theta = cr_acos(clampf_ref(dir.y, -1.0f, 1.0f)) / PI;
    const float r = sqrtf(dir.x * dir.x + dir.z * dir.z);
    float u = 0.5f * cr_acos(r > FLT_EPS_ ? clampf_ref(dir.x / r, -1.0f, 1.0f) : 0.0f) / PI;
    if (dir.z < 0.0f) u = 1.0f - u;
    const TexLevel lv = t.lv[0];
    const float posx = (float)lv.px, posy = (float)lv.py;
    const float sizex = (float)(t.width & 0x7FFFu), sizey = (float)t.height;
    const float ux = posx + u * sizex + 1.0f, uy = posy + theta * sizey + 1.0f;
    const uint32_t p00 = texel(sc.texels, lv, f2i_x86(ux + 0), f2i_x86(uy + 0));
    const uint32_t p01 = texel(sc.texels, lv, f2i_x86(ux + 1), f2i_x86(uy + 0));
    const uint32_t p10 = texel(sc.texels, lv, f2i_x86(ux + 0), f2i_x86(uy + 1));
    const uint32_t p11 = texel(sc.texels, lv, f2i_x86(ux + 1), f2i_x86(uy + 1));
    const float kx = ux - simd_floor(ux), ky = uy - simd_floor(uy);
    const F4 a00 = rgbe_to_rgb(p00), a01 = rgbe_to_rgb(p01), a10 = rgbe_to_rgb(p10), a11 = rgbe_to_rgb(p11);
    F4 o;
    o.x = (a11.x * kx + a10.x * (1 - kx)) * ky + (a01.x * kx + a00.x * (1 - kx)) * (1 - ky);
    o.y = (a11.y * kx + a10.y * (1 - kx)) * ky + (a01.y * kx + a00.y * (1 - kx)) * (1 - ky);
    o.z = (a11.z * kx + a10.z * (1 - kx)) * ky + (a01.z * kx + a00.z * (1 - kx)) * (1 - ky);
    o.w = (a11.w * kx + a10.w * (1 - kx)) * ky + (a01.w * kx + a00.w * (1 - kx)) * (1 - ky);
    return o;
}

// srgb_to_rgb, CoreRef.cpp:377-389
__device__ __forceinline__ F4 srgb_to_rgb(F4 c) {
    float in[3] = {c.x, c.y, c.z}, out[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (in[i] > 0.04045f) out[i] = cr_pow((in[i] + 0.055f) / 1.055f, 2.4f);
        else out[i] = in[i] / 12.92f;
    }
    return F4{out[0], out[1], out[2], c.w};
}

// get_texture_lod, CoreRef.cpp:402-417
__device__ __forceinline__ float texture_lod(const RenderScene &sc, uint32_t tex, float dudx, float dvdx, float dudy, float dvdy) {
    if (tex >= sc.n_textures) return 0.0f;
    const TexDev &t = sc.textures[tex];
    const float szx = (float)(t.width & 0x7FFFu), szy = (float)t.height;
    const float ax = dudx * szx, ay = dvdx * szy, bx = dudy * szx, by = dvdy * szy;
    const float cx = ax + bx, cy = ay + by;
    float la = 0.0f, lb = 0.0f, lc = 0.0f;
    la += ax * ax;
    la += ay * ay;
    lb += bx * bx;
    lb += by * by;
    lc += cx * cx;
    lc += cy * cy;
    const float min_length2 = fmin_std(fmin_std(la, lb), lc);
    float lod = fast_log2(min_length2);
    lod = clampf_ref(0.5f * lod - 1.0f, 0.0f, 13.0f);
    return lod;
}

// BRDF_OrenNayar, CoreRef.cpp:1579-1603
__device__ __forceinline__ float brdf_oren_nayar(V3 L, V3 I, V3 N, V3 T, float sigma) {
    const float sigma_sqr = sigma * sigma;
    const float A = 1.0f - (sigma_sqr / (2.0f * (sigma_sqr + 0.33f)));
    const float B = (0.45f * sigma_sqr) / (sigma_sqr + 0.09f);
    const float cos_theta_I = dot(L, N);
    const float cos_theta_O = -dot(I, N);
    const float sin_theta_I = sqrtf(fmax_std(0.0f, 1.0f - (cos_theta_I * cos_theta_I)));
    const float sin_theta_O = sqrtf(fmax_std(0.0f, 1.0f - (cos_theta_O * cos_theta_O)));
    const float cos_phi_I = dot(L, T);
    const float cos_phi_O = -dot(I, T);
    const float sin_phi_I = sqrtf(fmax_std(0.0f, 1.0f - (cos_phi_I * cos_phi_I)));
    const float sin_phi_O = sqrtf(fmax_std(0.0f, 1.0f - (cos_phi_O * cos_phi_O)));
    const float temp = fmax_std(0.0f, (cos_phi_I * cos_phi_O) + (sin_phi_I * sin_phi_O));
    float sin_alpha, tan_beta;
    if (cos_theta_I > cos_theta_O) {
        sin_alpha = sin_theta_O;
        tan_beta = (sin_theta_I / cos_theta_I);
    } else {
        sin_alpha = sin_theta_I;
        tan_beta = (sin_theta_O / cos_theta_O);
    }
    const float result = (A + (B * temp * sin_alpha * tan_beta));
    return clampf_ref(result, 0.0f, 1.0f);
}

// The same Oren-Nayar factor and its derivative with respect to sigma:
// A = 1 - s^2 / (2 (s^2 + 0.33)), B = 0.45 s^2 / (s^2 + 0.09), so
// dA/ds = -0.33 s / (s^2 + 0.33)^2 and dB/ds = 0.081 s / (s^2 + 0.09)^2;
// where the reference clamps the result to [0, 1] the derivative is 0.
__device__ __forceinline__ float brdf_oren_nayar_d(V3 L, V3 I, V3 N, V3 T, float sigma, float &d_sigma) {
    const float sigma_sqr = sigma * sigma;
    const float A = 1.0f - (sigma_sqr / (2.0f * (sigma_sqr + 0.33f)));
    const float B = (0.45f * sigma_sqr) / (sigma_sqr + 0.09f);
    const float cos_theta_I = dot(L, N);
    const float cos_theta_O = -dot(I, N);
    const float sin_theta_I = sqrtf(fmax_std(0.0f, 1.0f - (cos_theta_I * cos_theta_I)));
    const float sin_theta_O = sqrtf(fmax_std(0.0f, 1.0f - (cos_theta_O * cos_theta_O)));
    const float cos_phi_I = dot(L, T);
    const float cos_phi_O = -dot(I, T);
    const float sin_phi_I = sqrtf(fmax_std(0.0f, 1.0f - (cos_phi_I * cos_phi_I)));
    const float sin_phi_O = sqrtf(fmax_std(0.0f, 1.0f - (cos_phi_O * cos_phi_O)));
    const float temp = fmax_std(0.0f, (cos_phi_I * cos_phi_O) + (sin_phi_I * sin_phi_O));
    float sin_alpha, tan_beta;
    if (cos_theta_I > cos_theta_O) {
        sin_alpha = sin_theta_O;
        tan_beta = (sin_theta_I / cos_theta_I);
    } else {
        sin_alpha = sin_theta_I;
        tan_beta = (sin_theta_O / cos_theta_O);
    }
    const float g = temp * sin_alpha * tan_beta;
    const float result = (A + (B * g));
    const float a2 = sigma_sqr + 0.33f, b2 = sigma_sqr + 0.09f;
    const float dA = -0.33f * sigma / (a2 * a2), dB = 0.081f * sigma / (b2 * b2);
    d_sigma = (result > 0.0f && result < 1.0f) ? dA + dB * g : 0.0f;
    return clampf_ref(result, 0.0f, 1.0f);
}

// ExtractPlaneNormal, Core.cpp:216-228 (the reference scales by the length,
// not its inverse; kept as is)
__device__ __forceinline__ V3 plane_normal(const TriRec &tri) {
    float n[3];
    const int iw = tri.ci & TRI_W_BITS;
    const int nu_i = iw == 0 ? 1 : 0, nv_i = iw == 2 ? 1 : 2;
    n[iw] = 1.0f;
    n[nu_i] = tri.nu;
    n[nv_i] = tri.nv;
    float inv_l = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (tri.ci & TRI_INV_NORMAL_BIT) inv_l = -inv_l;
    return V3{n[0] * inv_l, n[1] * inv_l, n[2] * inv_l};
}

// TransformNormal, CoreRef.cpp:1625-1629. inv: the instance's inverse
// transform as 12 floats, column-major without the last row.
__device__ __forceinline__ V3 transform_normal(V3 n, const float *inv) {
    return V3{inv[0] * n.x + inv[1] * n.y + inv[2] * n.z, inv[3] * n.x + inv[4] * n.y + inv[5] * n.z,
              inv[6] * n.x + inv[7] * n.y + inv[8] * n.z};
}

struct Derivs {
    V3 do_dx, do_dy, dd_dx, dd_dy;
    float duv_dx[2], duv_dy[2];
    V3 dndx, dndy;
    float ddn_dx, ddn_dy;
};

// ComputeDerivatives, CoreRef.cpp:1993-2052
__device__ __forceinline__ void compute_derivatives(V3 I, float t, V3 do_dx, V3 do_dy, V3 dd_dx, V3 dd_dy, const VertexRec &va,
                                                    const VertexRec &vb, const VertexRec &vc, V3 plane_N, Derivs &o) {
    const float dot_I_N = -dot(I, plane_N);
    const float inv_dot = fabsf(dot_I_N) < FLT_EPS_ ? 0.0f : 1.0f / dot_I_N;
    const float dt_dx = dot(do_dx + t * dd_dx, plane_N) * inv_dot;
    const float dt_dy = dot(do_dy + t * dd_dy, plane_N) * inv_dot;

    o.do_dx = (do_dx + t * dd_dx) + dt_dx * I;
    o.do_dy = (do_dy + t * dd_dy) + dt_dy * I;
    o.dd_dx = dd_dx;
    o.dd_dy = dd_dy;

    const float duv13[2] = {va.t[0][0] - vc.t[0][0], va.t[0][1] - vc.t[0][1]};
    const float duv23[2] = {vb.t[0][0] - vc.t[0][0], vb.t[0][1] - vc.t[0][1]};
    const V3 dp13 = v3(va.p) - v3(vc.p), dp23 = v3(vb.p) - v3(vc.p);

    const float det_uv = duv13[0] * duv23[1] - duv13[1] * duv23[0];
    const float inv_det_uv = fabsf(det_uv) < FLT_EPS_ ? 0 : 1.0f / det_uv;
    const V3 dpdu = (duv23[1] * dp13 - duv13[1] * dp23) * inv_det_uv;
    const V3 dpdv = (-duv23[0] * dp13 + duv13[0] * dp23) * inv_det_uv;

    float A00 = dpdu.x, A01 = dpdv.x, A10 = dpdu.y, A11 = dpdv.y;
    float Bx0 = o.do_dx.x, Bx1 = o.do_dx.y, By0 = o.do_dy.x, By1 = o.do_dy.y;
    if (fabsf(plane_N.x) > fabsf(plane_N.y) && fabsf(plane_N.x) > fabsf(plane_N.z)) {
        A00 = dpdu.y; A01 = dpdv.y;
        A10 = dpdu.z; A11 = dpdv.z;
        Bx0 = o.do_dx.y; Bx1 = o.do_dx.z;
        By0 = o.do_dy.y; By1 = o.do_dy.z;
    } else if (fabsf(plane_N.y) > fabsf(plane_N.z)) {
        A10 = dpdu.z; A11 = dpdv.z;
        Bx0 = o.do_dx.x; Bx1 = o.do_dx.z;
        By0 = o.do_dy.x; By1 = o.do_dy.z;
    }

    const float det = A00 * A11 - A01 * A10;
    const float inv_det = fabsf(det) < FLT_EPS_ ? 0 : 1.0f / det;
    o.duv_dx[0] = (A11 * Bx0 - A01 * Bx1) * inv_det;
    o.duv_dx[1] = (A00 * Bx1 - A10 * Bx0) * inv_det;
    o.duv_dy[0] = (A11 * By0 - A01 * By1) * inv_det;
    o.duv_dy[1] = (A00 * By1 - A10 * By0) * inv_det;

    const V3 dn1 = v3(va.n) - v3(vc.n), dn2 = v3(vb.n) - v3(vc.n);
    const V3 dndu = (duv23[1] * dn1 - duv13[1] * dn2) * inv_det_uv;
    const V3 dndv = (-duv23[0] * dn1 + duv13[0] * dn2) * inv_det_uv;

    o.dndx = dndu * o.duv_dx[0] + dndv * o.duv_dx[1];
    o.dndy = dndu * o.duv_dy[0] + dndv * o.duv_dy[1];

    o.ddn_dx = dot(dd_dx, plane_N) + dot(I, o.dndx);
    o.ddn_dy = dot(dd_dy, plane_N) + dot(I, o.dndy);
}

} // namespace shade
} // namespace rg
