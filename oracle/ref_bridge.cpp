// Accessor for the reference Ray library, compiled together with the
// reference's own sources (src/Ray/_Ray*.cpp, built where they lie) into
// oracle/_ref/libray_ref.so. Test infrastructure only: the tests use it to pin
// the C restatement in ray_oracle.c and the GPU results, and the benchmark's
// reference arm times the reference's CPU traversal through it.
//
// Everything goes through the reference's public API (CreateRenderer,
// SceneBase, RenderScene) except closest-hit tracing, ray sorting and primary
// ray generation, which call the reference's free functions
// (Ref::Traverse_MacroTree_WithStack_ClosestHit, CoreRef.cpp:1133;
// Avx2::Traverse_MacroTree_WithStack_ClosestHit, CoreSIMD.h:1869;
// Ref::SortRays_CPU, CoreRef.cpp:615; Ref::GeneratePrimaryRays, CoreRef.cpp:427)
// on the scene the public API built.

#include <cstring>
#include <functional>
#include <memory>
#include <random>
#include <ostream>
#include <thread>
#include <vector>

#ifdef RB_WITH_LOADER
#include <sstream>
#include <string>

#include "load/Load.h"
#endif

#include "Ray/RendererFactory.h"
#include "Ray/internal/Halton.h"
#include "Ray/internal/RendererAVX2.h"
#include "Ray/internal/SceneRef.h"

namespace {
// Ref::Scene keeps its buffers protected; a derived type may read them.
struct SceneAccess : public Ray::Ref::Scene {
    explicit SceneAccess(bool wide) : Ray::Ref::Scene(wide) {}
    bool wide() const { return use_wide_bvh_; }
    const Ray::mbvh_node_t *mnodes() const { return mnodes_.empty() ? nullptr : mnodes_.data(); }
    const Ray::bvh_node_t *nodes() const { return nodes_.empty() ? nullptr : nodes_.data(); }
    uint32_t macro_root() const { return macro_nodes_root_; }
    const Ray::mesh_instance_t *mesh_instances() const { return mesh_instances_.empty() ? nullptr : mesh_instances_.data(); }
    const uint32_t *mi_indices() const { return mi_indices_.empty() ? nullptr : mi_indices_.data(); }
    const Ray::mesh_t *meshes() const { return meshes_.empty() ? nullptr : meshes_.data(); }
    const Ray::transform_t *transforms() const { return transforms_.empty() ? nullptr : transforms_.data(); }
    const Ray::tri_accel_t *tris() const { return tris_.empty() ? nullptr : tris_.data(); }
    const uint32_t *tri_indices() const { return tri_indices_.empty() ? nullptr : tri_indices_.data(); }
    size_t ntris() const { return tris_.size(); }
    size_t ninst() const { return mesh_instances_.size(); }
};

struct RendererHandle {
    std::shared_ptr<Ray::RendererBase> r;
    std::unique_ptr<Ray::RegionContext> region;
    int w = 0, h = 0;
};

template <typename F>
void parallel_for(int64_t n, int nthreads, F &&f) {
    if (nthreads < 1) nthreads = 1;
    std::vector<std::thread> th;
    const int64_t chunk = (n + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; t++) {
        const int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([=, &f] { f(b, e); });
    }
    for (auto &x : th) x.join();
}
} // namespace

extern "C" {

struct rb_mat_desc {
    int type;
    float main_color[3];
    uint32_t main_texture, normal_map, mix_materials[2];
    float roughness, strength, fresnel, int_ior, ext_ior;
};

struct rb_light_desc {
    int type;
    float position[3], radius, color[3], direction[3], angle;
};

struct rb_camera_desc {
    int type, filter, dtype;
    float origin[3], fwd[3], up[3];
    float fov, gamma, focus_distance, focus_factor;
    uint32_t mi_index, uv_index;
    int lighting_only, skip_direct_lighting, skip_indirect_lighting, no_background, clamp, output_sh, use_coherent_sampling;
    int max_diff_depth, max_glossy_depth, max_refr_depth, max_transp_depth, max_total_depth, termination_start_depth;
};

void *rb_scene_new(int use_wide) { return new std::shared_ptr<SceneAccess>(std::make_shared<SceneAccess>(use_wide != 0)); }
void rb_scene_free(void *s) { delete static_cast<std::shared_ptr<SceneAccess> *>(s); }
static SceneAccess *S(void *s) { return static_cast<std::shared_ptr<SceneAccess> *>(s)->get(); }

uint32_t rb_add_texture(void *s, const uint8_t *rgba, int w, int h, int is_srgb, int gen_mips) {
    Ray::tex_desc_t t;
    t.data = reinterpret_cast<const Ray::pixel_color8_t *>(rgba);
    t.w = w;
    t.h = h;
    t.is_srgb = is_srgb != 0;
    t.generate_mipmaps = gen_mips != 0;
    return S(s)->AddTexture(t);
}

uint32_t rb_add_material(void *s, const rb_mat_desc *d) {
    Ray::mat_desc_t m;
    m.type = Ray::eMaterialType(d->type);
    memcpy(m.main_color, d->main_color, sizeof(m.main_color));
    m.main_texture = d->main_texture;
    m.normal_map = d->normal_map;
    m.mix_materials[0] = d->mix_materials[0];
    m.mix_materials[1] = d->mix_materials[1];
    m.roughness = d->roughness;
    m.strength = d->strength;
    m.fresnel = d->fresnel;
    m.int_ior = d->int_ior;
    m.ext_ior = d->ext_ior;
    return S(s)->AddMaterial(m);
}

// shapes: 4 values each (mat, back_mat, vtx_start, vtx_count)
uint32_t rb_add_mesh(void *s, int layout, const float *attrs, size_t nvtx, const uint32_t *idx, size_t nidx, int base_vertex,
                     const uint32_t *shapes, int nshapes, int fast_bvh) {
    Ray::mesh_desc_t m;
    m.prim_type = Ray::TriangleList;
    m.layout = Ray::eVertexLayout(layout);
    m.vtx_attrs = attrs;
    m.vtx_attrs_count = nvtx;
    m.vtx_indices = idx;
    m.vtx_indices_count = nidx;
    m.base_vertex = base_vertex;
    m.use_fast_bvh_build = fast_bvh != 0;
    for (int i = 0; i < nshapes; i++)
        m.shapes.emplace_back(shapes[4 * i + 0], shapes[4 * i + 1], (size_t)shapes[4 * i + 2], (size_t)shapes[4 * i + 3]);
    return S(s)->AddMesh(m);
}

uint32_t rb_add_instance(void *s, uint32_t mesh, const float *xform) { return S(s)->AddMeshInstance(mesh, xform); }
void rb_remove_instance(void *s, uint32_t i) { S(s)->RemoveMeshInstance(i); }
void rb_set_instance_xform(void *s, uint32_t i, const float *xform) { S(s)->SetMeshInstanceTransform(i, xform); }

uint32_t rb_add_light(void *s, const rb_light_desc *d) {
    Ray::light_desc_t l;
    l.type = Ray::eLightType(d->type);
    memcpy(l.position, d->position, sizeof(l.position));
    l.radius = d->radius;
    memcpy(l.color, d->color, sizeof(l.color));
    memcpy(l.direction, d->direction, sizeof(l.direction));
    l.angle = d->angle;
    return S(s)->AddLight(l);
}

void rb_set_environment(void *s, const float *env_col, float env_clamp, uint32_t env_map) {
    Ray::environment_desc_t e;
    memcpy(e.env_col, env_col, sizeof(e.env_col));
    e.env_clamp = env_clamp;
    e.env_map = env_map;
    S(s)->SetEnvironment(e);
}

static Ray::camera_desc_t to_cam(const rb_camera_desc *d) {
    Ray::camera_desc_t c;
    c.type = Ray::eCamType(d->type);
    c.filter = Ray::eFilterType(d->filter);
    c.dtype = Ray::eDeviceType(d->dtype);
    memcpy(c.origin, d->origin, sizeof(c.origin));
    memcpy(c.fwd, d->fwd, sizeof(c.fwd));
    memcpy(c.up, d->up, sizeof(c.up));
    c.fov = d->fov;
    c.gamma = d->gamma;
    c.focus_distance = d->focus_distance;
    c.focus_factor = d->focus_factor;
    c.mi_index = d->mi_index;
    c.uv_index = d->uv_index;
    c.lighting_only = d->lighting_only != 0;
    c.skip_direct_lighting = d->skip_direct_lighting != 0;
    c.skip_indirect_lighting = d->skip_indirect_lighting != 0;
    c.no_background = d->no_background != 0;
    c.clamp = d->clamp != 0;
    c.output_sh = d->output_sh != 0;
    c.use_coherent_sampling = d->use_coherent_sampling != 0;
    c.max_diff_depth = (uint8_t)d->max_diff_depth;
    c.max_glossy_depth = (uint8_t)d->max_glossy_depth;
    c.max_refr_depth = (uint8_t)d->max_refr_depth;
    c.max_transp_depth = (uint8_t)d->max_transp_depth;
    c.max_total_depth = (uint8_t)d->max_total_depth;
    c.termination_start_depth = (uint8_t)d->termination_start_depth;
    return c;
}

uint32_t rb_add_camera(void *s, const rb_camera_desc *d) { return S(s)->AddCamera(to_cam(d)); }

uint32_t rb_triangle_count(void *s) { return S(s)->triangle_count(); }

// rays: 8 floats per ray (ox, oy, oz, tmax, dx, dy, dz, unused).
// backend 0: scalar Ref traversal; 1: AVX2 packets of 8 rays.
int rb_trace_closest(void *s, const float *rays, int64_t n, int32_t *prim, int32_t *obj, float *tuv, int nthreads, int backend) {
    SceneAccess *sc = S(s);
    if (sc->macro_root() == 0xffffffff) return -1;
    if (backend == 0) {
        parallel_for(n, nthreads, [&](int64_t b, int64_t e) {
            for (int64_t i = b; i < e; i++) {
                Ray::Ref::ray_packet_t r;
                memset(&r, 0, sizeof(r));
                memcpy(r.o, rays + 8 * i, 3 * sizeof(float));
                memcpy(r.d, rays + 8 * i + 4, 3 * sizeof(float));
                Ray::Ref::hit_data_t h;
                h.t = rays[8 * i + 3];
                if (sc->wide())
                    Ray::Ref::Traverse_MacroTree_WithStack_ClosestHit(r, sc->mnodes(), sc->macro_root(), sc->mesh_instances(), sc->mi_indices(),
                                                                      sc->meshes(), sc->transforms(), sc->tris(), sc->tri_indices(), h);
                else
                    Ray::Ref::Traverse_MacroTree_WithStack_ClosestHit(r, sc->nodes(), sc->macro_root(), sc->mesh_instances(), sc->mi_indices(),
                                                                      sc->meshes(), sc->transforms(), sc->tris(), sc->tri_indices(), h);
                prim[i] = h.mask_values[0] ? h.prim_indices[0] : -1;
                if (obj) obj[i] = h.mask_values[0] ? h.obj_indices[0] : -1;
                tuv[3 * i + 0] = h.t;
                tuv[3 * i + 1] = h.mask_values[0] ? h.u : 0.0f;
                tuv[3 * i + 2] = h.mask_values[0] ? h.v : 0.0f;
            }
        });
        return 0;
    }
    const int64_t npk = (n + 7) / 8;
    parallel_for(npk, nthreads, [&](int64_t b, int64_t e) {
        alignas(32) float ox[8], oy[8], oz[8], dx[8], dy[8], dz[8], tm[8];
        alignas(32) int mk[8], pr[8], ob[8];
        alignas(32) float tt[8], uu[8], vv[8];
        for (int64_t p = b; p < e; p++) {
            for (int j = 0; j < 8; j++) {
                const int64_t i = std::min<int64_t>(p * 8 + j, n - 1);
                ox[j] = rays[8 * i + 0]; oy[j] = rays[8 * i + 1]; oz[j] = rays[8 * i + 2]; tm[j] = rays[8 * i + 3];
                dx[j] = rays[8 * i + 4]; dy[j] = rays[8 * i + 5]; dz[j] = rays[8 * i + 6];
            }
            Ray::Avx2::ray_packet_t<8> r;
            r.o[0] = Ray::Avx2::simd_fvec<8>(ox); r.o[1] = Ray::Avx2::simd_fvec<8>(oy); r.o[2] = Ray::Avx2::simd_fvec<8>(oz);
            r.d[0] = Ray::Avx2::simd_fvec<8>(dx); r.d[1] = Ray::Avx2::simd_fvec<8>(dy); r.d[2] = Ray::Avx2::simd_fvec<8>(dz);
            Ray::Avx2::hit_data_t<8> h;
            h.t = Ray::Avx2::simd_fvec<8>(tm);
            const Ray::Avx2::simd_ivec<8> mask = {-1};
            if (sc->wide())
                Ray::Avx2::Traverse_MacroTree_WithStack_ClosestHit<8>(r, mask, sc->mnodes(), sc->macro_root(), sc->mesh_instances(), sc->mi_indices(),
                                                                      sc->meshes(), sc->transforms(), sc->tris(), sc->tri_indices(), h);
            else
                Ray::Avx2::Traverse_MacroTree_WithStack_ClosestHit<8>(r, mask, sc->nodes(), sc->macro_root(), sc->mesh_instances(), sc->mi_indices(),
                                                                      sc->meshes(), sc->transforms(), sc->tris(), sc->tri_indices(), h);
            h.mask.copy_to(mk); h.prim_index.copy_to(pr); h.obj_index.copy_to(ob);
            h.t.copy_to(tt); h.u.copy_to(uu); h.v.copy_to(vv);
            for (int j = 0; j < 8; j++) {
                const int64_t i = p * 8 + j;
                if (i >= n) break;
                prim[i] = mk[j] ? pr[j] : -1;
                if (obj) obj[i] = mk[j] ? ob[j] : -1;
                tuv[3 * i + 0] = tt[j];
                tuv[3 * i + 1] = mk[j] ? uu[j] : 0.0f;
                tuv[3 * i + 2] = mk[j] ? vv[j] : 0.0f;
            }
        }
    });
    return 0;
}

// Runs Ref::SortRays_CPU on rays given as 8 floats (o, tmax, d, unused); the
// ray's input index travels in its xy field, so the reordered rays give the
// permutation. keys_out: the hash values the sort computed (input order).
void rb_sort_rays(const float *rays, int64_t n, const float *root_min, const float *cell, uint32_t *keys_out, uint32_t *perm_out) {
    std::vector<Ray::Ref::ray_packet_t> rp((size_t)n);
    for (int64_t i = 0; i < n; i++) {
        memset(&rp[i], 0, sizeof(rp[i]));
        memcpy(rp[i].o, rays + 8 * i, 3 * sizeof(float));
        memcpy(rp[i].d, rays + 8 * i + 4, 3 * sizeof(float));
        rp[i].xy = (int)i;
    }
    std::vector<uint32_t> hv((size_t)n), sv((size_t)n);
    std::vector<Ray::ray_chunk_t> ch((size_t)n), cht((size_t)n);
    if (n) Ray::Ref::SortRays_CPU(rp.data(), (size_t)n, root_min, cell, hv.data(), sv.data(), ch.data(), cht.data());
    for (int64_t i = 0; i < n; i++) {
        keys_out[i] = hv[i];
        perm_out[i] = (uint32_t)rp[i].xy;
    }
}

void rb_construct_camera(const rb_camera_desc *d, float *out_cam_floats /* fov gamma fd ff origin fwd side up = 16 */) {
    Ray::camera_t cam;
    Ray::ConstructCamera(Ray::eCamType(d->type), Ray::eFilterType(d->filter), Ray::eDeviceType(d->dtype), d->origin, d->fwd, d->up,
                         d->fov, d->gamma, d->focus_distance, d->focus_factor, &cam);
    out_cam_floats[0] = cam.fov; out_cam_floats[1] = cam.gamma;
    out_cam_floats[2] = cam.focus_distance; out_cam_floats[3] = cam.focus_factor;
    memcpy(out_cam_floats + 4, cam.origin, 12);
    memcpy(out_cam_floats + 7, cam.fwd, 12);
    memcpy(out_cam_floats + 10, cam.side, 12);
    memcpy(out_cam_floats + 13, cam.up, 12);
}

// out: 96-byte Ref::ray_packet_t records, rect order
void rb_generate_primary_rays(const rb_camera_desc *d, int iteration, int rx, int ry, int rw, int rh, int w, int h, const float *halton,
                              void *out) {
    Ray::camera_t cam;
    Ray::ConstructCamera(Ray::eCamType(d->type), Ray::eFilterType(d->filter), Ray::eDeviceType(d->dtype), d->origin, d->fwd, d->up,
                         d->fov, d->gamma, d->focus_distance, d->focus_factor, &cam);
    Ray::aligned_vector<Ray::Ref::ray_packet_t> rays;
    Ray::Ref::GeneratePrimaryRays(iteration, cam, Ray::rect_t{rx, ry, rw, rh}, w, h, halton, rays);
    memcpy(out, rays.data(), rays.size() * sizeof(Ray::Ref::ray_packet_t));
}

// The sample table the Ref renderer uses for a given iteration
// (RendererRef.cpp:10-13, 327-358), built with the reference's Halton.h.
void rb_halton_table(int iteration, float *out) {
    auto rand_func = std::bind(std::uniform_int_distribution<int>(), std::mt19937(0));
    std::vector<uint16_t> perms = Ray::ComputeRadicalInversePermutations(Ray::g_primes, Ray::PrimesCount, rand_func);
    static const int primes[24] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89};
    (void)primes;
    for (int i = 0; i < Ray::HALTON_SEQ_LEN; i++) {
        const uint64_t a = (uint64_t)(iteration + i);
        float *o = out + i * 24;
        o[0] = Ray::ScrambledRadicalInverse<2>(&perms[0], a);
        o[1] = Ray::ScrambledRadicalInverse<3>(&perms[2], a);
        o[2] = Ray::ScrambledRadicalInverse<5>(&perms[5], a);
        o[3] = Ray::ScrambledRadicalInverse<7>(&perms[10], a);
        o[4] = Ray::ScrambledRadicalInverse<11>(&perms[17], a);
        o[5] = Ray::ScrambledRadicalInverse<13>(&perms[28], a);
        o[6] = Ray::ScrambledRadicalInverse<17>(&perms[41], a);
        o[7] = Ray::ScrambledRadicalInverse<19>(&perms[58], a);
        o[8] = Ray::ScrambledRadicalInverse<23>(&perms[77], a);
        o[9] = Ray::ScrambledRadicalInverse<29>(&perms[100], a);
        o[10] = Ray::ScrambledRadicalInverse<31>(&perms[129], a);
        o[11] = Ray::ScrambledRadicalInverse<37>(&perms[160], a);
        o[12] = Ray::ScrambledRadicalInverse<41>(&perms[197], a);
        o[13] = Ray::ScrambledRadicalInverse<43>(&perms[238], a);
        o[14] = Ray::ScrambledRadicalInverse<47>(&perms[281], a);
        o[15] = Ray::ScrambledRadicalInverse<53>(&perms[328], a);
        o[16] = Ray::ScrambledRadicalInverse<59>(&perms[381], a);
        o[17] = Ray::ScrambledRadicalInverse<61>(&perms[440], a);
        o[18] = Ray::ScrambledRadicalInverse<67>(&perms[501], a);
        o[19] = Ray::ScrambledRadicalInverse<71>(&perms[568], a);
        o[20] = Ray::ScrambledRadicalInverse<73>(&perms[639], a);
        o[21] = Ray::ScrambledRadicalInverse<79>(&perms[712], a);
        o[22] = Ray::ScrambledRadicalInverse<83>(&perms[791], a);
        o[23] = Ray::ScrambledRadicalInverse<89>(&perms[874], a);
    }
}

void rb_halton_perms(uint16_t *out) {
    auto rand_func = std::bind(std::uniform_int_distribution<int>(), std::mt19937(0));
    std::vector<uint16_t> perms = Ray::ComputeRadicalInversePermutations(Ray::g_primes, Ray::PrimesCount, rand_func);
    memcpy(out, perms.data(), perms.size() * sizeof(uint16_t));
}

// ---- renderer through the public API (CreateRenderer / RenderScene)
// type: Ray::eRendererType bit (1 Ref, 8 AVX2 ...)
void *rb_renderer_new(int type, int w, int h, int use_wide) {
    auto *rh = new RendererHandle;
    Ray::settings_t s;
    s.w = w;
    s.h = h;
    s.use_wide_bvh = use_wide != 0;
    // A stream without a buffer: CreateRenderer's log lines are dropped before
    // they reach the locale machinery, which is not safe to use when the host
    // process carries a second copy of the C++ runtime (a Python interpreter
    // that has loaded numpy, for one).
    std::ostream log(nullptr);
    rh->r = Ray::CreateRenderer(s, (uint32_t)type, log);
    rh->w = w;
    rh->h = h;
    return rh;
}

void rb_renderer_free(void *r) { delete static_cast<RendererHandle *>(r); }

int rb_renderer_type(void *r) { return (int)static_cast<RendererHandle *>(r)->r->type(); }

static void render_scene(RendererHandle *rh, const std::shared_ptr<Ray::SceneBase> &sp, int iterations, int rx, int ry, int rw, int rh_,
                         int reset, int nthreads);

// Renders `iterations` samples over `rect` (w == 0 -> whole image) with one
// RegionContext kept across calls; reset != 0 starts a new context.
void rb_render(void *r, void *s, int iterations, int rx, int ry, int rw, int rh_, int reset, int nthreads) {
    render_scene(static_cast<RendererHandle *>(r), *static_cast<std::shared_ptr<SceneAccess> *>(s), iterations, rx, ry, rw, rh_, reset,
                 nthreads);
}

static void render_scene(RendererHandle *rh, const std::shared_ptr<Ray::SceneBase> &sp, int iterations, int rx, int ry, int rw, int rh_,
                         int reset, int nthreads) {
    if (nthreads <= 1) {
        if (reset || !rh->region) rh->region.reset(new Ray::RegionContext(Ray::rect_t{rx, ry, rw, rh_}));
        for (int i = 0; i < iterations; i++) rh->r->RenderScene(sp, *rh->region);
        return;
    }
    // 64-px buckets on a thread pool, each with its own RegionContext
    // (the pattern of src/DemoLib/states/GSRayTest.cpp:44-66, 199-211).
    const int W = rw ? rw : rh->w, H = rw ? rh_ : rh->h, X0 = rw ? rx : 0, Y0 = rw ? ry : 0;
    std::vector<Ray::rect_t> rects;
    for (int y = 0; y < H; y += 64)
        for (int x = 0; x < W; x += 64) rects.push_back(Ray::rect_t{X0 + x, Y0 + y, std::min(64, W - x), std::min(64, H - y)});
    std::vector<std::unique_ptr<Ray::RegionContext>> ctx;
    for (auto &rc : rects) ctx.emplace_back(new Ray::RegionContext(rc));
    for (int it = 0; it < iterations; it++) {
        parallel_for((int64_t)rects.size(), nthreads, [&](int64_t b, int64_t e) {
            for (int64_t i = b; i < e; i++) rh->r->RenderScene(sp, *ctx[i]);
        });
    }
}

void rb_get_pixels(void *r, float *out) {
    auto *rh = static_cast<RendererHandle *>(r);
    memcpy(out, rh->r->get_pixels_ref(), sizeof(float) * 4 * rh->w * rh->h);
}

// get_sh_data_ref: w * h shl1_data_t (12 floats each); 0 when the renderer holds none.
int rb_get_sh(void *r, float *out) {
    auto *rh = static_cast<RendererHandle *>(r);
    const Ray::shl1_data_t *sh = rh->r->get_sh_data_ref();
    if (!sh) return 0;
    memcpy(out, sh, sizeof(Ray::shl1_data_t) * rh->w * rh->h);
    return 1;
}

void rb_get_stats(void *r, unsigned long long *out6) {
    Ray::RendererBase::stats_t st;
    static_cast<RendererHandle *>(r)->r->GetStats(st);
    memcpy(out6, &st, sizeof(st));
}

void rb_clear(void *r) { static_cast<RendererHandle *>(r)->r->Clear({0, 0, 0, 0}); }

#ifdef RB_WITH_LOADER
// ---- the demo's scene loader (src/DemoLib/load/Load.cpp) and its file readers

// LoadScene (Load.cpp:22-417) on renderer r from JSON text, file paths relative
// to the working directory. Null where the JSON does not parse or LoadScene
// returns null (its own parse errors).
void *rb_load_scene(void *r, const char *json) {
    JsObject js;
    std::stringstream ss{std::string(json)};
    if (!js.Read(ss)) return nullptr;
    std::shared_ptr<Ray::SceneBase> sc;
    try {
        sc = LoadScene(static_cast<RendererHandle *>(r)->r.get(), js);
    } catch (...) {
        return nullptr;
    }
    return sc ? new std::shared_ptr<Ray::SceneBase>(sc) : nullptr;
}

void rb_loaded_free(void *s) { delete static_cast<std::shared_ptr<Ray::SceneBase> *>(s); }

void rb_render_loaded(void *r, void *s, int iterations, int nthreads) {
    render_scene(static_cast<RendererHandle *>(r), *static_cast<std::shared_ptr<Ray::SceneBase> *>(s), iterations, 0, 0, 0, 0, 1, nthreads);
}

static Ray::SceneBase *L(void *s) { return static_cast<std::shared_ptr<Ray::SceneBase> *>(s)->get(); }

// The loaded scene's current camera (GetCamera), environment and counts.
void rb_loaded_camera(void *s, rb_camera_desc *d) {
    Ray::camera_desc_t c;
    L(s)->GetCamera(L(s)->current_cam(), c);
    d->type = c.type;
    d->filter = c.filter;
    d->dtype = c.dtype;
    memcpy(d->origin, c.origin, sizeof(d->origin));
    memcpy(d->fwd, c.fwd, sizeof(d->fwd));
    memcpy(d->up, c.up, sizeof(d->up));
    d->fov = c.fov;
    d->gamma = c.gamma;
    d->focus_distance = c.focus_distance;
    d->focus_factor = c.focus_factor;
    d->clamp = c.clamp;
    d->max_diff_depth = c.max_diff_depth;
    d->max_glossy_depth = c.max_glossy_depth;
    d->max_refr_depth = c.max_refr_depth;
    d->max_transp_depth = c.max_transp_depth;
    d->max_total_depth = c.max_total_depth;
    d->termination_start_depth = c.termination_start_depth;
}

void rb_loaded_environment(void *s, float *env_col, float *env_clamp, uint32_t *env_map) {
    Ray::environment_desc_t e;
    L(s)->GetEnvironment(e);
    memcpy(env_col, e.env_col, 3 * sizeof(float));
    *env_clamp = e.env_clamp;
    *env_map = e.env_map;
}

uint32_t rb_loaded_triangles(void *s) { return L(s)->triangle_count(); }

// The transform of mesh instance i (the Ref renderer's scene type); 0 past the last.
int rb_loaded_instance_xform(void *s, uint32_t i, float *out16) {
    const SceneAccess *a = static_cast<const SceneAccess *>(static_cast<const Ray::Ref::Scene *>(L(s)));
    if (i >= a->ninst()) return 0;
    memcpy(out16, a->transforms()[a->mesh_instances()[i].tr_index].xform, 16 * sizeof(float));
    return 1;
}

// Load_stb_image (Load.cpp:813-831), or LoadHDR (Load.cpp:679-811) with hdr != 0:
// w * h RGBA8 texels into out when cap allows; returns w * h, or -1 on error.
long long rb_load_image(const char *path, int hdr, int *w, int *h, uint8_t *out, size_t cap) {
    std::vector<Ray::pixel_color8_t> px;
    try {
        px = hdr ? LoadHDR(path, *w, *h) : Load_stb_image(path, *w, *h);
    } catch (...) {
        return -1;
    }
    const size_t n = (size_t)(*w) * (*h);
    if (out && cap >= 4 * n && px.size() >= n) memcpy(out, px.data(), 4 * n);
    return (long long)n;
}

// LoadOBJ (Load.cpp:515-634) or LoadBIN (Load.cpp:636-658): the three arrays'
// sizes into sizes[3] and, when the capacities allow, the arrays.
int rb_load_mesh(const char *path, int bin, float *attrs, size_t attrs_cap, uint32_t *idx, size_t idx_cap, uint32_t *groups,
                 size_t groups_cap, size_t *sizes) {
    std::vector<float> a;
    std::vector<unsigned> i, g;
    try {
        std::tie(a, i, g) = bin ? LoadBIN(path) : LoadOBJ(path);
    } catch (...) {
        return -1;
    }
    sizes[0] = a.size();
    sizes[1] = i.size();
    sizes[2] = g.size();
    if (attrs && attrs_cap >= a.size() && !a.empty()) memcpy(attrs, a.data(), a.size() * sizeof(float));
    if (idx && idx_cap >= i.size() && !i.empty()) memcpy(idx, i.data(), i.size() * sizeof(uint32_t));
    if (groups && groups_cap >= g.size() && !g.empty()) memcpy(groups, g.data(), g.size() * sizeof(uint32_t));
    return 0;
}
#endif
}
