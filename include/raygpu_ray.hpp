/* C++ adapter: this library behind the Ray library's own interface,
 * Ray::RendererBase (src/Ray/RendererBase.h:55-103) and Ray::SceneBase
 * (src/Ray/SceneBase.h:157-285), so that code written against that interface
 * -- the demo's states, its scene loader (src/DemoLib/load/Load.cpp), the
 * library's tests -- renders on the GPU unchanged.
 *
 * Header-only. A build that has the Ray library's headers on its include path
 * (and compiles the library's SceneBase.cpp, which holds the camera store)
 * includes this header and links libraygpu.so:
 *
 *     std::shared_ptr<Ray::RendererBase> r = Ray::Gpu::CreateRenderer(settings);
 *     auto scene = r->CreateScene();           // a Ray::Gpu::Scene
 *     ...                                      // SceneBase calls as for any backend
 *     r->RenderScene(scene, region);
 *
 * Behaviour follows the reference's conventions: failures of calls that return
 * nothing are silent, index-returning calls return 0xffffffff, RenderScene with
 * another backend's scene is a no-op (RendererRef.cpp:20-21); ray_last_error()
 * tells what failed. Cameras stay in SceneBase's own store (its camera API is
 * not virtual); RenderScene hands the current camera, as SceneBase constructed
 * it, to the library before each frame.
 */
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <utility>
#include <vector>

#include "Ray/RendererBase.h"
#include "raygpu.h"

namespace Ray {
namespace Gpu {

class Renderer;

class Scene : public SceneBase {
    friend class Renderer;
    ray_scene *h_ = nullptr;
    uint32_t cam_ = 0xffffffff; // the library's camera that mirrors SceneBase's current one

    // SceneBase's current camera_t into the library's camera cam_: the
    // description it was made from, then its constructed axes unchanged.
    void sync_camera() {
        if (current_cam_ == 0xffffffff || current_cam_ >= cams_.size()) return;
        const camera_t &c = cams_[current_cam_].cam;
        ray_camera_desc d;
        std::memset(&d, 0, sizeof(d));
        d.type = (int)c.type;
        d.filter = (int)c.filter;
        d.dtype = (int)c.dtype;
        std::memcpy(d.origin, c.origin, sizeof(d.origin));
        std::memcpy(d.fwd, c.fwd, sizeof(d.fwd));
        std::memcpy(d.up, c.up, sizeof(d.up));
        d.fov = c.fov;
        d.gamma = c.gamma;
        d.focus_distance = c.focus_distance;
        d.focus_factor = c.focus_factor;
        d.mi_index = c.mi_index;
        d.uv_index = c.uv_index;
        const uint32_t f = c.pass_settings.flags;
        d.skip_direct_lighting = (f & SkipDirectLight) != 0;
        d.skip_indirect_lighting = (f & SkipIndirectLight) != 0;
        d.lighting_only = (f & LightingOnly) != 0;
        d.no_background = (f & NoBackground) != 0;
        d.clamp = (f & Clamp) != 0;
        d.output_sh = (f & OutputSH) != 0;
        d.use_coherent_sampling = (f & UseCoherentSampling) != 0;
        d.max_diff_depth = c.pass_settings.max_diff_depth;
        d.max_glossy_depth = c.pass_settings.max_glossy_depth;
        d.max_refr_depth = c.pass_settings.max_refr_depth;
        d.max_transp_depth = c.pass_settings.max_transp_depth;
        d.max_total_depth = c.pass_settings.max_total_depth;
        d.termination_start_depth = c.pass_settings.termination_start_depth;
        // a Geo camera keeps its slot's display type: set it through a perspective description first
        ray_camera_desc p = d;
        p.type = RAY_CAM_PERSP;
        if (cam_ == 0xffffffff) {
            if (ray_scene_add_camera(h_, &p, &cam_) != RAY_OK) return;
        } else {
            ray_scene_set_camera(h_, cam_, &p);
        }
        if (d.type != RAY_CAM_PERSP) ray_scene_set_camera(h_, cam_, &d);
        if (d.type == RAY_CAM_PERSP) ray_scene_set_camera_axes(h_, cam_, c.side, c.up);
        ray_scene_set_current_cam(h_, cam_);
    }

  public:
    explicit Scene(ray_scene *h) : h_(h) {}
    ~Scene() override { ray_destroy_scene(h_); }
    Scene(const Scene &) = delete;
    Scene &operator=(const Scene &) = delete;
    ray_scene *handle() const { return h_; }

    void GetEnvironment(environment_desc_t &env) override {
        ray_environment_desc e;
        if (ray_scene_get_environment(h_, &e) != RAY_OK) return;
        std::memcpy(env.env_col, e.env_col, sizeof(env.env_col));
        env.env_clamp = e.env_clamp;
        env.env_map = e.env_map;
    }
    void SetEnvironment(const environment_desc_t &env) override {
        ray_environment_desc e;
        std::memcpy(e.env_col, env.env_col, sizeof(e.env_col));
        e.env_clamp = env.env_clamp;
        e.env_map = env.env_map;
        ray_scene_set_environment(h_, &e);
    }
    uint32_t AddTexture(const tex_desc_t &t) override {
        ray_tex_desc d{reinterpret_cast<const uint8_t *>(t.data), t.w, t.h, t.is_srgb ? 1 : 0, t.generate_mipmaps ? 1 : 0};
        uint32_t i = 0xffffffff;
        return ray_scene_add_texture(h_, &d, &i) == RAY_OK ? i : 0xffffffff;
    }
    void RemoveTexture(uint32_t i) override { ray_scene_remove_texture(h_, i); }
    uint32_t AddMaterial(const mat_desc_t &m) override {
        ray_mat_desc d;
        std::memset(&d, 0, sizeof(d));
        d.type = (int)m.type;
        std::memcpy(d.main_color, m.main_color, sizeof(d.main_color));
        d.main_texture = m.main_texture;
        d.normal_map = m.normal_map;
        d.mix_materials[0] = m.mix_materials[0];
        d.mix_materials[1] = m.mix_materials[1];
        d.roughness = m.roughness;
        d.strength = m.strength;
        d.fresnel = m.fresnel;
        d.int_ior = m.int_ior;
        d.ext_ior = m.ext_ior;
        uint32_t i = 0xffffffff;
        return ray_scene_add_material(h_, &d, &i) == RAY_OK ? i : 0xffffffff;
    }
    void RemoveMaterial(uint32_t i) override { ray_scene_remove_material(h_, i); }
    uint32_t AddMesh(const mesh_desc_t &m) override {
        std::vector<ray_shape_desc> sh;
        sh.reserve(m.shapes.size());
        for (const shape_desc_t &s : m.shapes) sh.push_back(ray_shape_desc{s.mat_index, s.back_mat_index, s.vtx_start, s.vtx_count});
        ray_mesh_desc d;
        std::memset(&d, 0, sizeof(d));
        d.prim_type = (int)m.prim_type;
        d.layout = (int)m.layout;
        d.vtx_attrs = m.vtx_attrs;
        d.vtx_attrs_count = m.vtx_attrs_count;
        d.vtx_indices = m.vtx_indices;
        d.vtx_indices_count = m.vtx_indices_count;
        d.base_vertex = m.base_vertex;
        d.shapes = sh.empty() ? nullptr : sh.data();
        d.shapes_count = sh.size();
        d.allow_spatial_splits = m.allow_spatial_splits ? 1 : 0;
        d.use_fast_bvh_build = m.use_fast_bvh_build ? 1 : 0;
        uint32_t i = 0xffffffff;
        return ray_scene_add_mesh(h_, &d, &i) == RAY_OK ? i : 0xffffffff;
    }
    void RemoveMesh(uint32_t i) override { ray_scene_remove_mesh(h_, i); }
    uint32_t AddLight(const light_desc_t &l) override {
        ray_light_desc d;
        std::memset(&d, 0, sizeof(d));
        d.type = (int)l.type;
        std::memcpy(d.position, l.position, sizeof(d.position));
        d.radius = l.radius;
        std::memcpy(d.color, l.color, sizeof(d.color));
        std::memcpy(d.direction, l.direction, sizeof(d.direction));
        d.angle = l.angle;
        uint32_t i = 0xffffffff;
        return ray_scene_add_light(h_, &d, &i) == RAY_OK ? i : 0xffffffff;
    }
    void RemoveLight(uint32_t i) override { ray_scene_remove_light(h_, i); }
    uint32_t AddMeshInstance(uint32_t m_index, const float *xform) override {
        uint32_t i = 0xffffffff;
        return ray_scene_add_mesh_instance(h_, m_index, xform, &i) == RAY_OK ? i : 0xffffffff;
    }
    void SetMeshInstanceTransform(uint32_t mi_index, const float *xform) override {
        ray_scene_set_mesh_instance_transform(h_, mi_index, xform);
    }
    void RemoveMeshInstance(uint32_t mi_index) override { ray_scene_remove_mesh_instance(h_, mi_index); }
    uint32_t triangle_count() override {
        uint32_t n = 0;
        ray_scene_triangle_count(h_, &n);
        return n;
    }
    uint32_t node_count() override {
        uint32_t n = 0;
        ray_scene_node_count(h_, &n);
        return n;
    }
};

class Renderer : public RendererBase {
    ray_renderer *h_ = nullptr;

  public:
    // settings_t's use_wide_bvh is accepted and ignored (the GPU builds its own wide BVH)
    explicit Renderer(const settings_t &s, int device = 0) {
        ray_settings rs{s.w, s.h, s.use_wide_bvh ? 1 : 0, device};
        if (ray_create_renderer(&rs, &h_) != RAY_OK) throw std::runtime_error(ray_last_error());
    }
    ~Renderer() override { ray_destroy_renderer(h_); }
    Renderer(const Renderer &) = delete;
    Renderer &operator=(const Renderer &) = delete;
    ray_renderer *handle() const { return h_; }

    // the reference's eRendererType has no GPU entry: this library reports its own bit
    eRendererType type() const override { return eRendererType(RAY_RENDERER_CUDA_SM100); }
    std::pair<int, int> size() const override {
        int w = 0, h = 0;
        ray_renderer_size(h_, &w, &h);
        return std::make_pair(w, h);
    }
    const pixel_color_t *get_pixels_ref() const override {
        const ray_pixel *p = nullptr;
        ray_get_pixels(h_, &p, 0);
        return reinterpret_cast<const pixel_color_t *>(p);
    }
    const shl1_data_t *get_sh_data_ref() const override {
        const ray_shl1 *p = nullptr;
        ray_get_sh_data(h_, &p);
        return reinterpret_cast<const shl1_data_t *>(p);
    }
    void Resize(int w, int h) override { ray_resize(h_, w, h); }
    void Clear(const pixel_color_t &c = {0, 0, 0, 0}) override {
        const ray_pixel p{c.r, c.g, c.b, c.a};
        ray_clear(h_, &p);
    }
    std::shared_ptr<SceneBase> CreateScene() override {
        ray_scene *s = nullptr;
        if (ray_create_scene(h_, &s) != RAY_OK) throw std::runtime_error(ray_last_error());
        return std::make_shared<Scene>(s);
    }
    void RenderScene(const std::shared_ptr<SceneBase> &s, RegionContext &region) override {
        const auto gs = std::dynamic_pointer_cast<Scene>(s);
        if (!gs) return;
        gs->sync_camera();
        const rect_t r = region.rect();
        // the sample table lives on the GPU; region.halton_seq stays unused
        ray_region rr{{r.x, r.y, r.w, r.h}, region.iteration};
        if (ray_render(h_, gs->h_, &rr) == RAY_OK) region.iteration = rr.iteration;
    }
    void GetStats(stats_t &st) override {
        ray_stats s;
        if (ray_get_stats(h_, &s) != RAY_OK) return;
        st.time_primary_ray_gen_us = s.time_primary_ray_gen_us;
        st.time_primary_trace_us = s.time_primary_trace_us;
        st.time_primary_shade_us = s.time_primary_shade_us;
        st.time_secondary_sort_us = s.time_secondary_sort_us;
        st.time_secondary_trace_us = s.time_secondary_trace_us;
        st.time_secondary_shade_us = s.time_secondary_shade_us;
    }
    void ResetStats() override { ray_reset_stats(h_); }
};

// Ray::CreateRenderer (RendererFactory.h:19) for this library: the reference's
// backend flags and log stream have no meaning here; `device` picks the GPU.
inline std::shared_ptr<RendererBase> CreateRenderer(const settings_t &s, int device = 0) { return std::make_shared<Renderer>(s, device); }

} // namespace Gpu
} // namespace Ray
