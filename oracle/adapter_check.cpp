// Test infrastructure: one scene built through the Ray library's own interface
// (SceneBase calls only), rendered by the reference's Ref renderer
// (Ray::CreateRenderer, src/Ray/RendererFactory.h:19) and by this library
// through include/raygpu_ray.hpp; prints the image difference as one JSON line.
// Built by oracle/Makefile from the reference's headers and objects where they
// lie, linked with libraygpu.so.
//
//   adapter_check <w> <h> <iterations> <mode> [scene.json]
//   mode 0: the built-in scene, perspective camera; 1: the same, lightmap camera;
//   2: the scene description scene.json read by the demo's own loader
//      (LoadScene, src/DemoLib/load/Load.cpp) for each renderer (paths in it
//      relative to the working directory)

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <ostream>
#include <vector>

#include "Ray/RendererFactory.h"
#include "raygpu_ray.hpp"

#ifdef RB_WITH_LOADER
#include <fstream>
#include <sstream>

#include "load/Load.h"
#endif

namespace {

// a quad (p0 p1 p2 p3, normal n) as PxyzNxyzTuvTuv rows, its second UV layer in atlas cell `cell` of 4 x 4
void quad(std::vector<float> &v, std::vector<uint32_t> &idx, const float p[4][3], const float n[3], int cell) {
    const float uv[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
    const uint32_t base = (uint32_t)(v.size() / 10);
    for (int k = 0; k < 4; k++) {
        v.insert(v.end(), {p[k][0], p[k][1], p[k][2], n[0], n[1], n[2], uv[k][0], uv[k][1]});
        v.push_back(((cell % 4) + 0.05f + uv[k][0] * 0.9f) / 4.0f);
        v.push_back(((cell / 4) + 0.05f + uv[k][1] * 0.9f) / 4.0f);
    }
    for (uint32_t t : {0u, 1u, 2u, 0u, 2u, 3u}) idx.push_back(base + t);
}

void build(Ray::SceneBase &s, bool geo) {
    Ray::environment_desc_t env;
    env.env_col[0] = 0.05f, env.env_col[1] = 0.06f, env.env_col[2] = 0.08f;
    s.SetEnvironment(env);
    const Ray::pixel_color8_t white = {255, 255, 255, 255};
    Ray::tex_desc_t td;
    td.data = &white;
    td.w = td.h = 1;
    td.generate_mipmaps = false;
    const uint32_t tex = s.AddTexture(td);
    Ray::mat_desc_t m;
    m.type = Ray::DiffuseMaterial;
    m.main_texture = tex;
    const float cols[5][3] = {{0.7f, 0.7f, 0.7f}, {0.7f, 0.7f, 0.7f}, {0.6f, 0.6f, 0.5f}, {0.7f, 0.2f, 0.2f}, {0.2f, 0.7f, 0.2f}};
    uint32_t mats[7];
    for (int k = 0; k < 5; k++) {
        m.main_color[0] = cols[k][0], m.main_color[1] = cols[k][1], m.main_color[2] = cols[k][2];
        mats[k] = s.AddMaterial(m);
    }
    Ray::mat_desc_t g;
    g.type = Ray::GlossyMaterial;
    g.main_texture = tex;
    g.roughness = 0.2f;
    mats[5] = s.AddMaterial(g);
    Ray::mat_desc_t e;
    e.type = Ray::EmissiveMaterial;
    e.main_texture = tex;
    e.strength = 12.0f;
    mats[6] = s.AddMaterial(e);

    std::vector<float> v;
    std::vector<uint32_t> idx;
    std::vector<Ray::shape_desc_t> shapes;
    const float walls[5][4][3] = {{{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}},
                                  {{0, 1, 0}, {0, 1, 1}, {1, 1, 1}, {1, 1, 0}},
                                  {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}},
                                  {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}},
                                  {{1, 0, 0}, {1, 1, 0}, {1, 1, 1}, {1, 0, 1}}};
    const float wn[5][3] = {{0, 1, 0}, {0, -1, 0}, {0, 0, -1}, {1, 0, 0}, {-1, 0, 0}};
    for (int k = 0; k < 5; k++) {
        const size_t start = idx.size();
        quad(v, idx, walls[k], wn[k], k);
        shapes.emplace_back(mats[k], mats[k], start, idx.size() - start);
    }
    // a glossy block: its four sides and top
    const float bx0 = 0.55f, bx1 = 0.8f, bz0 = 0.5f, bz1 = 0.75f, by = 0.4f;
    const float block[5][4][3] = {{{bx0, 0, bz0}, {bx0, by, bz0}, {bx1, by, bz0}, {bx1, 0, bz0}},
                                  {{bx1, 0, bz1}, {bx1, by, bz1}, {bx0, by, bz1}, {bx0, 0, bz1}},
                                  {{bx0, 0, bz1}, {bx0, by, bz1}, {bx0, by, bz0}, {bx0, 0, bz0}},
                                  {{bx1, 0, bz0}, {bx1, by, bz0}, {bx1, by, bz1}, {bx1, 0, bz1}},
                                  {{bx0, by, bz0}, {bx0, by, bz1}, {bx1, by, bz1}, {bx1, by, bz0}}};
    const float bn[5][3] = {{0, 0, -1}, {0, 0, 1}, {-1, 0, 0}, {1, 0, 0}, {0, 1, 0}};
    {
        const size_t start = idx.size();
        for (int k = 0; k < 5; k++) quad(v, idx, block[k], bn[k], 5 + k);
        shapes.emplace_back(mats[5], mats[5], start, idx.size() - start);
    }
    const float lamp[4][3] = {{0.35f, 0.999f, 0.35f}, {0.35f, 0.999f, 0.65f}, {0.65f, 0.999f, 0.65f}, {0.65f, 0.999f, 0.35f}};
    const float ln[3] = {0, -1, 0};
    {
        const size_t start = idx.size();
        quad(v, idx, lamp, ln, 10);
        shapes.emplace_back(mats[6], mats[6], start, idx.size() - start);
    }
    Ray::mesh_desc_t md;
    md.prim_type = Ray::TriangleList;
    md.layout = Ray::PxyzNxyzTuvTuv;
    md.vtx_attrs = v.data();
    md.vtx_attrs_count = v.size() / 10;
    md.vtx_indices = idx.data();
    md.vtx_indices_count = idx.size();
    md.shapes = shapes;
    const uint32_t mesh = s.AddMesh(md);
    const float eye[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    s.AddMeshInstance(mesh, eye);

    Ray::light_desc_t l;
    l.type = Ray::PointLight;
    l.position[0] = 0.3f, l.position[1] = 0.8f, l.position[2] = 0.4f;
    l.radius = 0.05f;
    l.color[0] = l.color[1] = l.color[2] = 1.5f;
    l.direction[0] = l.direction[2] = 0.0f, l.direction[1] = -1.0f;
    l.angle = 0.0f;
    s.AddLight(l);

    Ray::camera_desc_t c;
    if (geo) {
        c.type = Ray::Geo;
        c.mi_index = 0;
        c.uv_index = 1;
        c.output_sh = true;
    } else {
        c.type = Ray::Persp;
        c.filter = Ray::Tent;
        c.dtype = Ray::SRGB;
        c.origin[0] = 0.5f, c.origin[1] = 0.5f, c.origin[2] = -1.0f;
        c.fwd[0] = 0.0f, c.fwd[1] = 0.0f, c.fwd[2] = 1.0f;
        c.up[0] = 0.0f, c.up[1] = 1.0f, c.up[2] = 0.0f;
        c.fov = 45.0f;
        c.clamp = true;
    }
    c.gamma = 1.0f;
    c.max_total_depth = c.max_diff_depth = c.max_glossy_depth = 4;
    c.termination_start_depth = 4;
    s.set_current_cam(s.AddCamera(c));
}

std::vector<Ray::pixel_color_t> render(Ray::RendererBase &r, int w, int h, int iterations, int mode, const char *json, uint32_t &tris) {
    std::shared_ptr<Ray::SceneBase> s;
    if (mode == 2) {
#ifdef RB_WITH_LOADER
        std::ifstream f(json, std::ios::binary);
        std::stringstream text;
        text << f.rdbuf();
        JsObject js;
        if (!js.Read(text)) return {};
        s = LoadScene(&r, js);
#endif
        if (!s) return {};
    } else {
        s = r.CreateScene();
        build(*s, mode == 1);
    }
    tris = s->triangle_count();
    r.Clear();
    Ray::RegionContext reg({0, 0, w, h});
    for (int k = 0; k < iterations; k++) r.RenderScene(s, reg);
    const Ray::pixel_color_t *p = r.get_pixels_ref();
    return std::vector<Ray::pixel_color_t>(p, p + (size_t)w * h);
}

} // namespace

int main(int argc, char **argv) {
    const int w = argc > 1 ? std::atoi(argv[1]) : 96, h = argc > 2 ? std::atoi(argv[2]) : 80;
    const int iterations = argc > 3 ? std::atoi(argv[3]) : 4;
    const int mode = argc > 4 ? std::atoi(argv[4]) : 0;
    const char *json = argc > 5 ? argv[5] : "";
    Ray::settings_t st;
    st.w = w;
    st.h = h;
    std::ostream log(nullptr);
    auto ref = Ray::CreateRenderer(st, Ray::RendererRef, log);
    std::shared_ptr<Ray::RendererBase> gpu;
    try {
        gpu = Ray::Gpu::CreateRenderer(st);
    } catch (const std::exception &ex) {
        std::printf("{\"error\": \"%s\"}\n", ex.what());
        return 2;
    }
    uint32_t tr = 0, tg = 0;
    const auto a = render(*ref, w, h, iterations, mode, json, tr);
    const auto b = render(*gpu, w, h, iterations, mode, json, tg);
    if (a.empty() || a.size() != b.size()) {
        std::printf("{\"error\": \"no scene\"}\n");
        return 3;
    }
    double se = 0.0, mean = 0.0;
    size_t same = 0;
    for (size_t i = 0; i < a.size(); i++) {
        const float da[4] = {a[i].r, a[i].g, a[i].b, a[i].a}, db[4] = {b[i].r, b[i].g, b[i].b, b[i].a};
        bool eq = true;
        for (int k = 0; k < 4; k++) {
            eq = eq && da[k] == db[k];
            if (k < 3) {
                se += (double(da[k]) - db[k]) * (double(da[k]) - db[k]);
                mean += db[k];
            }
        }
        same += eq ? 1 : 0;
    }
    const double n = (double)a.size();
    const auto sz = gpu->size();
    std::printf("{\"rmse\": %.9g, \"identical_px\": %.6f, \"mean\": %.6f, \"tris_ref\": %u, \"tris_gpu\": %u, \"type\": %d, \"w\": %d, "
                "\"h\": %d, \"sh\": %d}\n",
                std::sqrt(se / (3.0 * n)), same / n, mean / (3.0 * n), tr, tg, (int)gpu->type(), sz.first, sz.second,
                gpu->get_sh_data_ref() != nullptr ? 1 : 0);
    return 0;
}
