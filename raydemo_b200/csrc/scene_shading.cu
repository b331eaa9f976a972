// Host side of the scene's shading data: texture mip chains and their atlas
// placement, the tangent basis of meshes without one, and the device copies
// the shading kernels read.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>

#include "scene.hpp"

namespace rg {

namespace {

constexpr int ATLAS_RES = 8192;     // TEXTURE_ATLAS_SIZE, Core.h:98
constexpr float FLT_EPS_H = 0.0000001f;

// TextureSplitter::Insert_Recursive (TextureSplitter.cpp:56-100): the same
// guillotine placement, so that every level lands where the reference puts
// it. Returns the node index or -1.
int split_insert(std::vector<SplitNode> &nodes, int i, const int res[2]) {
    if (!nodes[i].is_free || res[0] > nodes[i].size[0] || res[1] > nodes[i].size[1]) return -1;
    if (nodes[i].child[0] != -1) {
        const int c0 = nodes[i].child[0], c1 = nodes[i].child[1];
        const int r = split_insert(nodes, c0, res);
        if (r != -1) return r;
        return split_insert(nodes, c1, res);
    }
    if (res[0] == nodes[i].size[0] && res[1] == nodes[i].size[1]) {
        nodes[i].is_free = false;
        return i;
    }
    const int c0 = (int)nodes.size();
    nodes.emplace_back();
    const int c1 = (int)nodes.size();
    nodes.emplace_back();
    nodes[i].child[0] = c0;
    nodes[i].child[1] = c1;
    const SplitNode n = nodes[i];
    const int dw = n.size[0] - res[0], dh = n.size[1] - res[1];
    if (dw > dh) {
        nodes[c0].pos[0] = n.pos[0];
        nodes[c0].pos[1] = n.pos[1];
        nodes[c0].size[0] = res[0];
        nodes[c0].size[1] = n.size[1];
        nodes[c1].pos[0] = n.pos[0] + res[0];
        nodes[c1].pos[1] = n.pos[1];
        nodes[c1].size[0] = n.size[0] - res[0];
        nodes[c1].size[1] = n.size[1];
    } else {
        nodes[c0].pos[0] = n.pos[0];
        nodes[c0].pos[1] = n.pos[1];
        nodes[c0].size[0] = n.size[0];
        nodes[c0].size[1] = res[1];
        nodes[c1].pos[0] = n.pos[0];
        nodes[c1].pos[1] = n.pos[1] + res[1];
        nodes[c1].size[0] = n.size[0];
        nodes[c1].size[1] = n.size[1] - res[1];
    }
    nodes[c0].parent = nodes[c1].parent = i;
    return split_insert(nodes, c0, res);
}

std::vector<SplitNode> new_page() {
    std::vector<SplitNode> p(1);
    p[0].size[0] = ATLAS_RES;
    p[0].size[1] = ATLAS_RES;
    return p;
}

// TextureAtlasTiled::Allocate (TextureAtlasRef.cpp:131-169): a level of
// w x h texels takes (w + 2) x (h + 2) with its border; pages are tried in
// order and doubled when none has room.
int atlas_allocate(ray_scene *s, int w, int h, int pos[2]) {
    const int res[2] = {w + 2, h + 2};
    if (res[0] > ATLAS_RES || res[1] > ATLAS_RES) return -1;
    if (s->atlas_pages.empty()) s->atlas_pages.push_back(new_page());
    while (true) {
        for (size_t p = 0; p < s->atlas_pages.size(); p++) {
            const int i = split_insert(s->atlas_pages[p], 0, res);
            if (i != -1) {
                pos[0] = s->atlas_pages[p][i].pos[0];
                pos[1] = s->atlas_pages[p][i].pos[1];
                return (int)p;
            }
        }
        const size_t n = s->atlas_pages.size();
        for (size_t k = 0; k < n; k++) s->atlas_pages.push_back(new_page());
    }
}

// DownsampleTexture (TextureUtilsRef.cpp:9-38): 2x2 box filter with integer
// truncation; a level with a side of 1 is passed on unchanged. Reads past the
// end of an odd-sized level (where the reference reads beyond its buffer)
// take the last texel instead.
std::vector<uint32_t> downsample(const std::vector<uint32_t> &tex, int w, int h) {
    if (w == 1 || h == 1) return tex;
    std::vector<uint32_t> out;
    out.reserve((size_t)w * h / 4);
    const size_t last = tex.size() - 1;
    auto at = [&](size_t i) { return tex[i < last ? i : last]; };
    for (int j = 0; j < h; j += 2) {
        for (int i = 0; i < w; i += 2) {
            const uint32_t a = at((size_t)j * w + i), b = at((size_t)j * w + i + 1), c = at((size_t)(j + 1) * w + i),
                           d = at((size_t)(j + 1) * w + i + 1);
            uint32_t o = 0;
            for (int ch = 0; ch < 4; ch++) {
                const int sum = (int)((a >> (8 * ch)) & 0xFF) + (int)((b >> (8 * ch)) & 0xFF) + (int)((c >> (8 * ch)) & 0xFF) +
                                (int)((d >> (8 * ch)) & 0xFF);
                o |= (uint32_t)(uint8_t)(sum / 4) << (8 * ch);
            }
            out.push_back(o);
        }
    }
    return out;
}

struct F3 {
    float v[3];
    float &operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
};
inline F3 f3(float x, float y, float z) { return F3{{x, y, z}}; }
inline F3 sub(F3 a, F3 b) { return f3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline F3 mul(F3 a, float s) { return f3(a[0] * s, a[1] * s, a[2] * s); }
inline F3 cross3(F3 a, F3 b) { return f3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]); }
inline float len3(F3 a) {
    float t = 0.0f;
    t += a[0] * a[0];
    t += a[1] * a[1];
    t += a[2] * a[2];
    return std::sqrt(t);
}
inline F3 norm3(F3 a) {
    const float l = len3(a);
    return f3(a[0] / l, a[1] / l, a[2] / l);
}

} // namespace

int add_texture(ray_scene *s, const uint8_t *data, int w, int h, bool srgb, bool mips, uint32_t *out) {
    // AddTexture, SceneRef.cpp:62-114
    if (!data || w <= 0 || h <= 0 || w > 0x7FFF || h > 0xFFFF) {
        set_error("invalid texture description");
        return RAY_ERR_INVALID_ARG;
    }
    TextureRec t;
    t.w = w;
    t.h = h;
    t.srgb = srgb;
    std::vector<uint32_t> lvl((size_t)w * h);
    memcpy(lvl.data(), data, lvl.size() * 4);
    int res[2] = {w, h};
    int mip = 0;
    while (res[0] >= 1 && res[1] >= 1 && mip < NUM_MIP_LEVELS) {
        int pos[2];
        const int page = atlas_allocate(s, res[0], res[1], pos);
        if (page == -1) {
            set_error("texture does not fit the atlas");
            return RAY_ERR_INVALID_ARG;
        }
        t.page[mip] = (uint8_t)page;
        t.pos[mip][0] = (uint16_t)pos[0];
        t.pos[mip][1] = (uint16_t)pos[1];
        t.lw.push_back(res[0]);
        t.lh.push_back(res[1]);
        t.levels.push_back(lvl);
        mip++;
        if (!mips) break;
        lvl = downsample(lvl, res[0], res[1]);
        res[0] /= 2;
        res[1] /= 2;
    }
    for (int i = mip; i < NUM_MIP_LEVELS; i++) {
        t.page[i] = t.page[mip - 1];
        t.pos[i][0] = t.pos[mip - 1][0];
        t.pos[i][1] = t.pos[mip - 1][1];
    }
    s->textures.push_back(std::move(t));
    s->shade_dirty = true;
    *out = (uint32_t)(s->textures.size() - 1);
    return RAY_OK;
}

// ComputeTangentBasis (TextureUtilsRef.cpp:40-178) as the Ref scene calls it
// (SceneRef.cpp:256-258): vertices is the scene's vertex array, indices the
// new mesh's (already offset) indices, which are rewritten where a vertex is
// split; split vertices are appended to the scene's array.
void compute_tangent_basis(std::vector<VertexRec> &vertices, std::vector<uint32_t> &idx, size_t vtx_start) {
    const size_t n0 = vertices.size();
    std::vector<std::array<uint32_t, 3>> twin(n0, std::array<uint32_t, 3>{0, 0, 0});
    std::vector<F3> binormals(n0, f3(0.0f, 0.0f, 0.0f));
    for (size_t i = 0; i + 2 < idx.size(); i += 3) {
        size_t vi[3] = {idx[i + 0], idx[i + 1], idx[i + 2]};
        const size_t bi[3] = {idx[i + 0], idx[i + 1], idx[i + 2]};
        const VertexRec &v0 = vertices[vi[0]], &v1 = vertices[vi[1]], &v2 = vertices[vi[2]];
        const F3 dp1 = sub(f3(v1.p[0], v1.p[1], v1.p[2]), f3(v0.p[0], v0.p[1], v0.p[2]));
        const F3 dp2 = sub(f3(v2.p[0], v2.p[1], v2.p[2]), f3(v0.p[0], v0.p[1], v0.p[2]));
        const float dt1[2] = {v1.t[0][0] - v0.t[0][0], v1.t[0][1] - v0.t[0][1]};
        const float dt2[2] = {v2.t[0][0] - v0.t[0][0], v2.t[0][1] - v0.t[0][1]};
        F3 tangent, binormal;
        const float det = dt1[0] * dt2[1] - dt1[1] * dt2[0];
        if (std::abs(det) > FLT_EPS_H) {
            const float inv_det = 1.0f / det;
            tangent = mul(sub(mul(dp1, dt2[1]), mul(dp2, dt1[1])), inv_det);
            binormal = mul(sub(mul(dp2, dt1[0]), mul(dp1, dt2[0])), inv_det);
        } else {
            const F3 plane_N = cross3(dp1, dp2);
            int w = 2;
            tangent = f3(0.0f, 1.0f, 0.0f);
            if (std::abs(plane_N[0]) <= std::abs(plane_N[1]) && std::abs(plane_N[0]) <= std::abs(plane_N[2])) {
                tangent = f3(1.0f, 0.0f, 0.0f);
                w = 1;
            } else if (std::abs(plane_N[2]) <= std::abs(plane_N[0]) && std::abs(plane_N[2]) <= std::abs(plane_N[1])) {
                tangent = f3(0.0f, 0.0f, 1.0f);
                w = 0;
            }
            if (std::abs(plane_N[w]) > FLT_EPS_H) {
                binormal = norm3(cross3(plane_N, tangent));
                tangent = norm3(cross3(plane_N, binormal));
            } else {
                binormal = f3(0.0f, 0.0f, 0.0f);
                tangent = f3(0.0f, 0.0f, 0.0f);
            }
        }
        for (int k = 0; k < 3; k++) {
            const VertexRec &v = vertices[vi[k]];
            const F3 &b = binormals[bi[k]];
            const int i1 = (v.b[0] * tangent[0] + v.b[1] * tangent[1] + v.b[2] * tangent[2]) < 0;
            const int i2 = 2 * (b[0] * binormal[0] + b[1] * binormal[1] + b[2] * binormal[2] < 0);
            if (i1 || i2) {
                uint32_t index = twin[bi[k]][i1 + i2 - 1];
                if (index == 0) {
                    index = (uint32_t)vertices.size();
                    VertexRec copy = vertices[vi[k]];
                    copy.b[0] = copy.b[1] = copy.b[2] = 0.0f;
                    vertices.push_back(copy);
                    twin[bi[k]][i1 + i2 - 1] = index;
                }
                idx[i + k] = index;
                vi[k] = index;
            } else {
                binormals[bi[k]] = binormal;
            }
            VertexRec &t = vertices[vi[k]];
            t.b[0] += tangent[0];
            t.b[1] += tangent[1];
            t.b[2] += tangent[2];
        }
    }
    for (size_t i = vtx_start; i < vertices.size(); i++) {
        VertexRec &v = vertices[i];
        if (std::abs(v.b[0]) > FLT_EPS_H || std::abs(v.b[1]) > FLT_EPS_H || std::abs(v.b[2]) > FLT_EPS_H) {
            const F3 tangent = f3(v.b[0], v.b[1], v.b[2]);
            F3 binormal = cross3(f3(v.n[0], v.n[1], v.n[2]), tangent);
            const float l = len3(binormal);
            if (l > FLT_EPS_H) {
                binormal = f3(binormal[0] / l, binormal[1] / l, binormal[2] / l);
                v.b[0] = binormal[0];
                v.b[1] = binormal[1];
                v.b[2] = binormal[2];
            }
        }
    }
}

int upload_shading(ray_scene *s) {
    if (!s->shade_dirty) return RAY_OK;
    cudaStream_t st = s->stream;
    RG_CUDA_TRY(cudaSetDevice(s->device));
    // vertices and indices
    RG_CUDA_TRY(s->d_vertices.ensure(std::max<size_t>(s->vertices.size(), 1) * sizeof(VertexRec)));
    RG_CUDA_TRY(s->d_vtx_indices.ensure(std::max<size_t>(s->vtx_indices.size(), 1) * sizeof(uint32_t)));
    if (!s->vertices.empty())
        RG_CUDA_TRY(cudaMemcpyAsync(s->d_vertices.p, s->vertices.data(), s->vertices.size() * sizeof(VertexRec), cudaMemcpyHostToDevice, st));
    if (!s->vtx_indices.empty())
        RG_CUDA_TRY(cudaMemcpyAsync(s->d_vtx_indices.p, s->vtx_indices.data(), s->vtx_indices.size() * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, st));
    // materials and lights
    RG_CUDA_TRY(s->d_materials.ensure(std::max<size_t>(s->materials.size(), 1) * sizeof(MaterialRec)));
    if (!s->materials.empty())
        RG_CUDA_TRY(cudaMemcpyAsync(s->d_materials.p, s->materials.data(), s->materials.size() * sizeof(MaterialRec), cudaMemcpyHostToDevice,
                                    st));
    RG_CUDA_TRY(s->d_lights.ensure(std::max<size_t>(s->lights.size(), 1) * sizeof(LightRec)));
    if (!s->lights.empty())
        RG_CUDA_TRY(cudaMemcpyAsync(s->d_lights.p, s->lights.data(), s->lights.size() * sizeof(LightRec), cudaMemcpyHostToDevice, st));
    RG_CUDA_TRY(s->d_area_lights.ensure(std::max<size_t>(s->area_lights.size(), 1) * sizeof(AreaLight)));
    if (!s->area_lights.empty())
        RG_CUDA_TRY(cudaMemcpyAsync(s->d_area_lights.p, s->area_lights.data(), s->area_lights.size() * sizeof(AreaLight),
                                    cudaMemcpyHostToDevice, st));
    // textures: one bordered block per stored level (TextureAtlasTiled::Allocate,
    // TextureAtlasRef.cpp:138-163: top border = last row, bottom border = first
    // row, left column = last column, right column = first column, corners wrapped)
    std::vector<TexDev> td(s->textures.size());
    std::vector<uint32_t> texels;
    for (size_t ti = 0; ti < s->textures.size(); ti++) {
        const TextureRec &t = s->textures[ti];
        TexDev &d = td[ti];
        d.width = (uint32_t)t.w | (t.srgb ? 0x8000u : 0u);
        d.height = (uint32_t)t.h;
        const int nl = (int)t.levels.size();
        for (int L = 0; L < nl; L++) {
            const int w = t.lw[L], h = t.lh[L];
            const std::vector<uint32_t> &src = t.levels[L];
            const size_t off = texels.size();
            const int pw = w + 2, ph = h + 2;
            texels.resize(off + (size_t)pw * ph);
            uint32_t *b = texels.data() + off;
            auto px = [&](int x, int y) { return src[(size_t)y * w + x]; };
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++) b[(size_t)(y + 1) * pw + x + 1] = px(x, y);
            for (int x = 0; x < w; x++) {
                b[x + 1] = px(x, h - 1);
                b[(size_t)(ph - 1) * pw + x + 1] = px(x, 0);
            }
            for (int y = 0; y < ph; y++) {
                const int sy = y == 0 ? h - 1 : (y == ph - 1 ? 0 : y - 1);
                b[(size_t)y * pw] = px(w - 1, sy);
                b[(size_t)y * pw + pw - 1] = px(0, sy);
            }
            d.lv[L].off = (uint32_t)off;
            d.lv[L].px = t.pos[L][0];
            d.lv[L].py = t.pos[L][1];
            d.lv[L].pitch = (uint16_t)pw;
            d.lv[L].rows = (uint16_t)ph;
        }
        for (int L = nl; L < NUM_MIP_LEVELS; L++) d.lv[L] = d.lv[nl - 1];
    }
    if (texels.size() > 0xFFFFFFFFull) {
        set_error("texture data too large");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(s->d_textures.ensure(std::max<size_t>(td.size(), 1) * sizeof(TexDev)));
    RG_CUDA_TRY(s->d_texels.ensure(std::max<size_t>(texels.size(), 1) * sizeof(uint32_t)));
    if (!td.empty()) RG_CUDA_TRY(cudaMemcpyAsync(s->d_textures.p, td.data(), td.size() * sizeof(TexDev), cudaMemcpyHostToDevice, st));
    if (!texels.empty())
        RG_CUDA_TRY(cudaMemcpyAsync(s->d_texels.p, texels.data(), texels.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    RG_CUDA_TRY(wait_stream(st));
    s->shade_dirty = false;
    return RAY_OK;
}

RenderScene render_scene_view(const ray_scene *s) {
    RenderScene r{};
    r.sv = SceneView{static_cast<const WideNode *>(s->d_nodes.p), static_cast<const TriRec *>(s->d_leaf.p),
                     static_cast<const InstanceRec *>(s->d_inst.p), s->n_inst_dev, s->tlas.nodes};
    r.tris = static_cast<const TriRec *>(s->d_tris_ref.p);
    r.vtx_indices = static_cast<const uint32_t *>(s->d_vtx_indices.p);
    r.vertices = static_cast<const VertexRec *>(s->d_vertices.p);
    r.materials = static_cast<const MaterialRec *>(s->d_materials.p);
    r.textures = static_cast<const TexDev *>(s->d_textures.p);
    r.texels = static_cast<const uint32_t *>(s->d_texels.p);
    r.lights = static_cast<const LightRec *>(s->d_lights.p);
    r.area_lights = static_cast<const AreaLight *>(s->d_area_lights.p);
    r.n_area_lights = (uint32_t)s->area_lights.size();
    r.n_tris = s->total_tris;
    r.n_materials = (uint32_t)s->materials.size();
    r.n_textures = (uint32_t)s->textures.size();
    r.n_lights = (uint32_t)s->lights.size();
    r.principled_only = s->materials.empty() ? 0u : 1u;
    for (const MaterialRec &m : s->materials)
        if (m.type != (uint32_t)RAY_MAT_PRINCIPLED) r.principled_only = 0u;
    for (int k = 0; k < 3; k++) r.env_col[k] = s->env.env_col[k];
    r.env_clamp = s->env.env_clamp;
    r.env_map = s->env.env_map;
    r.diff_albedo = s->diff_albedo;
    r.diff_rough = s->diff_rough;
    r.diff_rough_sampling = s->diff_rough_sampling;
    r.diff_color = s->diff_color;
    r.diff_aw = (uint32_t)s->diff_aw;
    r.diff_ah = (uint32_t)s->diff_ah;
    r.n_diff_rough = (uint32_t)s->n_diff_rough;
    return r;
}

} // namespace rg
