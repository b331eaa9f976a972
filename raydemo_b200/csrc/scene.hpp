// Host-side scene and renderer state behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/raygpu.h"
#include "bvh.cuh"
#include "common.cuh"

namespace rg {

// material_t (src/Ray/internal/Core.h:121-131): textures[] holds the normal
// map, the main texture and, for mix materials, the two mixed materials.
struct MaterialRec {
    uint32_t textures[4];
    float main_color[3], pad;
    uint32_t type;
    float roughness_or_strength;
    float int_ior, ext_ior;
};
static_assert(sizeof(MaterialRec) == 48, "MaterialRec must stay 48 bytes");

// light_t (Core.h:133-138)
struct LightRec {
    float pos[3], radius;
    float col[3], brightness;
    float dir[3], spot;
};
static_assert(sizeof(LightRec) == 48, "LightRec must stay 48 bytes");

// vertex_t (Core.h:259-262)
struct VertexRec {
    float p[3], n[3], b[3], t[2][2];
};
static_assert(sizeof(VertexRec) == 52, "VertexRec must stay 52 bytes");

struct TextureRec {
    int w = 0, h = 0;
    bool srgb = true, mips = false;
    std::vector<uint8_t> rgba; // level 0 followed by the mip chain when mips
    std::vector<uint32_t> level_offset, level_w, level_h;
    bool alive = true;
};

struct MeshRec {
    uint32_t tris_index = 0, tris_count = 0; // global triangle range (insertion order)
    std::vector<float> verts;                // 9 floats per triangle (BVH input)
    std::vector<uint32_t> mat;               // front, back, solid per triangle
    bool built = false;
    MeshBvh bvh;
    TriRec *tris_ref = nullptr; // device, tris_count records in insertion order
};

struct InstanceRecHost {
    uint32_t mesh;
    float xform[16], inv_xform[16];
    float bbox_min[3], bbox_max[3];
};

struct CameraRec {
    ray_camera_desc desc;
    // camera_t fields (Types.h:59-71) as constructed by ConstructCamera
    float origin[3], fwd[3], side[3], up[3];
    bool alive = true;
    uint32_t next_free = RAY_INVALID_INDEX;
};

struct DeviceBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n);
    void release();
    ~DeviceBuf() { release(); }
};

} // namespace rg

struct ray_scene {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<rg::MeshRec> meshes;
    std::vector<rg::InstanceRecHost> instances;
    std::vector<rg::MaterialRec> materials;
    std::vector<rg::TextureRec> textures;
    std::vector<rg::LightRec> lights;
    std::vector<rg::CameraRec> cameras;
    uint32_t cam_first_free = RAY_INVALID_INDEX, current_cam = RAY_INVALID_INDEX;
    ray_environment_desc env{};
    uint32_t default_env_texture = 0, default_normals_texture = 0;

    // shading data (insertion order)
    std::vector<rg::VertexRec> vertices;
    std::vector<uint32_t> vtx_indices;

    bool geom_dirty = true;
    uint32_t total_tris = 0, total_nodes = 0;

    // device arrays assembled at commit
    rg::DeviceBuf d_nodes, d_leaf, d_inst, d_tris_ref;
    uint32_t n_inst_dev = 0;

    // batch-trace staging and diagnostics
    rg::DeviceBuf d_rays, d_hits, d_obj, d_err, d_counters, d_next_ray;
    ray_trace_tuning tuning{2, 8, 0};
    bool counting = false;
    ray_trace_info last_info{};
    bool info_pending = false;
    cudaStream_t info_stream = nullptr;

    ~ray_scene();
};

struct ray_renderer {
    int device = 0;
    int w = 0, h = 0;
    cudaStream_t stream = nullptr;
    ray_stats stats{};
    std::vector<ray_pixel> host_pixels;
    rg::DeviceBuf d_sort_scratch;
    ~ray_renderer();
};
