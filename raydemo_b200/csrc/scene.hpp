// Host-side scene and renderer state behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/raygpu.h"
#include "bvh.cuh"
#include "common.cuh"
#include "render.cuh"

namespace rg {

// A texture with its mip chain (RGBA8, one uint32 per texel) and the atlas
// position the reference's splitter gives each level (texture_t, Core.h:103-108).
struct TextureRec {
    int w = 0, h = 0;
    bool srgb = true;
    std::vector<std::vector<uint32_t>> levels;
    std::vector<int> lw, lh;
    uint16_t pos[NUM_MIP_LEVELS][2] = {};
    uint8_t page[NUM_MIP_LEVELS] = {};
};

// Node of the guillotine splitter that places textures in the reference's
// atlas pages (TextureSplitter, src/Ray/internal/TextureSplitter.cpp).
struct SplitNode {
    int parent = -1;
    int child[2] = {-1, -1};
    int pos[2] = {0, 0}, size[2] = {0, 0};
    bool is_free = true;
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

// api.cu: the lock every C-ABI entry point holds while it runs. The entry
// points only enqueue GPU work (and wait where the call is synchronous), so
// concurrent calls from several threads -- the reference renders disjoint
// regions of one renderer and scene from a thread pool -- are serialised onto
// the renderer's stream in the order they take the lock.
std::recursive_mutex &api_mutex();
// api.cu: the handles that ray_create_* returned and ray_destroy_* has not
// destroyed (read and changed under the API lock): an entry point given any
// other pointer returns RAY_ERR_INVALID_ARG instead of dereferencing it.
bool live_scene(const ray_scene *s);
bool live_renderer(const ray_renderer *r);
// The process-wide API lock, with the calling thread's nesting depth (an
// entry point called from another holds it twice); a host-buffer trace lets
// it go while it waits for its GPU work when it holds it once.
extern thread_local int t_api_depth;
struct ApiLock {
    std::lock_guard<std::recursive_mutex> g;
    ApiLock() : g(api_mutex()) { ++t_api_depth; }
    ~ApiLock() { --t_api_depth; }
    ApiLock(const ApiLock &) = delete;
    ApiLock &operator=(const ApiLock &) = delete;
};
#define RG_API_LOCK rg::ApiLock rg_api_lock_
// Waits (bounded) for st's work with the API lock let go meanwhile, when the
// calling thread holds it once; the caller re-checks its handles afterwards
// (another thread may have changed or destroyed them) and waits again under
// the lock for work enqueued in between.
cudaError_t wait_stream_unlocked(cudaStream_t st);

// api.cu: builds pending BVHs and uploads pending scene data, after the
// kernels already enqueued that read the arrays it overwrites
int commit(ray_scene *s);
// api.cu: records that work just enqueued on st reads the scene's device arrays
cudaError_t note_use(ray_scene *s, cudaStream_t st);

// scene_shading.cu
int add_texture(ray_scene *s, const uint8_t *data, int w, int h, bool srgb, bool mips, uint32_t *out);
void compute_tangent_basis(std::vector<VertexRec> &vertices, std::vector<uint32_t> &indices, size_t vtx_start);
int upload_shading(ray_scene *s); // device copies of vertices, materials, textures and lights
RenderScene render_scene_view(const ray_scene *s);

// A cached CUDA graph of a launch sequence (render.cu: graph_run).
struct GraphSlot {
    uint64_t key = 0;
    int runs = 0;
    bool failed = false;
    cudaGraphExec_t exec = nullptr;
};

} // namespace rg

struct ray_scene {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<rg::MeshRec> meshes;
    std::vector<rg::InstanceRecHost> instances;
    std::vector<rg::MaterialRec> materials;
    std::vector<rg::TextureRec> textures;
    std::vector<std::vector<rg::SplitNode>> atlas_pages;
    std::vector<rg::LightRec> lights;
    std::vector<rg::AreaLight> area_lights; // RAY_LIGHT_QUAD / RAY_LIGHT_SUN
    std::vector<rg::CameraRec> cameras;
    uint32_t cam_first_free = RAY_INVALID_INDEX, current_cam = RAY_INVALID_INDEX;
    ray_environment_desc env{};
    uint32_t default_env_texture = 0, default_normals_texture = 0;

    // shading data (insertion order)
    std::vector<rg::VertexRec> vertices;
    std::vector<uint32_t> vtx_indices;

    bool geom_dirty = true, shade_dirty = true;
    bool inst_dirty = false;                      // instances added, moved or removed (meshes unchanged)
    std::vector<uint32_t> node_base, tri_base;    // each mesh's offsets in the scene arrays (commit)
    // the streams that read this scene's device arrays and an event after each's
    // latest use: a commit's uploads wait for them (rg::note_use)
    std::vector<std::pair<cudaStream_t, cudaEvent_t>> users;
    uint32_t total_tris = 0, total_nodes = 0, max_depth = 0;
    float world_min[3] = {0.0f, 0.0f, 0.0f}, world_max[3] = {0.0f, 0.0f, 0.0f}; // union of the instance boxes
    // differentiable parameters (caller-owned device arrays, ray_scene_set_diff_params)
    const float *diff_albedo = nullptr, *diff_rough = nullptr, *diff_rough_sampling = nullptr, *diff_color = nullptr;
    int diff_aw = 0, diff_ah = 0, n_diff_rough = 0;

    // device arrays assembled at commit
    rg::DeviceBuf d_nodes, d_leaf, d_inst, d_tris_ref;
    uint32_t n_inst_dev = 0;
    rg::InstTree tlas;               // the instance tree (built at commit from TLAS_MIN_INSTANCES instances)
    double last_tlas_ms = 0.0;       // host time of the last commit's instance-tree build or refit
    int last_tlas_refit = 0;         // 1: it was a refit
    rg::DeviceBuf d_vertices, d_vtx_indices, d_materials, d_textures, d_texels, d_lights, d_area_lights;

    // batch-trace staging and diagnostics
    rg::DeviceBuf d_rays, d_hits, d_obj, d_err, d_counters, d_next_ray;
    rg::DeviceBuf d_order[2]; // reordered traces: keys, order and sort scratch of each of two concurrent chunks
    ray_trace_tuning tuning{3, 8, 0, 0, 32, 64, 16, 0, 0, 0};
    bool counting = false;
    ray_trace_info last_info{};
    bool info_pending = false;
    cudaStream_t info_stream = nullptr;
    uint64_t trace_seq = 0; // traces enqueued on the scene so far
    // host-buffer traces: the chunk pipeline's upload, download and second trace
    // streams and its events (created on first use)
    cudaStream_t copy_st[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t pipe_ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // host-buffer traces of this scene run one at a time (they share the
    // staging buffers and events above); a shared pointer, so that a caller
    // can wait for it without holding the API lock while the scene lives on
    std::shared_ptr<std::mutex> host_mu = std::make_shared<std::mutex>();
    uint32_t *h_info = nullptr; // page-locked copy of the error word and counters of the last host-buffer trace

    ~ray_scene();
};

struct ray_renderer {
    int device = 0;
    int w = 0, h = 0;
    cudaStream_t stream = nullptr;     // where the renderer's work goes: own_stream or the caller's
    cudaStream_t own_stream = nullptr;
    ray_stats stats{};
    std::vector<ray_pixel> host_pixels;
    std::vector<ray_shl1> host_sh;
    rg::DeviceBuf d_sort_scratch, d_loop_sort;
    rg::DeviceBuf d_geo_best; // Geo cameras: the covering triangle per texel

    // framebuffers (w * h): the sample being accumulated, the running mean,
    // the toned output; spherical-harmonics data when a camera asks for it
    rg::DeviceBuf d_temp, d_clean, d_final, d_temp_sh, d_clean_sh;
    // wavefront: two ray buffers (trace record + payload, job ids), hits,
    // instance ids, light samples waiting for their shadow rays; counters
    // [0..1] ray counts, [2] persistent-trace work counter, [3] errors,
    // [4..7] rays and shadow segments traced (two uint64), [8] light samples
    rg::DeviceBuf d_rays[2], d_pay[2], d_job[2], d_hits, d_obj, d_counters, d_shadow, d_shadow_rays, d_shadow_job;
    // differentiable form: the samples' sample buffers, the adjoint's per-ray state and light samples
    rg::DeviceBuf d_diff_temp, d_adj[2], d_adj_shadow;
    rg::DeviceBuf d_halton, d_perms;
    int halton_base = -1; // base iteration of the table in d_halton
    bool pixels_on_host = false, sh_on_host = false;
    // phase events of the last two frames (stats): start, after ray generation,
    // primary trace and shade, three per bounce (after its sort, trace and
    // shade), and the frame's end
    static constexpr int N_EVENTS = 35;
    cudaEvent_t ev_sets[2][N_EVENTS] = {};
    bool ev_frame_pending[2] = {false, false};
    int ev_bounces[2] = {0, 0};
    uint64_t frame = 0;
    cudaEvent_t ev_sync = nullptr;        // orders this renderer's stream against a batch
    cudaEvent_t ev_batch[2] = {};         // times the batches of the kernel choice

    // kernel choice: 0 by timing per frame configuration, 1 wavefront, 2 path kernel
    int kernel = 0, last_kernel = 0;
    // ray sorting before the wavefront's bounces: -1 chosen per bounce by
    // timing, else a mask (bit b: sort before secondary bounce b)
    int sort_policy = -1;
    uint32_t last_sort_mask = 0;
    // the wavefront's trace settings: -1 chosen by timing, else an index of
    // rg::TRACE_VARIANTS (0: the scene's own settings)
    int trace_policy = -1;
    int last_trace_var = 0;
    // A frame configuration being timed. Variants: 0 wavefront without
    // sorting (or with the fixed mask), 1 path kernel, 2 wavefront sorting
    // before every bounce.
    // Variants: 0 wavefront without sorting (or with the fixed mask), 1 path
    // kernel, 2 wavefront sorting before every bounce, 3.. the wavefront of
    // variant 0 with trace settings rg::TRACE_VARIANTS[1..] (render.cu).
    static constexpr int N_VARIANTS = 8;
    struct TuneEntry {
        const void *scene = nullptr;
        uint32_t tris = 0, lights = 0, pixels = 0;
        int bounces = 0;
        int kernel_setting = 0, sort_setting = -1, trace_setting = -1;
        int choice = 0;                        // 0 while timing, else the kernel
        uint32_t mask = 0;                     // the sort mask chosen with kernel 1
        int trace_var = 0;                     // the trace settings chosen with kernel 1
        float best[N_VARIANTS] = {1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f}; // best frame time (ms) of each variant
        float bounce_ms[2][10] = {};           // variants 0 and 2: best time of each bounce (sort + trace + shade)
        int n[N_VARIANTS] = {}, pending[N_VARIANTS] = {};
    };
    std::vector<TuneEntry> tune;
    int ev_tune[2] = {-1, -1}; // tune entry timed by the frame in each event set
    int ev_kernel[2] = {0, 0};
    int ev_variant[2] = {0, 0};
    rg::DeviceBuf d_jobs;      // FrameJob array of the path kernel
    // a batch's launch sequence as a CUDA graph (render.cu: graph_run)
    rg::GraphSlot batch_graph;
    ~ray_renderer();
};
