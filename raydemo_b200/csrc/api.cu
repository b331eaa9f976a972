// C ABI: scene storage, lazy GPU build, batch closest-hit tracing.
// Scene semantics follow the reference Ref::Scene (src/Ray/internal/SceneRef.cpp)
// and SceneBase (src/Ray/SceneBase.cpp); file:line citations per function.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <tuple>
#include <vector>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_set>

#include "../../include/raygpu.h"
#include "radix_sort.cuh"
#include "scene.hpp"
#include "sort.cuh"
#include "trace.cuh"

namespace rg {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string &msg) { g_last_error = msg; }

namespace {
std::atomic<long long> g_wait_timeout_ms{300000};
std::atomic<long long> g_fail_alloc_after{-1}; // >= 0: allocations to let through before one fails
} // namespace

cudaError_t device_alloc(void **p, size_t bytes) {
    long long k = g_fail_alloc_after.load();
    while (k >= 0) {
        if (g_fail_alloc_after.compare_exchange_weak(k, k - 1)) {
            if (k == 0) { // this one fails, as cudaMalloc does when the device is full
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
            break;
        }
    }
    return cudaMalloc(p, bytes);
}

namespace {
// Polls query() until it stops returning cudaErrorNotReady: spinning for the
// first milliseconds (short GPU work returns promptly), then sleeping 50 us
// between polls, up to the wait bound.
template <typename Q>
cudaError_t bounded_wait(Q query) {
    const auto t0 = std::chrono::steady_clock::now();
    const long long limit = g_wait_timeout_ms.load();
    for (uint64_t k = 0;; k++) {
        const cudaError_t e = query();
        if (e != cudaErrorNotReady) return e;
        const long long ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
        if (ms >= limit) return cudaErrorTimeout;
        if (ms >= 20) std::this_thread::sleep_for(std::chrono::microseconds(50));
        else std::this_thread::yield();
    }
}
} // namespace

cudaError_t wait_event(cudaEvent_t e) { return bounded_wait([&] { return cudaEventQuery(e); }); }
cudaError_t wait_stream(cudaStream_t s) { return bounded_wait([&] { return cudaStreamQuery(s); }); }

cudaError_t DeviceBuf::ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    release();
    const size_t want = std::max<size_t>(n, 256);
    cudaError_t e = device_alloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        return e;
    }
    bytes = want;
    return cudaSuccess;
}

void DeviceBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

// InverseMatrix, src/Ray/internal/Core.cpp:909-949 (same operation order).
static void inverse_matrix(const float m[16], float o[16]) {
    const float A2323 = m[10] * m[15] - m[11] * m[14];
    const float A1323 = m[9] * m[15] - m[11] * m[13];
    const float A1223 = m[9] * m[14] - m[10] * m[13];
    const float A0323 = m[8] * m[15] - m[11] * m[12];
    const float A0223 = m[8] * m[14] - m[10] * m[12];
    const float A0123 = m[8] * m[13] - m[9] * m[12];
    const float A2313 = m[6] * m[15] - m[7] * m[14];
    const float A1313 = m[5] * m[15] - m[7] * m[13];
    const float A1213 = m[5] * m[14] - m[6] * m[13];
    const float A2312 = m[6] * m[11] - m[7] * m[10];
    const float A1312 = m[5] * m[11] - m[7] * m[9];
    const float A1212 = m[5] * m[10] - m[6] * m[9];
    const float A0313 = m[4] * m[15] - m[7] * m[12];
    const float A0213 = m[4] * m[14] - m[6] * m[12];
    const float A0312 = m[4] * m[11] - m[7] * m[8];
    const float A0212 = m[4] * m[10] - m[6] * m[8];
    const float A0113 = m[4] * m[13] - m[5] * m[12];
    const float A0112 = m[4] * m[9] - m[5] * m[8];
    const float det = m[0] * (m[5] * A2323 - m[6] * A1323 + m[7] * A1223) - m[1] * (m[4] * A2323 - m[6] * A0323 + m[7] * A0223) +
                      m[2] * (m[4] * A1323 - m[5] * A0323 + m[7] * A0123) - m[3] * (m[4] * A1223 - m[5] * A0223 + m[6] * A0123);
    const float inv_det = 1.0f / det;
    o[0] = inv_det * (m[5] * A2323 - m[6] * A1323 + m[7] * A1223);
    o[1] = inv_det * -(m[1] * A2323 - m[2] * A1323 + m[3] * A1223);
    o[2] = inv_det * (m[1] * A2313 - m[2] * A1313 + m[3] * A1213);
    o[3] = inv_det * -(m[1] * A2312 - m[2] * A1312 + m[3] * A1212);
    o[4] = inv_det * -(m[4] * A2323 - m[6] * A0323 + m[7] * A0223);
    o[5] = inv_det * (m[0] * A2323 - m[2] * A0323 + m[3] * A0223);
    o[6] = inv_det * -(m[0] * A2313 - m[2] * A0313 + m[3] * A0213);
    o[7] = inv_det * (m[0] * A2312 - m[2] * A0312 + m[3] * A0212);
    o[8] = inv_det * (m[4] * A1323 - m[5] * A0323 + m[7] * A0123);
    o[9] = inv_det * -(m[0] * A1323 - m[1] * A0323 + m[3] * A0123);
    o[10] = inv_det * (m[0] * A1313 - m[1] * A0313 + m[3] * A0113);
    o[11] = inv_det * -(m[0] * A1312 - m[1] * A0312 + m[3] * A0112);
    o[12] = inv_det * -(m[4] * A1223 - m[5] * A0223 + m[6] * A0123);
    o[13] = inv_det * (m[0] * A1223 - m[1] * A0223 + m[2] * A0123);
    o[14] = inv_det * -(m[0] * A1213 - m[1] * A0213 + m[2] * A0113);
    o[15] = inv_det * (m[0] * A1212 - m[1] * A0212 + m[2] * A0112);
}

// TransformBoundingBox, src/Ray/internal/Core.cpp:888-907
static void transform_bbox(const float bmin[3], const float bmax[3], const float *x, float omin[3], float omax[3]) {
    for (int j = 0; j < 3; j++) omin[j] = omax[j] = x[12 + j];
    for (int j = 0; j < 3; j++) {
        for (int i = 0; i < 3; i++) {
            const float a = x[i * 4 + j] * bmin[i];
            const float b = x[i * 4 + j] * bmax[i];
            if (a < b) {
                omin[j] += a;
                omax[j] += b;
            } else {
                omin[j] += b;
                omax[j] += a;
            }
        }
    }
}

static float len3(const float *v) {
    float t = 0.0f;
    t += v[0] * v[0];
    t += v[1] * v[1];
    t += v[2] * v[2];
    return std::sqrt(t);
}

// ConstructCamera, src/Ray/internal/Core.cpp:856-886 (perspective)
static void construct_camera(CameraRec &c) {
    const ray_camera_desc &d = c.desc;
    float u[3] = {d.up[0], d.up[1], d.up[2]};
    float l2 = 0.0f;
    l2 += u[0] * u[0];
    l2 += u[1] * u[1];
    l2 += u[2] * u[2];
    if (l2 < FLT_EPS_) {
        if (std::abs(d.fwd[1]) >= 0.999f) {
            u[0] = 1.0f; u[1] = 0.0f; u[2] = 0.0f;
        } else {
            u[0] = 0.0f; u[1] = 1.0f; u[2] = 0.0f;
        }
    }
    const float *f = d.fwd;
    float s[3] = {f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0]};
    const float ls = len3(s);
    for (int k = 0; k < 3; k++) s[k] = s[k] / ls;
    const float nu[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
    for (int k = 0; k < 3; k++) {
        c.origin[k] = d.origin[k];
        c.fwd[k] = f[k];
        c.side[k] = s[k];
        c.up[k] = nu[k];
    }
}

// SceneBase::SetCamera, SceneBase.cpp:56-84. A Geo camera takes its kind,
// gamma, instance and UV layer and leaves the perspective fields (filter,
// dtype, origin, axes, fov, focus) as the slot held them: zero for a new
// slot, a previous camera's where one is replaced. A perspective camera
// leaves mi_index / uv_index as they were.
static void set_camera(CameraRec &rec, const ray_camera_desc &c) {
    ray_camera_desc &d = rec.desc;
    d.type = c.type;
    d.gamma = c.gamma;
    if (c.type != RAY_CAM_GEO) {
        d.filter = c.filter;
        d.dtype = c.dtype;
        memcpy(d.origin, c.origin, sizeof(d.origin));
        memcpy(d.fwd, c.fwd, sizeof(d.fwd));
        memcpy(d.up, c.up, sizeof(d.up));
        d.fov = c.fov;
        d.focus_distance = c.focus_distance;
        d.focus_factor = c.focus_factor;
        construct_camera(rec);
    } else {
        d.mi_index = c.mi_index;
        d.uv_index = c.uv_index;
    }
    d.lighting_only = c.lighting_only;
    d.skip_direct_lighting = c.skip_direct_lighting;
    d.skip_indirect_lighting = c.skip_indirect_lighting;
    d.no_background = c.no_background;
    d.clamp = c.clamp;
    d.output_sh = c.output_sh;
    d.use_coherent_sampling = c.use_coherent_sampling;
    d.max_diff_depth = c.max_diff_depth;
    d.max_glossy_depth = c.max_glossy_depth;
    d.max_refr_depth = c.max_refr_depth;
    d.max_transp_depth = c.max_transp_depth;
    d.max_total_depth = c.max_total_depth;
    d.termination_start_depth = c.termination_start_depth;
}

std::recursive_mutex &api_mutex() {
    static std::recursive_mutex m;
    return m;
}

namespace {
std::unordered_set<const void *> &live_handles() {
    static std::unordered_set<const void *> h;
    return h;
}
} // namespace

bool live_scene(const ray_scene *s) { return live_handles().count(s) != 0; }
thread_local int t_api_depth = 0;

cudaError_t wait_stream_unlocked(cudaStream_t st) {
    if (t_api_depth != 1) return wait_stream(st);
    api_mutex().unlock();
    const cudaError_t e = wait_stream(st);
    api_mutex().lock();
    return e;
}
bool live_renderer(const ray_renderer *r) { return live_handles().count(r) != 0; }

cudaError_t note_use(ray_scene *s, cudaStream_t st) {
    for (auto &u : s->users)
        if (u.first == st) return cudaEventRecord(u.second, st);
    if (s->users.size() >= 8) { // a short list: the oldest user's wait goes onto the scene's stream now
        cudaError_t e = cudaStreamWaitEvent(s->stream, s->users.front().second, 0);
        if (e != cudaSuccess) return e;
        cudaEventDestroy(s->users.front().second);
        s->users.erase(s->users.begin());
    }
    cudaEvent_t ev = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    s->users.emplace_back(st, ev);
    return cudaEventRecord(ev, st);
}

int commit(ray_scene *s) {
    if (!s->geom_dirty && !s->inst_dirty && !s->shade_dirty) return RAY_OK;
    const bool geom_changed = s->geom_dirty;
    RG_CUDA_TRY(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    // the frames and traces in flight read the arrays about to be rewritten
    for (auto &u : s->users) RG_CUDA_TRY(cudaStreamWaitEvent(st, u.second, 0));
    if (!s->geom_dirty && !s->inst_dirty) return upload_shading(s);
    if (s->geom_dirty) {
    // 1. build the meshes that have no BVH yet
    for (MeshRec &m : s->meshes) {
        if (m.built) continue;
        const uint32_t n = m.tris_count;
        if (m.tris_ref) {
            cudaFree(m.tris_ref);
            m.tris_ref = nullptr;
        }
        if (n) {
            DeviceBuf verts, mat, aabb;
            RG_CUDA_TRY(verts.ensure(m.verts.size() * sizeof(float)));
            RG_CUDA_TRY(mat.ensure(m.mat.size() * sizeof(uint32_t)));
            RG_CUDA_TRY(aabb.ensure((size_t)n * 6 * sizeof(float)));
            RG_CUDA_TRY(device_alloc(reinterpret_cast<void **>(&m.tris_ref), (size_t)n * sizeof(TriRec)));
            RG_CUDA_TRY(cudaMemcpyAsync(verts.p, m.verts.data(), m.verts.size() * sizeof(float), cudaMemcpyHostToDevice, st));
            RG_CUDA_TRY(cudaMemcpyAsync(mat.p, m.mat.data(), m.mat.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
            RG_CUDA_TRY(launch_preprocess_tris(static_cast<const float *>(verts.p), static_cast<const uint32_t *>(mat.p), n, m.tris_ref,
                                               static_cast<float *>(aabb.p), st));
            free_mesh_bvh(m.bvh); // what an earlier, failed build of this mesh left
            const int rc = build_mesh_bvh(m.tris_ref, static_cast<const float *>(aabb.p), n, m.bvh, st);
            if (rc != RAY_OK) return rc;
            RG_CUDA_TRY(wait_stream(st));
        }
        m.built = true;
    }
    // 2. assemble the scene arrays
    uint64_t nodes = 0, tris = 0;
    for (const MeshRec &m : s->meshes) {
        nodes += m.bvh.node_count;
        tris += m.tris_count;
    }
    if (nodes > 0xffffffffull || tris > 0x7fffffffull) {
        set_error("scene too large");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(s->d_nodes.ensure(nodes * sizeof(WideNode)));
    RG_CUDA_TRY(s->d_leaf.ensure(tris * sizeof(TriRec)));
    RG_CUDA_TRY(s->d_tris_ref.ensure(tris * sizeof(TriRec)));
    std::vector<uint32_t> &node_base = s->node_base, &tri_base = s->tri_base;
    node_base.assign(s->meshes.size(), 0);
    tri_base.assign(s->meshes.size(), 0);
    uint64_t nb = 0, tb = 0;
    for (size_t i = 0; i < s->meshes.size(); i++) {
        const MeshRec &m = s->meshes[i];
        node_base[i] = (uint32_t)nb;
        tri_base[i] = (uint32_t)tb;
        if (m.bvh.node_count) {
            RG_CUDA_TRY(cudaMemcpyAsync(static_cast<WideNode *>(s->d_nodes.p) + nb, m.bvh.nodes, m.bvh.node_count * sizeof(WideNode),
                                        cudaMemcpyDeviceToDevice, st));
            RG_CUDA_TRY(cudaMemcpyAsync(static_cast<TriRec *>(s->d_leaf.p) + tb, m.bvh.leaf_tris, m.bvh.tri_count * sizeof(TriRec),
                                        cudaMemcpyDeviceToDevice, st));
            RG_CUDA_TRY(cudaMemcpyAsync(static_cast<TriRec *>(s->d_tris_ref.p) + m.tris_index, m.tris_ref, m.tris_count * sizeof(TriRec),
                                        cudaMemcpyDeviceToDevice, st));
        }
        nb += m.bvh.node_count;
        tb += m.bvh.tri_count;
    }
    s->total_nodes = (uint32_t)nodes;
    s->max_depth = 0;
    for (const MeshRec &m : s->meshes) s->max_depth = std::max(s->max_depth, m.bvh.depth);
    }
    // 3. instances (SetMeshInstanceTransform, SceneRef.cpp:370-414). The
    // instance level is a list the traversal tests box by box, so a moved
    // instance costs this upload of its record and no rebuild.
    const std::vector<uint32_t> &node_base = s->node_base, &tri_base = s->tri_base;
    std::vector<InstanceRec> inst;
    for (const InstanceRecHost &ih : s->instances) {
        const MeshRec &m = s->meshes[ih.mesh];
        if (m.tris_count == 0) continue;
        InstanceRec r{};
        const float *x = ih.inv_xform;
        const int sel[12] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14};
        for (int k = 0; k < 12; k++) r.inv_xform[k] = x[sel[k]];
        float bmn[3], bmx[3];
        transform_bbox(m.bvh.bmin, m.bvh.bmax, ih.xform, bmn, bmx);
        for (int k = 0; k < 3; k++) {
            r.bbox_min[k] = bmn[k];
            r.bbox_max[k] = bmx[k];
        }
        r.node_base = node_base[ih.mesh];
        r.tri_base = tri_base[ih.mesh];
        r.prim_base = m.tris_index;
        r.mesh = ih.mesh;
        r.node_count = m.bvh.node_count;
        r.tri_count = m.bvh.tri_count;
        inst.push_back(r);
    }
    // keep the instance index the reference reports (mesh_instances_ position)
    RG_CUDA_TRY(s->d_inst.ensure(std::max<size_t>(inst.size(), 1) * sizeof(InstanceRec)));
    if (!inst.empty())
        RG_CUDA_TRY(cudaMemcpyAsync(s->d_inst.p, inst.data(), inst.size() * sizeof(InstanceRec), cudaMemcpyHostToDevice, st));
    s->n_inst_dev = (uint32_t)inst.size();
    // the instance tree: a refit when only instances moved (same count, no
    // mesh rebuilt), else a build; none below the tuning's instance count
    {
        const uint32_t ni = (uint32_t)inst.size();
        const int mode = s->tuning.instance_tree;
        const bool want = mode >= 0 && ni >= 2 && (mode == 1 || ni >= TLAS_MIN_INSTANCES);
        if (!want) {
            free_inst_tree(s->tlas);
        } else {
            std::vector<float> boxes(6 * (size_t)ni);
            for (size_t i = 0; i < inst.size(); i++)
                for (int k = 0; k < 3; k++) {
                    boxes[6 * i + k] = inst[i].bbox_min[k];
                    boxes[6 * i + 3 + k] = inst[i].bbox_max[k];
                }
            const bool refit = !geom_changed && s->tlas.n == ni;
            const auto t0 = std::chrono::steady_clock::now();
            const int rc = build_inst_tree(boxes.data(), ni, refit, s->tlas, st);
            if (rc != RAY_OK) return rc;
            RG_CUDA_TRY(wait_stream(st));
            s->last_tlas_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            s->last_tlas_refit = refit ? 1 : 0;
        }
    }
    // the scene's box: the union of the instance boxes (the ray hash grid of the render loop's sort)
    for (int k = 0; k < 3; k++) {
        s->world_min[k] = inst.empty() ? 0.0f : inst[0].bbox_min[k];
        s->world_max[k] = inst.empty() ? 0.0f : inst[0].bbox_max[k];
    }
    for (const InstanceRec &q : inst)
        for (int k = 0; k < 3; k++) {
            s->world_min[k] = std::min(s->world_min[k], q.bbox_min[k]);
            s->world_max[k] = std::max(s->world_max[k], q.bbox_max[k]);
        }
    RG_CUDA_TRY(wait_stream(st));
    s->geom_dirty = s->inst_dirty = false;
    return upload_shading(s);
}

} // namespace rg

using namespace rg;

#define RG_CHECK(cond, msg)                                                                                            \
    do {                                                                                                               \
        if (!(cond)) {                                                                                                 \
            set_error(msg);                                                                                            \
            return RAY_ERR_INVALID_ARG;                                                                                \
        }                                                                                                              \
    } while (0)

#define RG_GUARD_BEGIN try {
#define RG_GUARD_END                                                                                                   \
    }                                                                                                                  \
    catch (const std::bad_alloc &) {                                                                                   \
        set_error("host allocation failed");                                                                           \
        return RAY_ERR_OUT_OF_MEMORY;                                                                                  \
    }                                                                                                                  \
    catch (const std::exception &e) {                                                                                  \
        set_error(e.what());                                                                                           \
        return RAY_ERR_INVALID_ARG;                                                                                    \
    }

ray_scene::~ray_scene() {
    cudaSetDevice(device);
    free_inst_tree(tlas);
    for (MeshRec &m : meshes) {
        free_mesh_bvh(m.bvh);
        if (m.tris_ref) cudaFree(m.tris_ref);
    }
    if (stream) cudaStreamDestroy(stream);
    for (cudaStream_t c : copy_st)
        if (c) cudaStreamDestroy(c);
    for (cudaEvent_t e : pipe_ev)
        if (e) cudaEventDestroy(e);
    for (auto &u : users) cudaEventDestroy(u.second);
    if (h_info) cudaFreeHost(h_info);
}

extern "C" {

const char *ray_last_error(void) { return g_last_error.c_str(); }
int ray_version(void) { return 1; }

int ray_create_renderer(const ray_settings *s, ray_renderer **out) {
    RG_API_LOCK;
    RG_CHECK(s && out, "null argument");
    RG_CHECK(s->w > 0 && s->h > 0 && s->w <= 32768 && s->h <= 32768, "invalid framebuffer size");
    RG_GUARD_BEGIN
    int ndev = 0;
    RG_CUDA_TRY(cudaGetDeviceCount(&ndev));
    RG_CHECK(s->device >= 0 && s->device < ndev, "invalid CUDA device index");
    RG_CUDA_TRY(cudaSetDevice(s->device));
    auto *r = new ray_renderer;
    r->device = s->device;
    r->w = s->w;
    r->h = s->h;
    cudaError_t e = cudaStreamCreateWithFlags(&r->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete r;
        set_error(cudaGetErrorString(e));
        return RAY_ERR_CUDA;
    }
    r->stream = r->own_stream;
    live_handles().insert(r);
    *out = r;
    return RAY_OK;
    RG_GUARD_END
}

int ray_destroy_renderer(ray_renderer *r) {
    RG_API_LOCK;
    if (!r) return RAY_OK;
    RG_CHECK(live_renderer(r), "unknown or already destroyed renderer handle");
    live_handles().erase(r);
    delete r;
    return RAY_OK;
}

int ray_renderer_type(const ray_renderer *r, int *out_type) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    RG_CHECK(r && out_type, "null argument");
    *out_type = RAY_RENDERER_CUDA_SM100;
    return RAY_OK;
}

int ray_renderer_size(const ray_renderer *r, int *w, int *h) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    RG_CHECK(r && w && h, "null argument");
    *w = r->w;
    *h = r->h;
    return RAY_OK;
}

int ray_create_scene(ray_renderer *r, ray_scene **out) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    RG_CHECK(r && out, "null argument");
    RG_GUARD_BEGIN
    RG_CUDA_TRY(cudaSetDevice(r->device));
    auto *s = new ray_scene;
    s->device = r->device;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        set_error(cudaGetErrorString(e));
        return RAY_ERR_CUDA;
    }
    // Ref::Scene::Scene (SceneRef.cpp:8-44): a 1-pixel white RGBE environment
    // map and a 1-pixel flat normal map are textures 0 and 1.
    static const uint8_t env_px[4] = {255, 255, 255, 128};
    static const uint8_t nrm_px[4] = {127, 127, 255, 0};
    add_texture(s, env_px, 1, 1, true, false, &s->default_env_texture);
    add_texture(s, nrm_px, 1, 1, true, false, &s->default_normals_texture);
    s->env.env_col[0] = s->env.env_col[1] = s->env.env_col[2] = 0.0f;
    s->env.env_clamp = 0.0f;
    s->env.env_map = s->default_env_texture;
    live_handles().insert(s);
    *out = s;
    return RAY_OK;
    RG_GUARD_END
}

int ray_destroy_scene(ray_scene *s) {
    RG_API_LOCK;
    if (!s) return RAY_OK;
    RG_CHECK(live_scene(s), "unknown or already destroyed scene handle");
    live_handles().erase(s);
    delete s;
    return RAY_OK;
}

int ray_scene_get_environment(ray_scene *s, ray_environment_desc *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out, "null argument");
    *out = s->env;
    return RAY_OK;
}

int ray_scene_set_environment(ray_scene *s, const ray_environment_desc *env) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && env, "null argument");
    s->env = *env;
    if (s->env.env_map == RAY_INVALID_INDEX) s->env.env_map = s->default_env_texture; // SceneRef.cpp:52-59
    return RAY_OK;
}

int ray_scene_add_texture(ray_scene *s, const ray_tex_desc *t, uint32_t *out_index) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && t && out_index, "null argument");
    RG_GUARD_BEGIN
    return add_texture(s, t->data, t->w, t->h, t->is_srgb != 0, t->generate_mipmaps != 0, out_index);
    RG_GUARD_END
}

int ray_scene_remove_texture(ray_scene *s, uint32_t i) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s, "null argument");
    (void)i; // no-op in the reference too (SceneRef.h:84)
    return RAY_OK;
}

int ray_scene_add_material(ray_scene *s, const ray_mat_desc *m, uint32_t *out_index) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && m && out_index, "null argument");
    RG_CHECK((m->type >= RAY_MAT_DIFFUSE && m->type <= RAY_MAT_TRANSPARENT) || m->type == RAY_MAT_PRINCIPLED, "invalid material type");
    RG_CHECK(m->type != RAY_MAT_PRINCIPLED || (m->roughness >= 0.0f && m->roughness <= 1.0f && m->metallic >= 0.0f && m->metallic <= 1.0f),
             "roughness and metallic must lie in [0, 1]");
    RG_CHECK(m->type != RAY_MAT_PRINCIPLED || m->main_texture == RAY_INVALID_INDEX || m->main_texture < s->textures.size(),
             "main texture out of range");
    RG_GUARD_BEGIN
    // AddMaterial, SceneRef.cpp:118-150
    MaterialRec r{};
    r.type = (uint32_t)m->type;
    r.textures[1] = m->main_texture;
    r.textures[2] = r.textures[3] = RAY_INVALID_INDEX;
    for (int k = 0; k < 3; k++) r.main_color[k] = m->main_color[k];
    r.int_ior = m->int_ior;
    r.ext_ior = m->ext_ior;
    if (m->type == RAY_MAT_DIFFUSE || m->type == RAY_MAT_GLOSSY || m->type == RAY_MAT_REFRACTIVE) {
        r.roughness_or_strength = m->roughness;
    } else if (m->type == RAY_MAT_PRINCIPLED) {
        r.roughness_or_strength = m->roughness;
        r.metallic = m->metallic;
    } else if (m->type == RAY_MAT_EMISSIVE) {
        r.roughness_or_strength = m->strength;
    } else if (m->type == RAY_MAT_MIX) {
        r.roughness_or_strength = m->strength;
        r.textures[2] = m->mix_materials[0];
        r.textures[3] = m->mix_materials[1];
    }
    r.textures[0] = (m->normal_map != RAY_INVALID_INDEX) ? m->normal_map : s->default_normals_texture;
    s->materials.push_back(r);
    s->shade_dirty = true;
    *out_index = (uint32_t)(s->materials.size() - 1);
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_set_diff_params(ray_scene *s, const ray_diff_params *p) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s, "null scene");
    auto slotted = [](const MaterialRec &m) { return m.type == (uint32_t)RAY_MAT_PRINCIPLED || m.type == (uint32_t)RAY_MAT_DIFFUSE; };
    if (!p) {
        for (MaterialRec &m : s->materials)
            if (slotted(m) && m.textures[2] != RAY_INVALID_INDEX) {
                m.textures[2] = RAY_INVALID_INDEX;
                s->shade_dirty = true;
            }
        s->diff_albedo = s->diff_rough = s->diff_rough_sampling = s->diff_color = nullptr;
        s->diff_aw = s->diff_ah = s->n_diff_rough = 0;
        s->shade_dirty = true;
        return RAY_OK;
    }
    RG_CHECK(p->roughness, "the roughness array is required");
    RG_CHECK(!p->albedo || (p->albedo_w > 0 && p->albedo_h > 0), "albedo size");
    RG_CHECK(p->n_roughness > 0 && p->n_roughness <= 64, "1 to 64 roughness slots");
    RG_CHECK(!p->material_slot || p->n_materials == (int)s->materials.size(), "one slot entry per material of the scene");
    if (p->material_slot)
        for (size_t m = 0; m < s->materials.size(); m++) {
            const int32_t k = p->material_slot[m];
            RG_CHECK(k >= -1 && k < p->n_roughness, "material slot out of range");
            RG_CHECK(k < 0 || slotted(s->materials[m]), "slots are for RAY_MAT_PRINCIPLED and RAY_MAT_DIFFUSE materials");
            RG_CHECK(k < 0 || s->materials[m].type != (uint32_t)RAY_MAT_PRINCIPLED || p->albedo,
                     "a RAY_MAT_PRINCIPLED material in a slot needs the albedo texture");
        }
    // the slots live in the device material records: upload only when one changes
    // (the parameter arrays themselves are read through the pointers at each render)
    for (size_t m = 0; m < s->materials.size(); m++) {
        if (!slotted(s->materials[m])) continue;
        const int32_t k = p->material_slot ? p->material_slot[m] : -1;
        const uint32_t v = k >= 0 ? (uint32_t)k : RAY_INVALID_INDEX;
        if (s->materials[m].textures[2] != v) {
            s->materials[m].textures[2] = v;
            s->shade_dirty = true;
        }
    }
    s->diff_albedo = p->albedo;
    s->diff_rough = p->roughness;
    s->diff_rough_sampling = p->roughness_sampling;
    s->diff_color = p->color;
    s->diff_aw = p->albedo ? p->albedo_w : 0;
    s->diff_ah = p->albedo ? p->albedo_h : 0;
    s->n_diff_rough = p->n_roughness;
    return RAY_OK;
}

int ray_scene_remove_material(ray_scene *s, uint32_t i) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s, "null argument");
    (void)i; // no-op in the reference too (SceneRef.h:87)
    return RAY_OK;
}

int ray_scene_add_mesh(ray_scene *s, const ray_mesh_desc *d, uint32_t *out_index) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && d && out_index, "null argument");
    RG_CHECK(d->prim_type == 0, "only indexed triangle lists are supported");
    RG_CHECK(d->layout >= RAY_LAYOUT_PNT && d->layout <= RAY_LAYOUT_PNBTT, "invalid vertex layout");
    RG_CHECK(d->vtx_indices_count % 3 == 0, "index count must be a multiple of 3");
    RG_CHECK(d->vtx_indices_count == 0 || (d->vtx_indices && d->vtx_attrs), "null vertex data");
    RG_GUARD_BEGIN
    static const size_t strides[4] = {8, 10, 11, 13}; // AttrStrides, SceneBase.h:38-43
    const size_t stride = strides[d->layout];
    const uint64_t ntris = d->vtx_indices_count / 3;
    RG_CHECK((uint64_t)s->total_tris + ntris <= 0x7fffffffull, "too many triangles");
    for (uint64_t j = 0; j < d->vtx_indices_count; j++) {
        const int64_t v = (int64_t)d->vtx_indices[j] + d->base_vertex;
        RG_CHECK(v >= 0 && (uint64_t)v < d->vtx_attrs_count, "vertex index out of range");
    }
    // material of every triangle: AddMesh, SceneRef.cpp:184-215
    std::vector<uint32_t> mat(ntris * 3, 0u);
    for (uint64_t i = 0; i < ntris; i++) {
        mat[3 * i + 0] = 0;
        mat[3 * i + 1] = 0;
        mat[3 * i + 2] = 0;
    }
    for (uint64_t k = 0; k < d->shapes_count; k++) {
        const ray_shape_desc &sh = d->shapes[k];
        RG_CHECK(sh.mat_index < s->materials.size(), "shape material out of range");
        bool solid = true;
        uint32_t stack[32];
        uint32_t cnt = 0;
        stack[cnt++] = sh.mat_index;
        while (cnt) {
            const uint32_t mi = stack[--cnt];
            RG_CHECK(mi < s->materials.size(), "mix material out of range");
            const MaterialRec &mr = s->materials[mi];
            if (mr.type == RAY_MAT_MIX) {
                RG_CHECK(cnt + 2 <= 32, "mix materials nested too deeply");
                stack[cnt++] = mr.textures[2];
                stack[cnt++] = mr.textures[3];
            } else if (mr.type == RAY_MAT_TRANSPARENT) {
                solid = false;
                break;
            }
        }
        for (uint64_t i = sh.vtx_start; i < sh.vtx_start + sh.vtx_count && i / 3 < ntris; i += 3) {
            mat[3 * (i / 3) + 0] = sh.mat_index;
            mat[3 * (i / 3) + 1] = sh.back_mat_index;
            mat[3 * (i / 3) + 2] = solid ? 1u : 0u;
        }
    }
    MeshRec m;
    m.tris_index = s->total_tris;
    m.tris_count = (uint32_t)ntris;
    m.verts.resize(ntris * 9);
    m.mat = std::move(mat);
    for (uint64_t j = 0; j < d->vtx_indices_count; j++) {
        const size_t v = (size_t)((int64_t)d->vtx_indices[j] + d->base_vertex);
        memcpy(&m.verts[3 * j], d->vtx_attrs + v * stride, 3 * sizeof(float));
    }
    // shading attributes (SceneRef.cpp:220-260); layouts without tangents get
    // them from the triangles, which may split vertices
    const uint32_t vbase = (uint32_t)s->vertices.size();
    s->vertices.resize(vbase + d->vtx_attrs_count);
    for (uint64_t i = 0; i < d->vtx_attrs_count; i++) {
        VertexRec &v = s->vertices[vbase + i];
        memset(&v, 0, sizeof(v));
        const float *a = d->vtx_attrs + i * stride;
        memcpy(v.p, a, 12);
        memcpy(v.n, a + 3, 12);
        if (d->layout == RAY_LAYOUT_PNT) {
            memcpy(v.t[0], a + 6, 8);
        } else if (d->layout == RAY_LAYOUT_PNTT) {
            memcpy(v.t[0], a + 6, 8);
            memcpy(v.t[1], a + 8, 8);
        } else if (d->layout == RAY_LAYOUT_PNBT) {
            memcpy(v.b, a + 6, 12);
            memcpy(v.t[0], a + 9, 8);
        } else {
            memcpy(v.b, a + 6, 12);
            memcpy(v.t[0], a + 9, 8);
            memcpy(v.t[1], a + 11, 8);
        }
    }
    std::vector<uint32_t> ni(d->vtx_indices_count);
    for (uint64_t j = 0; j < d->vtx_indices_count; j++) ni[j] = (uint32_t)(d->vtx_indices[j] + d->base_vertex) + vbase;
    if (d->layout == RAY_LAYOUT_PNT || d->layout == RAY_LAYOUT_PNTT) compute_tangent_basis(s->vertices, ni, vbase);
    s->vtx_indices.insert(s->vtx_indices.end(), ni.begin(), ni.end());
    s->meshes.push_back(std::move(m));
    s->total_tris += (uint32_t)ntris;
    s->geom_dirty = true;
    s->shade_dirty = true;
    *out_index = (uint32_t)(s->meshes.size() - 1);
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_remove_mesh(ray_scene *s, uint32_t i) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && i < s->meshes.size(), "invalid mesh index");
    RG_GUARD_BEGIN
    // RemoveMesh, SceneRef.cpp:263-303: swap with the last mesh, drop the
    // instances that then refer to index i (this includes the instances of the
    // mesh that was moved into slot i, as in the reference), remove the
    // triangles and shift the triangle ranges of later meshes.
    const uint32_t last = (uint32_t)s->meshes.size() - 1;
    const uint32_t tris_index = s->meshes[i].tris_index, tris_count = s->meshes[i].tris_count;
    free_mesh_bvh(s->meshes[i].bvh);
    if (s->meshes[i].tris_ref) cudaFree(s->meshes[i].tris_ref);
    s->meshes[i].tris_ref = nullptr;
    std::swap(s->meshes[i], s->meshes[last]);
    s->meshes.pop_back();
    for (auto it = s->instances.begin(); it != s->instances.end();) {
        if (it->mesh == last) it->mesh = i;
        if (it->mesh == i) it = s->instances.erase(it);
        else ++it;
    }
    for (MeshRec &m : s->meshes)
        if (m.tris_index > tris_index) m.tris_index -= tris_count;
    // shading arrays keep insertion order: remove the triangle indices of the range
    s->vtx_indices.erase(s->vtx_indices.begin() + 3ull * tris_index, s->vtx_indices.begin() + 3ull * (tris_index + tris_count));
    s->total_tris -= tris_count;
    s->geom_dirty = true;
    s->shade_dirty = true;
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_add_light(ray_scene *s, const ray_light_desc *d, uint32_t *out_index) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && d && out_index, "null argument");
    RG_CHECK(d->type >= RAY_LIGHT_POINT && d->type <= RAY_LIGHT_SUN, "invalid light type");
    RG_GUARD_BEGIN
    const float PI = 3.141592653589793238463f;
    if (d->type == RAY_LIGHT_QUAD || d->type == RAY_LIGHT_SUN) {
        AreaLight a{};
        a.type = (uint32_t)d->type;
        for (int k = 0; k < 3; k++) a.L[k] = d->color[k];
        if (d->type == RAY_LIGHT_QUAD) {
            const float *u = d->edge_u, *v = d->edge_v;
            const float c[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
            const float area = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
            const float uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
            const float lu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]), lv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            RG_CHECK(area > 0.0f && std::abs(uv) <= 1e-4f * lu * lv, "a quad light needs two non-zero perpendicular edges");
            for (int k = 0; k < 3; k++) {
                a.p0[k] = d->position[k];
                a.u[k] = u[k];
                a.v[k] = v[k];
                a.n[k] = c[k] / area;
            }
            a.area = area;
        } else {
            const float *w = d->direction;
            const float l = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
            RG_CHECK(l > 0.0f && d->angle > 0.0f && d->angle < 180.0f, "a sun light needs a direction and an angle in (0, 180)");
            for (int k = 0; k < 3; k++) a.n[k] = -w[k] / l;
            a.cos_max = std::cos(0.5f * d->angle * PI / 180.0f);
        }
        s->area_lights.push_back(a);
        s->shade_dirty = true;
        *out_index = (uint32_t)(s->lights.size() + s->area_lights.size() - 1);
        return RAY_OK;
    }
    // AddLight, SceneRef.cpp:305-349
    LightRec l{};
    memcpy(l.pos, d->position, 12);
    l.radius = d->radius;
    memcpy(l.col, d->color, 12);
    if (d->type == RAY_LIGHT_SPOT) {
        for (int k = 0; k < 3; k++) l.dir[k] = -d->direction[k];
        l.spot = std::cos(d->angle * PI / 180.0f);
    } else if (d->type == RAY_LIGHT_POINT) {
        l.dir[0] = l.dir[2] = 0.0f;
        l.dir[1] = 1.0f;
        l.spot = -1.0f;
    } else {
        const float dist = 9999999.0f;
        for (int k = 0; k < 3; k++) l.dir[k] = -d->direction[k];
        for (int k = 0; k < 3; k++) l.pos[k] = l.dir[k] * dist;
        l.radius = dist * std::tan(d->angle * PI / 180.0f) + 1.0f;
        float kk = 1.0f + dist / l.radius;
        kk *= kk;
        for (int k = 0; k < 3; k++) l.col[k] = d->color[k] * kk;
        l.spot = 0.0f;
    }
    l.brightness = std::max(l.col[0], std::max(l.col[1], l.col[2]));
    s->lights.push_back(l);
    s->shade_dirty = true;
    *out_index = (uint32_t)(s->lights.size() + s->area_lights.size() - 1);
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_remove_light(ray_scene *s, uint32_t i) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s, "null argument");
    (void)i; // a no-op in the reference (SceneRef.cpp:351-354)
    return RAY_OK;
}

int ray_scene_add_mesh_instance(ray_scene *s, uint32_t mesh_index, const float xform[16], uint32_t *out_index) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && xform && out_index, "null argument");
    RG_CHECK(mesh_index < s->meshes.size(), "invalid mesh index");
    RG_GUARD_BEGIN
    InstanceRecHost ih{};
    ih.mesh = mesh_index;
    memcpy(ih.xform, xform, 64);
    inverse_matrix(ih.xform, ih.inv_xform);
    s->instances.push_back(ih);
    s->inst_dirty = true;
    *out_index = (uint32_t)(s->instances.size() - 1);
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_set_mesh_instance_transform(ray_scene *s, uint32_t mi, const float xform[16]) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && xform && mi < s->instances.size(), "invalid instance");
    memcpy(s->instances[mi].xform, xform, 64);
    inverse_matrix(s->instances[mi].xform, s->instances[mi].inv_xform);
    s->inst_dirty = true;
    return RAY_OK;
}

int ray_scene_remove_mesh_instance(ray_scene *s, uint32_t mi) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && mi < s->instances.size(), "invalid instance");
    s->instances.erase(s->instances.begin() + mi);
    s->inst_dirty = true;
    return RAY_OK;
}

int ray_scene_add_camera(ray_scene *s, const ray_camera_desc *c, uint32_t *out_index) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && c && out_index, "null argument");
    RG_GUARD_BEGIN
    // SceneBase::AddCamera, SceneBase.cpp:8-20
    uint32_t i;
    if (s->cam_first_free == RAY_INVALID_INDEX) {
        i = (uint32_t)s->cameras.size();
        s->cameras.emplace_back();
    } else {
        i = s->cam_first_free;
        s->cam_first_free = s->cameras[i].next_free;
    }
    s->cameras[i].alive = true;
    set_camera(s->cameras[i], *c);
    if (s->current_cam == RAY_INVALID_INDEX) s->current_cam = i;
    *out_index = i;
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_get_camera(ray_scene *s, uint32_t i, ray_camera_desc *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out && i < s->cameras.size() && s->cameras[i].alive, "invalid camera");
    // SceneBase::GetCamera, SceneBase.cpp:22-54: the fields of the camera's kind only
    // (origin, fwd and up of the constructed camera_t: up is the orthonormalised one)
    const CameraRec &rec = s->cameras[i];
    const ray_camera_desc &d = rec.desc;
    out->type = d.type;
    out->dtype = d.dtype;
    out->gamma = d.gamma;
    if (d.type != RAY_CAM_GEO) {
        out->filter = d.filter;
        memcpy(out->origin, rec.origin, sizeof(out->origin));
        memcpy(out->fwd, rec.fwd, sizeof(out->fwd));
        memcpy(out->up, rec.up, sizeof(out->up));
        out->fov = d.fov;
        out->focus_distance = d.focus_distance;
        out->focus_factor = d.focus_factor;
    } else {
        out->mi_index = d.mi_index;
        out->uv_index = d.uv_index;
    }
    out->lighting_only = d.lighting_only;
    out->skip_direct_lighting = d.skip_direct_lighting;
    out->skip_indirect_lighting = d.skip_indirect_lighting;
    out->no_background = d.no_background;
    out->clamp = d.clamp;
    out->output_sh = d.output_sh;
    out->use_coherent_sampling = d.use_coherent_sampling;
    out->max_diff_depth = d.max_diff_depth;
    out->max_glossy_depth = d.max_glossy_depth;
    out->max_refr_depth = d.max_refr_depth;
    out->max_transp_depth = d.max_transp_depth;
    out->max_total_depth = d.max_total_depth;
    out->termination_start_depth = d.termination_start_depth;
    return RAY_OK;
}

int ray_scene_set_camera(ray_scene *s, uint32_t i, const ray_camera_desc *c) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && c && i < s->cameras.size() && s->cameras[i].alive, "invalid camera");
    set_camera(s->cameras[i], *c);
    return RAY_OK;
}

int ray_scene_set_camera_axes(ray_scene *s, uint32_t i, const float side[3], const float up[3]) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && side && up && i < s->cameras.size() && s->cameras[i].alive, "invalid camera");
    memcpy(s->cameras[i].side, side, 3 * sizeof(float));
    memcpy(s->cameras[i].up, up, 3 * sizeof(float));
    return RAY_OK;
}

int ray_scene_remove_camera(ray_scene *s, uint32_t i) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && i < s->cameras.size() && s->cameras[i].alive, "invalid camera");
    s->cameras[i].alive = false;
    s->cameras[i].next_free = s->cam_first_free;
    s->cam_first_free = i;
    return RAY_OK;
}

int ray_scene_current_cam(ray_scene *s, uint32_t *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out, "null argument");
    *out = s->current_cam;
    return RAY_OK;
}

int ray_scene_set_current_cam(ray_scene *s, uint32_t i) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s, "null argument");
    s->current_cam = i;
    return RAY_OK;
}

int ray_scene_triangle_count(ray_scene *s, uint32_t *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out, "null argument");
    *out = s->total_tris;
    return RAY_OK;
}

int ray_scene_node_count(ray_scene *s, uint32_t *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out, "null argument");
    RG_GUARD_BEGIN
    const int rc = commit(s);
    if (rc != RAY_OK) return rc;
    *out = s->total_nodes;
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_commit(ray_scene *s) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s, "null argument");
    RG_GUARD_BEGIN
    return commit(s);
    RG_GUARD_END
}

int ray_scene_mesh_bvh_info(ray_scene *s, uint32_t mesh, ray_bvh_info *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out && mesh < s->meshes.size(), "invalid mesh");
    RG_GUARD_BEGIN
    const int rc = commit(s);
    if (rc != RAY_OK) return rc;
    const MeshRec &m = s->meshes[mesh];
    out->nodes = m.bvh.node_count;
    out->tris = m.bvh.tri_count;
    out->depth = m.bvh.depth;
    out->root = 0;
    for (int k = 0; k < 3; k++) {
        out->bbox_min[k] = m.bvh.bmin[k];
        out->bbox_max[k] = m.bvh.bmax[k];
    }
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_instance_tree_info(ray_scene *s, ray_instance_tree_info *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out, "null argument");
    RG_GUARD_BEGIN
    const int rc = commit(s);
    if (rc != RAY_OK) return rc;
    out->instances = s->tlas.nodes ? s->tlas.n : 0;
    out->refit = s->last_tlas_refit;
    out->ms = s->last_tlas_ms;
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_set_trace_tuning(ray_scene *s, const ray_trace_tuning *t) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && t, "null argument");
    RG_CHECK(t->kernel >= 0 && t->kernel <= 3, "kernel must be 1 (per ray), 2 (persistent) or 3 (persistent, one triangle per step)");
    RG_CHECK(t->refill_min <= 32, "refill_min is a lane count, at most 32");
    RG_CHECK(t->deep_stack == 0 || t->deep_stack == 1, "deep_stack is 0 or 1");
    RG_CHECK(t->reorder >= 0 && t->reorder <= 2, "reorder is 0 (input order), 1 (ray hash) or 2 (origin cell first)");
    RG_CHECK(t->reorder_bits == 0 || (t->reorder_bits >= 8 && t->reorder_bits <= 32), "reorder_bits is 0 or 8..32");
    RG_CHECK(t->block == 0 || t->block == 64 || t->block == 128 || t->block == 256, "block is 0, 64, 128 or 256");
    RG_CHECK(t->smem_stack == 0 || t->smem_stack == 16 || t->smem_stack == 24 || t->smem_stack == 32, "smem_stack is 0, 16, 24 or 32");
    RG_CHECK(!((t->block == 256) && t->smem_stack == 32), "256 threads with 32 stack entries exceed the block's shared memory");
    RG_CHECK(t->stream_hint == 0 || t->stream_hint == 1, "stream_hint is 0 or 1");
    RG_CHECK(t->l2_persist >= 0 && t->l2_persist <= 2, "l2_persist is 0, 1 (nodes) or 2 (leaf triangles)");
    RG_CHECK(t->instance_tree >= -1 && t->instance_tree <= 1, "instance_tree is -1, 0 or 1");
    if (t->kernel > 0) s->tuning.kernel = t->kernel;
    if (t->refill_min > 0) s->tuning.refill_min = t->refill_min;
    s->tuning.deep_stack = t->deep_stack;
    s->tuning.reorder = t->reorder;
    s->tuning.reorder_bits = t->reorder_bits ? t->reorder_bits : 32;
    s->tuning.block = t->block ? t->block : 64;
    s->tuning.smem_stack = t->smem_stack ? t->smem_stack : 16;
    s->tuning.stream_hint = t->stream_hint;
    s->tuning.l2_persist = t->l2_persist;
    if (t->instance_tree != s->tuning.instance_tree) s->inst_dirty = true; // built or dropped at the next commit
    s->tuning.instance_tree = t->instance_tree;
    return RAY_OK;
}

int ray_scene_get_trace_tuning(ray_scene *s, ray_trace_tuning *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out, "null argument");
    *out = s->tuning;
    return RAY_OK;
}

int ray_scene_set_counting(ray_scene *s, int enable) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s, "null argument");
    s->counting = enable != 0;
    return RAY_OK;
}

int ray_scene_last_trace_info(ray_scene *s, ray_trace_info *out) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out, "null argument");
    if (s->info_pending) {
        RG_CUDA_TRY(cudaSetDevice(s->device));
        RG_CUDA_TRY(wait_stream(s->info_stream));
        uint32_t err = 0;
        unsigned long long cnt[2] = {0, 0};
        RG_CUDA_TRY(cudaMemcpy(&err, s->d_err.p, 4, cudaMemcpyDeviceToHost));
        RG_CUDA_TRY(cudaMemcpy(cnt, s->d_counters.p, 16, cudaMemcpyDeviceToHost));
        s->last_info.error_flags = err;
        s->last_info.node_visits = cnt[0];
        s->last_info.tri_tests = cnt[1];
        s->info_pending = false;
    }
    *out = s->last_info;
    return RAY_OK;
}

namespace {
// Page-locked (or registered) host memory: copies from and to it run asynchronously.
bool host_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Rays per full chunk of a pipelined host-buffer trace: a quarter of the rays
// (the ends ramp down to quarter chunks), none below 256K rays (a chunk still
// fills the GPU); n itself when that leaves one. Measured on the 4M-ray
// microbench: 4.83 ms per call against 5.00 (eighths), 5.48 (sixteenths) and
// 7.79 without the pipeline. RAY_HOST_CHUNK=<rays> in the environment sets
// the chunk size (0: no pipeline).
uint64_t host_chunk(uint64_t n) {
    uint64_t c = std::max<uint64_t>(262144, ((n + 3) / 4 + 1023) & ~uint64_t(1023));
    if (const char *e = std::getenv("RAY_HOST_CHUNK")) {
        const long long v = std::atoll(e);
        c = v > 0 ? std::max<uint64_t>(1024, ((uint64_t)v + 1023) & ~uint64_t(1023)) : n;
    }
    return c >= n ? n : c;
}
} // namespace

// Reordered traces only from this many rays: below it the sort's fixed cost
// outweighs what the trace gains.
constexpr uint64_t kReorderMinRays = 65536;

int ray_scene_trace_closest(ray_scene *s, const float *rays, uint64_t n, ray_hit *hits, int32_t *obj, int mem, void *stream) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s, "null scene");
    RG_CHECK(n == 0 || (rays && hits), "null buffer");
    RG_CHECK(mem == RAY_MEM_HOST || mem == RAY_MEM_DEVICE, "invalid memory space");
    RG_CHECK(n <= 0xffffffffull, "too many rays in one call");
    RG_GUARD_BEGIN
    // host-buffer traces of one scene run one at a time; a caller that has to
    // wait for another thread's lets the API lock go meanwhile (the scene's
    // mutex first, then the API lock: the order every such call takes them)
    std::shared_ptr<std::mutex> host_mu;
    std::unique_lock<std::mutex> host_lock;
    if (mem == RAY_MEM_HOST) {
        host_mu = s->host_mu;
        host_lock = std::unique_lock<std::mutex>(*host_mu, std::try_to_lock);
        if (!host_lock.owns_lock()) {
            RG_CHECK(t_api_depth == 1, "a host-buffer trace of this scene is already running on this thread");
            api_mutex().unlock();
            try {
                host_lock.lock();
            } catch (...) {
                api_mutex().lock();
                throw;
            }
            api_mutex().lock();
            RG_CHECK(live_scene(s), "scene destroyed while the call waited for it");
        }
    }
    RG_CUDA_TRY(cudaSetDevice(s->device));
    int rc = commit(s);
    if (rc != RAY_OK) return rc;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
    RG_CUDA_TRY(s->d_err.ensure(4));
    RG_CUDA_TRY(s->d_counters.ensure(16));
    RG_CUDA_TRY(cudaMemsetAsync(s->d_err.p, 0, 4, st));
    RG_CUDA_TRY(cudaMemsetAsync(s->d_counters.p, 0, 16, st));
    const float4 *d_rays = reinterpret_cast<const float4 *>(rays);
    float4 *d_hits = reinterpret_cast<float4 *>(hits);
    int32_t *d_obj = obj;
    // host buffers in page-locked memory: a pipeline of chunks -- uploads on
    // one stream, downloads on another, the chunks' traces alternating between
    // the call's stream and a second one, so that copies overlap traces and a
    // chunk's trace starts while the previous one drains its last rays
    // (pageable buffers: one chunk)
    uint64_t chunk = n;
    if (mem == RAY_MEM_HOST && n) {
        RG_CUDA_TRY(s->d_rays.ensure(n * 32));
        RG_CUDA_TRY(s->d_hits.ensure(n * 16));
        if (obj) RG_CUDA_TRY(s->d_obj.ensure(n * 4));
        d_rays = static_cast<const float4 *>(s->d_rays.p);
        d_hits = static_cast<float4 *>(s->d_hits.p);
        d_obj = obj ? static_cast<int32_t *>(s->d_obj.p) : nullptr;
        if (host_pinned(rays) && host_pinned(hits) && (!obj || host_pinned(obj))) chunk = host_chunk(n);
    }
    const bool piped = chunk < n;
    // chunk boundaries: with three or more full chunks, the first two and the
    // last two ramp (a quarter, a half of a chunk) so that the first trace
    // starts early and the last download is short
    std::vector<uint64_t> cut{0};
    if (piped && n >= 4 * chunk) {
        const uint64_t q = std::max<uint64_t>(1024, (chunk / 4) & ~uint64_t(1023));
        const uint64_t mid = n - 6 * q, parts = (mid + chunk - 1) / chunk, step = ((mid + parts - 1) / parts + 1023) & ~uint64_t(1023);
        cut.push_back(q);
        cut.push_back(3 * q);
        for (uint64_t b = 3 * q + step; b < n - 3 * q; b += step) cut.push_back(b);
        cut.push_back(n - 3 * q);
        cut.push_back(n - q);
    } else {
        for (uint64_t b = chunk; b < n; b += chunk) cut.push_back(b);
    }
    cut.push_back(n);
    cudaStream_t up = st, down = st, other = st;
    if (piped) {
        for (int k = 0; k < 3; k++)
            if (!s->copy_st[k]) RG_CUDA_TRY(cudaStreamCreateWithFlags(&s->copy_st[k], cudaStreamNonBlocking));
        for (int k = 0; k < 4; k++)
            if (!s->pipe_ev[k]) RG_CUDA_TRY(cudaEventCreateWithFlags(&s->pipe_ev[k], cudaEventDisableTiming));
        up = s->copy_st[0];
        down = s->copy_st[1];
        other = s->copy_st[2];
        // the uploads and traces touch the staging buffers only after the caller's earlier work on st
        RG_CUDA_TRY(cudaEventRecord(s->pipe_ev[0], st));
        RG_CUDA_TRY(cudaStreamWaitEvent(up, s->pipe_ev[0], 0));
        RG_CUDA_TRY(cudaStreamWaitEvent(other, s->pipe_ev[0], 0));
    }
    SceneView sv{static_cast<const WideNode *>(s->d_nodes.p), static_cast<const TriRec *>(s->d_leaf.p),
                 static_cast<const InstanceRec *>(s->d_inst.p), s->n_inst_dev, s->tlas.nodes};
    RG_CUDA_TRY(s->d_next_ray.ensure(8)); // a work counter for each of two concurrent traces
    TraceParams tp;
    tp.persistent = s->tuning.kernel >= 2;
    tp.one_tri = s->tuning.kernel == 3;
    tp.refill_min = s->tuning.refill_min;
    tp.block = s->tuning.block;
    tp.smem_stack = s->tuning.smem_stack;
    tp.stream_hint = s->tuning.stream_hint;
    tp.tlas = s->tlas.nodes != nullptr;
    // L2 residency of the nodes or leaf triangles: an access-policy window on
    // the streams the traces run on, taken off again once they are enqueued
    cudaStreamAttrValue win{};
    if (s->tuning.l2_persist && n) {
        const DeviceBuf &b = s->tuning.l2_persist == 1 ? s->d_nodes : s->d_leaf;
        const size_t bytes = s->tuning.l2_persist == 1 ? (size_t)s->total_nodes * sizeof(WideNode) : (size_t)s->total_tris * sizeof(TriRec);
        int max_win = 0, max_persist = 0;
        RG_CUDA_TRY(cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, s->device));
        RG_CUDA_TRY(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, s->device));
        if (b.p && bytes && max_win > 0 && max_persist > 0) {
            const size_t w = std::min(bytes, (size_t)max_win);
            size_t limit = 0;
            RG_CUDA_TRY(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize));
            if (limit < std::min(w, (size_t)max_persist)) {
                RG_CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, std::min(w, (size_t)max_persist)));
                RG_CUDA_TRY(cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize));
            }
            win.accessPolicyWindow.base_ptr = b.p;
            win.accessPolicyWindow.num_bytes = w;
            win.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)limit / (double)w);
            win.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
            win.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        }
    }
    for (const MeshRec &m : s->meshes) tp.max_depth = std::max(tp.max_depth, m.bvh.depth);
    if (s->tuning.deep_stack) tp.max_depth = 0xffffffffu;
    uint32_t *next_ray = static_cast<uint32_t *>(s->d_next_ray.p);
    // reordered traces: the hash grid of SortRays_CPU over the scene's box (RendererRef.cpp:48-77)
    const bool reorder = s->tuning.reorder != 0;
    float cell[3];
    for (int a = 0; a < 3; a++) cell[a] = (s->world_max[a] - s->world_min[a]) / 255.0f;
    int k = 0;
    for (size_t c = 0; c + 1 < cut.size(); c++, k++) {
        const uint64_t b = cut[c], m = cut[c + 1] - b;
        // chunk k's trace: on st or `other` in turn, with its own work counter
        // (the chunk before the previous one, on the same stream, is done with it)
        cudaStream_t ts = (k & 1) ? other : st;
        tp.next_ray = next_ray + (k & 1);
        if (mem == RAY_MEM_HOST && m) {
            RG_CUDA_TRY(cudaMemcpyAsync(static_cast<float4 *>(s->d_rays.p) + 2 * b, rays + 8 * b, m * 32, cudaMemcpyHostToDevice, up));
            if (piped) {
                RG_CUDA_TRY(cudaEventRecord(s->pipe_ev[1], up));
                RG_CUDA_TRY(cudaStreamWaitEvent(ts, s->pipe_ev[1], 0));
            }
        }
        tp.order = nullptr;
        if (reorder && m >= kReorderMinRays && m <= RS_MAX_ITEMS) {
            // the chunk's trace order (scratch of this chunk's parity, like the work counter)
            RG_CUDA_TRY(s->d_order[k & 1].ensure(order_scratch_bytes(m)));
            uint32_t *order = nullptr;
            RG_CUDA_TRY(order_rays(d_rays + 2 * b, (uint32_t)m, s->world_min, cell, s->tuning.reorder, s->tuning.reorder_bits,
                                   s->d_order[k & 1].p, &order, ts));
            tp.order = order;
        }
        if (win.accessPolicyWindow.num_bytes) RG_CUDA_TRY(cudaStreamSetAttribute(ts, cudaStreamAttributeAccessPolicyWindow, &win));
        RG_CUDA_TRY(launch_trace_closest(sv, d_rays + 2 * b, (uint32_t)m, d_hits + b, d_obj ? d_obj + b : nullptr,
                                         static_cast<uint32_t *>(s->d_err.p), static_cast<unsigned long long *>(s->d_counters.p), s->counting,
                                         ts, tp));
        if (win.accessPolicyWindow.num_bytes) {
            cudaStreamAttrValue off{};
            RG_CUDA_TRY(cudaStreamSetAttribute(ts, cudaStreamAttributeAccessPolicyWindow, &off));
        }
        if (mem == RAY_MEM_HOST && m && piped) { // (pageable buffers: the download below, without the API lock)
            RG_CUDA_TRY(cudaEventRecord(s->pipe_ev[2], ts));
            RG_CUDA_TRY(cudaStreamWaitEvent(down, s->pipe_ev[2], 0));
            RG_CUDA_TRY(cudaMemcpyAsync(hits + b, d_hits + b, m * 16, cudaMemcpyDeviceToHost, down));
            if (obj) RG_CUDA_TRY(cudaMemcpyAsync(obj + b, d_obj + b, m * 4, cudaMemcpyDeviceToHost, down));
        }
        if (n == 0) break;
    }
    if (piped) { // the call's stream ends after the last download
        RG_CUDA_TRY(cudaEventRecord(s->pipe_ev[3], down));
        RG_CUDA_TRY(cudaStreamWaitEvent(st, s->pipe_ev[3], 0));
    }
    RG_CUDA_TRY(note_use(s, st));
    s->info_pending = true;
    s->info_stream = st;
    const uint64_t seq = ++s->trace_seq;
    if (mem == RAY_MEM_HOST) {
        // this call's error word and counters, copied behind its work (another
        // thread's trace of the scene may reset the device words meanwhile)
        if (!s->h_info) RG_CUDA_TRY(cudaHostAlloc(reinterpret_cast<void **>(&s->h_info), 32, cudaHostAllocDefault));
        RG_CUDA_TRY(cudaMemcpyAsync(s->h_info, s->d_err.p, 4, cudaMemcpyDeviceToHost, st));
        RG_CUDA_TRY(cudaMemcpyAsync(s->h_info + 2, s->d_counters.p, 16, cudaMemcpyDeviceToHost, st));
        // the download of pageable buffers and the wait for the GPU work, without
        // the API lock when this is the outermost entry point of the thread
        const bool release = t_api_depth == 1;
        if (release) api_mutex().unlock();
        cudaError_t we = cudaSuccess;
        if (!piped && n) {
            we = cudaMemcpyAsync(hits, d_hits, n * 16, cudaMemcpyDeviceToHost, st);
            if (we == cudaSuccess && obj) we = cudaMemcpyAsync(obj, d_obj, n * 4, cudaMemcpyDeviceToHost, st);
        }
        if (we == cudaSuccess) we = wait_stream(st);
        if (release) api_mutex().lock();
        RG_CHECK(live_scene(s), "scene destroyed while the call waited for its GPU work");
        RG_CUDA_TRY(we);
        ray_trace_info info;
        info.error_flags = s->h_info[0];
        unsigned long long cnt[2];
        memcpy(cnt, s->h_info + 2, 16);
        info.node_visits = cnt[0];
        info.tri_tests = cnt[1];
        if (s->trace_seq == seq) { // no later trace of the scene was enqueued meanwhile
            s->last_info = info;
            s->info_pending = false;
        }
        if (info.error_flags & TRACE_ERR_STACK) {
            set_error("traversal stack overflow");
            return RAY_ERR_STACK_OVERFLOW;
        }
        if (info.error_flags) {
            set_error("traversal found a corrupt BVH (index or visit bound)");
            return RAY_ERR_CUDA;
        }
    }
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_debug_read(ray_scene *s, int what, void *dst, uint64_t bytes, uint64_t *out_bytes) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && out_bytes, "null argument");
    RG_CHECK(what >= 0 && what <= 2, "invalid array selector");
    RG_GUARD_BEGIN
    RG_CUDA_TRY(cudaSetDevice(s->device));
    const int rc = commit(s);
    if (rc != RAY_OK) return rc;
    uint64_t total = 0;
    const void *src = nullptr;
    if (what == 0) {
        total = (uint64_t)s->total_nodes * sizeof(WideNode);
        src = s->d_nodes.p;
    } else if (what == 1) {
        total = (uint64_t)s->total_tris * sizeof(TriRec);
        src = s->d_leaf.p;
    } else {
        total = (uint64_t)s->n_inst_dev * sizeof(InstanceRec);
        src = s->d_inst.p;
    }
    *out_bytes = total;
    const uint64_t n = std::min(total, bytes);
    if (n && dst) RG_CUDA_TRY(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost));
    return RAY_OK;
    RG_GUARD_END
}

int ray_scene_debug_write(ray_scene *s, int what, uint64_t offset, const void *src, uint64_t bytes) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && (src || bytes == 0), "null argument");
    RG_CHECK(what == 0 || what == 1, "invalid array selector");
    RG_GUARD_BEGIN
    RG_CUDA_TRY(cudaSetDevice(s->device));
    const int rc = commit(s);
    if (rc != RAY_OK) return rc;
    const uint64_t total = what == 0 ? (uint64_t)s->total_nodes * sizeof(WideNode) : (uint64_t)s->total_tris * sizeof(TriRec);
    RG_CHECK(offset <= total && bytes <= total - offset, "write outside the array");
    char *dst = static_cast<char *>(what == 0 ? s->d_nodes.p : s->d_leaf.p);
    // after the work in flight that reads the scene
    for (auto &u : s->users) RG_CUDA_TRY(cudaStreamWaitEvent(s->stream, u.second, 0));
    if (bytes) RG_CUDA_TRY(cudaMemcpyAsync(dst + offset, src, bytes, cudaMemcpyHostToDevice, s->stream));
    RG_CUDA_TRY(wait_stream(s->stream));
    return RAY_OK;
    RG_GUARD_END
}

int ray_debug_fail_device_alloc(int64_t after) {
    g_fail_alloc_after.store(after < 0 ? -1 : (long long)after);
    return RAY_OK;
}

int ray_set_wait_timeout_ms(int64_t ms) {
    g_wait_timeout_ms.store(ms <= 0 ? 300000 : (long long)ms);
    return RAY_OK;
}

namespace {
// Scene signature -> the tuner's choice (process-wide, under the API lock).
struct TuneKey {
    uint64_t tris, nodes, inst, depth, log2n;
    bool operator<(const TuneKey &o) const {
        return std::tie(tris, nodes, inst, depth, log2n) < std::tie(o.tris, o.nodes, o.inst, o.depth, o.log2n);
    }
};
std::map<TuneKey, ray_trace_tuning> &tune_cache() {
    static std::map<TuneKey, ray_trace_tuning> c;
    return c;
}
} // namespace

int ray_scene_tune_trace(ray_scene *s, const float *rays, uint64_t n, ray_hit *hits, int flags, void *stream, ray_trace_tuning *out,
                         char *report, uint64_t report_cap) {
    RG_API_LOCK;
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    RG_CHECK(s && rays && hits && n > 0, "null argument or no rays");
    RG_CHECK(n <= 0xffffffffull, "too many rays in one call");
    RG_GUARD_BEGIN
    RG_CUDA_TRY(cudaSetDevice(s->device));
    int rc = commit(s);
    if (rc != RAY_OK) return rc;
    uint64_t lg = 0;
    while ((2ull << lg) <= n) lg++;
    const TuneKey key{s->total_tris, s->total_nodes, s->n_inst_dev, s->max_depth, lg};
    std::string log;
    auto finish = [&]() {
        if (out) *out = s->tuning;
        if (report && report_cap) {
            const size_t m = std::min<size_t>(log.size(), report_cap - 1);
            memcpy(report, log.data(), m);
            report[m] = 0;
        }
    };
    auto it = tune_cache().find(key);
    if (it != tune_cache().end() && !(flags & 1)) {
        s->tuning = it->second;
        log = "cached";
        finish();
        return RAY_OK;
    }
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    RG_CUDA_TRY(cudaEventCreate(&e0));
    RG_CUDA_TRY(cudaEventCreate(&e1));
    auto time_of = [&](const ray_trace_tuning &t, float &best) -> int {
        s->tuning = t;
        best = 1e30f;
        for (int k = 0; k < 3; k++) {
            RG_CUDA_TRY(cudaEventRecord(e0, st));
            const int r2 = ray_scene_trace_closest(s, rays, n, hits, nullptr, RAY_MEM_DEVICE, st);
            if (r2 != RAY_OK) return r2;
            RG_CUDA_TRY(cudaEventRecord(e1, st));
            RG_CUDA_TRY(wait_event(e1));
            float ms = 0.0f;
            RG_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
            if (k > 0) best = std::min(best, ms); // the first is the untimed one
        }
        return RAY_OK;
    };
    ray_trace_tuning cur = s->tuning;
    float cur_ms = 0.0f;
    auto name_of = [](const ray_trace_tuning &t) {
        char b[160];
        snprintf(b, sizeof b, "k%d_r%d_l2%d_h%d_b%d_s%d_o%d_%d", t.kernel, t.refill_min, t.l2_persist, t.stream_hint, t.block, t.smem_stack,
                 t.reorder, t.reorder_bits);
        return std::string(b);
    };
    rc = time_of(cur, cur_ms);
    if (rc == RAY_OK) {
        log += name_of(cur) + "=" + std::to_string(cur_ms) + ";";
        // one setting at a time, each stage starting from the best so far
        using Mut = std::function<void(ray_trace_tuning &)>;
        std::vector<std::vector<Mut>> stages = {
            {[](ray_trace_tuning &t) { t.kernel = 2; }, [](ray_trace_tuning &t) { t.kernel = 3; }, [](ray_trace_tuning &t) { t.kernel = 1; }},
            {[](ray_trace_tuning &t) { t.l2_persist = 0; }, [](ray_trace_tuning &t) { t.l2_persist = 1; },
             [](ray_trace_tuning &t) { t.l2_persist = 2; }},
            {[](ray_trace_tuning &t) { t.stream_hint = 0; }, [](ray_trace_tuning &t) { t.stream_hint = 1; }},
            {[](ray_trace_tuning &t) { t.refill_min = 4; }, [](ray_trace_tuning &t) { t.refill_min = 8; },
             [](ray_trace_tuning &t) { t.refill_min = 12; }, [](ray_trace_tuning &t) { t.refill_min = 16; }},
            {[](ray_trace_tuning &t) { t.block = 64; t.smem_stack = 16; }, [](ray_trace_tuning &t) { t.block = 128; t.smem_stack = 24; },
             [](ray_trace_tuning &t) { t.block = 64; t.smem_stack = 24; },
             [](ray_trace_tuning &t) { t.block = 256; t.smem_stack = 24; }, [](ray_trace_tuning &t) { t.block = 128; t.smem_stack = 16; },
             [](ray_trace_tuning &t) { t.block = 64; t.smem_stack = 32; }, [](ray_trace_tuning &t) { t.block = 256; t.smem_stack = 16; }},
            {[](ray_trace_tuning &t) { t.reorder = 0; t.reorder_bits = 32; }, [](ray_trace_tuning &t) { t.reorder = 1; t.reorder_bits = 32; },
             [](ray_trace_tuning &t) { t.reorder = 2; t.reorder_bits = 24; }}};
        for (size_t si = 0; si < stages.size() && rc == RAY_OK; si++) {
            if (si > 0 && cur.kernel == 1 && si != 5) continue; // the per-ray kernel takes only the trace order
            ray_trace_tuning best_t = cur;
            float best_ms = cur_ms;
            for (const Mut &mut : stages[si]) {
                ray_trace_tuning t = cur;
                mut(t);
                if (memcmp(&t, &cur, sizeof t) == 0) continue;
                float ms = 0.0f;
                rc = time_of(t, ms);
                if (rc != RAY_OK) break;
                log += name_of(t) + "=" + std::to_string(ms) + ";";
                if (ms < best_ms) {
                    best_ms = ms;
                    best_t = t;
                }
            }
            cur = best_t;
            cur_ms = best_ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->tuning = cur;
    if (rc != RAY_OK) return rc;
    tune_cache()[key] = cur;
    log += "chosen=" + name_of(cur);
    finish();
    return RAY_OK;
    RG_GUARD_END
}

// ---- renderer entry points that do not need the render loop
} // extern "C"
