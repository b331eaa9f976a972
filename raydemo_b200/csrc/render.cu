// Render-loop entry points of the C ABI: RendererBase::RenderScene as a
// wavefront on one stream (ray generation, then per bounce a closest-hit
// trace and a shading kernel that appends the continuation rays), the
// framebuffer accessors, Resize/Clear and the stats.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <random>
#include <tuple>

#include "../../include/raygpu.h"
#include "radix_sort.cuh"
#include "scene.hpp"
#include "sort.cuh"

using namespace rg;

#define RG_CHECK(cond, msg)                                                                                            \
    do {                                                                                                               \
        if (!(cond)) {                                                                                                 \
            set_error(msg);                                                                                            \
            return RAY_ERR_INVALID_ARG;                                                                                \
        }                                                                                                              \
    } while (0)

namespace {

constexpr int MAX_BOUNCES = 10; // Core.h:53
constexpr int TUNE_SAMPLES = 2; // timed frames per kernel before the choice
constexpr int N_EVENTS = ray_renderer::N_EVENTS; // 4 + 3 * MAX_BOUNCES + 1
static_assert(N_EVENTS == 5 + 3 * MAX_BOUNCES, "one event per phase");
constexpr uint32_t SORT_ALL = (1u << MAX_BOUNCES) - 1u;
// events of bounce b: it starts at ev[3 + 3b] (the end of the previous shade)
constexpr int ev_sorted(int b) { return 4 + 3 * b; }
constexpr int ev_traced(int b) { return 5 + 3 * b; }
constexpr int ev_shaded(int b) { return 6 + 3 * b; }

// ComputeRadicalInversePermutations + Shuffle (src/Ray/internal/Halton.h:7-43)
// fed as RendererRef.cpp:10-13 does: uniform_int_distribution<int> over mt19937(0).
std::vector<uint16_t> halton_permutations() {
    static const int primes[HALTON_COUNT] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89};
    auto rand_func = std::bind(std::uniform_int_distribution<int>(), std::mt19937(0));
    std::vector<uint16_t> perms;
    for (int i = 0; i < HALTON_COUNT; i++) {
        const int count = primes[i];
        const size_t base = perms.size();
        for (int j = 0; j < count; j++) perms.push_back((uint16_t)j);
        uint16_t *p = perms.data() + base;
        for (int j = 0; j < count; j++) {
            const uint32_t thres = (~((uint32_t)count) + 1u) % (uint32_t)count;
            int other;
            while (true) {
                const uint32_t r = (uint32_t)rand_func();
                if (r >= thres) {
                    other = (int)(r % (uint32_t)count);
                    break;
                }
            }
            std::swap(p[j], p[other]);
        }
    }
    return perms;
}

int ensure_frame_buffers(ray_renderer *r, bool sh) {
    const size_t n = (size_t)r->w * r->h;
    const bool fresh = r->d_temp.p == nullptr;
    RG_CUDA_TRY(r->d_temp.ensure(n * sizeof(float4)));
    RG_CUDA_TRY(r->d_clean.ensure(n * sizeof(float4)));
    RG_CUDA_TRY(r->d_final.ensure(n * sizeof(float4)));
    if (fresh) {
        RG_CUDA_TRY(cudaMemsetAsync(r->d_temp.p, 0, n * sizeof(float4), r->stream));
        RG_CUDA_TRY(cudaMemsetAsync(r->d_clean.p, 0, n * sizeof(float4), r->stream));
        RG_CUDA_TRY(cudaMemsetAsync(r->d_final.p, 0, n * sizeof(float4), r->stream));
    }
    if (sh && r->d_temp_sh.p == nullptr) {
        RG_CUDA_TRY(r->d_temp_sh.ensure(n * sizeof(SHData)));
        RG_CUDA_TRY(r->d_clean_sh.ensure(n * sizeof(SHData)));
        RG_CUDA_TRY(cudaMemsetAsync(r->d_temp_sh.p, 0, n * sizeof(SHData), r->stream));
        RG_CUDA_TRY(cudaMemsetAsync(r->d_clean_sh.p, 0, n * sizeof(SHData), r->stream));
    }
    return RAY_OK;
}

// The wavefront's ray buffers: two generations of n rays, their hits and instance ids.
int ensure_ray_buffers(ray_renderer *r, size_t n) {
    for (int k = 0; k < 2; k++) {
        RG_CUDA_TRY(r->d_rays[k].ensure(n * 2 * sizeof(float4)));
        RG_CUDA_TRY(r->d_pay[k].ensure(n * sizeof(RayPayload)));
    }
    RG_CUDA_TRY(r->d_hits.ensure(n * sizeof(float4)));
    RG_CUDA_TRY(r->d_obj.ensure(n * sizeof(int32_t)));
    return RAY_OK;
}

// Counters, the sample table and its permutations, the stats events.
int ensure_frame_state(ray_renderer *r) {
    RG_CUDA_TRY(r->d_counters.ensure(16 * sizeof(uint32_t)));
    if (!r->d_perms.p) {
        const std::vector<uint16_t> perms = halton_permutations();
        RG_CUDA_TRY(r->d_perms.ensure(perms.size() * sizeof(uint16_t)));
        RG_CUDA_TRY(cudaMemcpy(r->d_perms.p, perms.data(), perms.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
        RG_CUDA_TRY(r->d_halton.ensure(HALTON_TABLE_FLOATS * sizeof(float)));
        RG_CUDA_TRY(cudaMemsetAsync(r->d_halton.p, 0, HALTON_TABLE_FLOATS * sizeof(float), r->stream));
    }
    if (!r->ev_sets[0][0]) {
        for (int s = 0; s < 2; s++)
            for (int e = 0; e < N_EVENTS; e++) RG_CUDA_TRY(cudaEventCreate(&r->ev_sets[s][e]));
        RG_CUDA_TRY(cudaEventCreateWithFlags(&r->ev_sync, cudaEventDisableTiming));
        for (int e = 0; e < 2; e++) RG_CUDA_TRY(cudaEventCreate(&r->ev_batch[e]));
    }
    return RAY_OK;
}

// Trace settings the frame tuner times for the wavefront: one triangle test
// per lane and step (bit 0: in the closest-hit traces, bit 1: in the
// shadow-ray traces) or a node's triangles at once, a refill
// threshold, threads per block and shared stack entries (the block and stack
// apply to one-scene closest-hit launches). Index 0 takes the scene's refill,
// block and stack (ray_scene_set_trace_tuning) with a node's triangles at
// once: measured on the atrium (1280x720, 16 spp; refill 16, 128 threads, 24
// entries), one triangle per step made the closest-hit traces 2.5 ms and the
// shadow-ray traces 1.7 ms per frame slower (62.7 ms per frame with neither,
// 67.7 with both), while it is the faster form for the incoherent rays of
// ray_scene_trace_closest.
struct TraceVariant {
    int one, refill, block, stack;
};
constexpr TraceVariant TRACE_VARIANTS[] = {{0, 0, 0, 0}, {0, 8, 128, 24}, {0, 16, 128, 24}, {0, 8, 64, 24}, {3, 4, 64, 16}, {3, 8, 128, 16}};
constexpr int N_TRACE_VARIANTS = (int)(sizeof(TRACE_VARIANTS) / sizeof(TRACE_VARIANTS[0]));
static_assert(3 + N_TRACE_VARIANTS - 1 == ray_renderer::N_VARIANTS, "frame variants: 3 plus the trace variants after the first");

// The tuner's choices across renderers: a frame configuration seen before
// (triangle and light counts, pixels, bounces, the renderer's settings) takes
// the kernel, sort mask and trace settings chosen then, with no timed frames.
struct TuneSig {
    uint32_t tris, lights, pixels;
    int bounces, kernel_setting, sort_setting, trace_setting;
    bool operator<(const TuneSig &o) const {
        return std::tie(tris, lights, pixels, bounces, kernel_setting, sort_setting, trace_setting) <
               std::tie(o.tris, o.lights, o.pixels, o.bounces, o.kernel_setting, o.sort_setting, o.trace_setting);
    }
};
struct TuneChoice {
    int kernel;
    uint32_t mask;
    int trace_var;
};
std::map<TuneSig, TuneChoice> &tune_cache() {
    static std::map<TuneSig, TuneChoice> c;
    return c;
}
TuneSig sig_of(const ray_renderer::TuneEntry &t) {
    return TuneSig{t.tris, t.lights, t.pixels, t.bounces, t.kernel_setting, t.sort_setting, t.trace_setting};
}

// Finishes the timing of a tune entry once every variant it times has its
// samples: the sort mask (per bounce, sorting where its timed bounce was
// faster) and the kernel (the path kernel against the wavefront's time with
// that mask, estimated from the per-bounce times).
void finish_tune(ray_renderer::TuneEntry &t) {
    const bool tune_kernel = t.kernel_setting == 0, tune_sort = t.sort_setting < 0, tune_trace = t.trace_setting < 0;
    if (t.n[0] < TUNE_SAMPLES || (tune_kernel && t.n[1] < TUNE_SAMPLES) || (tune_sort && t.n[2] < TUNE_SAMPLES)) return;
    if (tune_trace)
        for (int v = 3; v < ray_renderer::N_VARIANTS; v++)
            if (t.n[v] < TUNE_SAMPLES) return;
    // the trace settings: the fastest unsorted wavefront frame among them
    int tv = tune_trace ? 0 : t.trace_setting;
    float trace_gain = 0.0f;
    if (tune_trace)
        for (int v = 3; v < ray_renderer::N_VARIANTS; v++)
            if (t.best[v] < t.best[0] - trace_gain) {
                trace_gain = t.best[0] - t.best[v];
                tv = v - 2;
            }
    t.trace_var = tv;
    float wave = t.best[0] - trace_gain;
    uint32_t mask = tune_sort ? 0u : (uint32_t)t.sort_setting & SORT_ALL;
    if (tune_sort) {
        for (int b = 0; b < t.bounces && b < MAX_BOUNCES; b++) {
            if (t.bounce_ms[1][b] < t.bounce_ms[0][b]) {
                mask |= 1u << b;
                wave -= t.bounce_ms[0][b] - t.bounce_ms[1][b];
            }
        }
        wave = std::min(wave, t.best[2]);
        if (t.best[2] < t.best[0] && mask == 0) mask = SORT_ALL; // per-bounce noise hid the gain
    }
    t.mask = mask;
    t.choice = (tune_kernel && t.best[1] < wave) ? 2 : 1;
    tune_cache()[sig_of(t)] = TuneChoice{t.choice, t.mask, t.trace_var};
}

// Adds the phase times of a finished frame to the stats (stats_t, RendererBase.h:93-100).
int resolve_stats(ray_renderer *r, int set) {
    if (!r->ev_frame_pending[set]) return RAY_OK;
    cudaEvent_t *e = r->ev_sets[set];
    const int nb = r->ev_bounces[set];
    RG_CUDA_TRY(wait_event(e[N_EVENTS - 1]));
    auto ms_between = [&](int a, int b) -> float {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e[a], e[b]);
        return ms;
    };
    auto us = [&](int a, int b) -> unsigned long long { return (unsigned long long)(ms_between(a, b) * 1000.0f); };
    r->stats.time_primary_ray_gen_us += us(0, 1);
    r->stats.time_primary_trace_us += us(1, 2);
    r->stats.time_primary_shade_us += us(2, 3);
    for (int b = 0; b < nb; b++) {
        r->stats.time_secondary_sort_us += us(3 + 3 * b, ev_sorted(b));
        r->stats.time_secondary_trace_us += us(ev_sorted(b), ev_traced(b));
        r->stats.time_secondary_shade_us += us(ev_traced(b), ev_shaded(b));
    }
    // a frame the kernel and sort choice is timing
    const int ti = r->ev_tune[set];
    if (ti >= 0 && ti < (int)r->tune.size()) {
        ray_renderer::TuneEntry &t = r->tune[ti];
        const int v = r->ev_variant[set];
        t.best[v] = std::min(t.best[v], ms_between(0, N_EVENTS - 1));
        if (v == 0 || v == 2)
            for (int b = 0; b < nb && b < MAX_BOUNCES; b++) {
                float &slot = t.bounce_ms[v == 2 ? 1 : 0][b];
                const float ms = ms_between(3 + 3 * b, ev_shaded(b));
                slot = (slot == 0.0f) ? ms : std::min(slot, ms);
            }
        t.n[v]++;
        if (t.pending[v] > 0) t.pending[v]--;
        finish_tune(t);
    }
    r->ev_tune[set] = -1;
    r->ev_frame_pending[set] = false;
    return RAY_OK;
}

// How a frame runs: the kernel, the sort mask of the wavefront, and, for a
// frame that times a variant of its configuration, the tune entry and variant.
struct FramePlan {
    int kernel = 1;
    uint32_t sort_mask = 0;
    int trace_var = 0; // index of TRACE_VARIANTS
    int tune_entry = -1, variant = 0;
};

// The variant of an untimed-enough entry to run next: the one with the
// fewest timed plus in-flight frames among those the settings leave open.
int next_variant(const ray_renderer::TuneEntry &t) {
    int best = 0;
    for (int v = 1; v < ray_renderer::N_VARIANTS; v++) {
        if (v == 1 && t.kernel_setting != 0) continue;
        if (v == 2 && t.sort_setting >= 0) continue;
        if (v >= 3 && t.trace_setting >= 0) continue;
        if (t.n[v] + t.pending[v] < t.n[best] + t.pending[best]) best = v;
    }
    return best;
}

FramePlan plan_of_variant(const ray_renderer::TuneEntry &t, int v) {
    FramePlan p;
    p.variant = v;
    p.kernel = v == 1 ? 2 : 1;
    p.sort_mask = v == 2 ? SORT_ALL : (t.sort_setting >= 0 ? (uint32_t)t.sort_setting & SORT_ALL : 0u);
    p.trace_var = v >= 3 ? v - 2 : (t.trace_setting >= 0 ? t.trace_setting : 0);
    return p;
}

// Per frame configuration (scene, its triangle and light counts, rect size,
// bounces, the renderer's settings), the kernel and the sort mask: the
// caller's fixed settings, else timed on the configuration's first frames
// (TUNE_SAMPLES per variant, the best kept; every variant gives the same image).
// bounces < 0 marks a batch configuration (-samples; lights then holds the count).
FramePlan plan_frame(ray_renderer *r, const void *s, uint32_t tris, uint32_t lights, uint32_t pixels, int bounces, bool geo = false) {
    FramePlan p;
    if (geo) { // the path kernel generates camera rays only: Geo cameras run on the wavefront
        p.sort_mask = r->sort_policy >= 0 ? (uint32_t)r->sort_policy & SORT_ALL : 0u;
        return p;
    }
    if (r->kernel == 2) {
        p.kernel = 2;
        return p;
    }
    if (r->kernel == 1 && r->sort_policy >= 0 && r->trace_policy >= 0) {
        p.sort_mask = (uint32_t)r->sort_policy & SORT_ALL;
        p.trace_var = r->trace_policy;
        return p;
    }
    for (size_t i = 0; i < r->tune.size(); i++) {
        ray_renderer::TuneEntry &t = r->tune[i];
        if (t.scene == s && t.tris == tris && t.lights == lights && t.pixels == pixels && t.bounces == bounces &&
            t.kernel_setting == r->kernel && t.sort_setting == r->sort_policy && t.trace_setting == r->trace_policy) {
            if (t.choice) {
                p.kernel = t.choice;
                p.sort_mask = t.choice == 1 ? t.mask : 0u;
                p.trace_var = t.choice == 1 ? t.trace_var : 0;
                return p;
            }
            p = plan_of_variant(t, next_variant(t));
            p.tune_entry = (int)i;
            return p;
        }
    }
    if (r->tune.size() >= 64) { // forget them all (the frames in flight lose their timing)
        r->tune.clear();
        r->ev_tune[0] = r->ev_tune[1] = -1;
    }
    ray_renderer::TuneEntry t;
    t.scene = s;
    t.tris = tris;
    t.lights = lights;
    t.pixels = pixels;
    t.bounces = bounces;
    t.kernel_setting = r->kernel;
    t.sort_setting = r->sort_policy;
    t.trace_setting = r->trace_policy;
    const auto cached = tune_cache().find(sig_of(t));
    if (cached != tune_cache().end()) { // chosen before for this signature
        t.choice = cached->second.kernel;
        t.mask = cached->second.mask;
        t.trace_var = cached->second.trace_var;
        r->tune.push_back(t);
        p.kernel = t.choice;
        p.sort_mask = t.choice == 1 ? t.mask : 0u;
        p.trace_var = t.choice == 1 ? t.trace_var : 0;
        return p;
    }
    r->tune.push_back(t);
    p = plan_of_variant(t, 0);
    p.tune_entry = (int)r->tune.size() - 1;
    return p;
}

// RegionContext's sample table (RendererRef.cpp:85-89): regenerated on the
// first call and every 256 iterations. For a region that starts at
// iteration 0 its base is 1 until iteration 255, then the iteration rounded
// down to a multiple of 256.
int table_base(int iteration) { return iteration < HALTON_SEQ_LEN ? 1 : (iteration & ~(HALTON_SEQ_LEN - 1)); }

constexpr int PREPARE_NOTHING = 1; // the call renders nothing (a scene of another device)

// One RenderScene call up to its kernels: checks, the scene's device data,
// frame buffers, the region's iteration and sample table (on the renderer's
// stream), and the job both kernels read.
int prepare_job(ray_renderer *r, ray_scene *s, ray_region *region, FrameJob &J, ray_rect &rect, int samples = 1) {
    if (!r || !s || !region) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (s->device != r->device) return PREPARE_NOTHING; // as the reference's failed scene cast: a no-op
    if (s->current_cam >= s->cameras.size() || !s->cameras[s->current_cam].alive) {
        set_error("the scene has no current camera");
        return RAY_ERR_INVALID_ARG;
    }
    const CameraRec &cam = s->cameras[s->current_cam];
    const ray_camera_desc &cd = cam.desc;
    if (cd.type != RAY_CAM_PERSP && cd.type != RAY_CAM_GEO) {
        set_error("only perspective and Geo cameras are rendered");
        return RAY_ERR_UNSUPPORTED;
    }
    if (cd.type == RAY_CAM_GEO && (cd.mi_index >= s->instances.size() || cd.uv_index > 1)) {
        set_error("Geo camera: mi_index must name an instance and uv_index be 0 or 1");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    int rc = commit(s);
    if (rc != RAY_OK) return rc;
    const int w = r->w, h = r->h;
    rect = region->rect;
    if (rect.w == 0 || rect.h == 0) rect = ray_rect{0, 0, w, h};
    if (rect.x < 0 || rect.y < 0 || rect.w < 0 || rect.h < 0 || rect.x + rect.w > w || rect.y + rect.h > h) {
        set_error("region outside the framebuffer");
        return RAY_ERR_INVALID_ARG;
    }
    const bool sh = cd.output_sh != 0;
    rc = ensure_frame_buffers(r, sh);
    if (rc != RAY_OK) return rc;
    rc = ensure_frame_state(r);
    if (rc != RAY_OK) return rc;

    // `samples` consecutive iterations, all in one block of the sample table
    const int it = region->iteration + 1;
    region->iteration += samples;
    const int base = table_base(it);
    if (base != r->halton_base) {
        RG_CUDA_TRY(launch_halton_table(static_cast<const uint16_t *>(r->d_perms.p), base, static_cast<float *>(r->d_halton.p), r->stream));
        r->halton_base = base;
    }

    J = FrameJob{};
    J.sc = render_scene_view(s);
    PassInfo &pi = J.pi;
    pi.iteration = it;
    pi.bounce = 2;
    pi.flags = (cd.lighting_only ? PASS_LIGHTING_ONLY : 0u) | (cd.skip_direct_lighting ? PASS_SKIP_DIRECT : 0u) |
               (cd.skip_indirect_lighting ? PASS_SKIP_INDIRECT : 0u) | (cd.no_background ? PASS_NO_BACKGROUND : 0u) |
               (cd.clamp ? PASS_CLAMP : 0u) | (cd.output_sh ? PASS_OUTPUT_SH : 0u) | (cd.use_coherent_sampling ? PASS_COHERENT : 0u);
    // pass_settings_t holds uint8 depths (Types.h:47-55); the total is capped at MAX_BOUNCES (RendererRef.cpp:111)
    pi.max_diff_depth = (uint8_t)cd.max_diff_depth;
    pi.max_glossy_depth = (uint8_t)cd.max_glossy_depth;
    pi.max_refr_depth = (uint8_t)cd.max_refr_depth;
    pi.max_transp_depth = (uint8_t)cd.max_transp_depth;
    pi.max_total_depth = std::min((int)(uint8_t)cd.max_total_depth, MAX_BOUNCES);
    pi.termination_start_depth = (uint8_t)cd.termination_start_depth;
    pi.w = w;
    // camera constants of GeneratePrimaryRays (CoreRef.cpp:430-432), computed on the host as on the CPU
    J.cam.filter = cd.filter;
    J.cam.fov = cd.fov;
    J.cam.focus_distance = cd.focus_distance;
    J.cam.focus_factor = cd.focus_factor;
    for (int k = 0; k < 3; k++) {
        J.cam.origin[k] = cam.origin[k];
        J.cam.fwd[k] = cam.fwd[k];
        J.cam.side[k] = cam.side[k];
        J.cam.up[k] = cam.up[k];
    }
    const float PI = 3.141592653589793238463f;
    J.k = float(w) / h;
    J.fov_k = std::tan(0.5f * cd.fov * PI / 180.0f) * cd.focus_distance;
    J.rx = rect.x;
    J.ry = rect.y;
    J.rw = rect.w;
    J.rh = rect.h;
    J.w = w;
    J.h = h;
    if (cd.type == RAY_CAM_GEO) {
        // the instance's mesh, its transform, and its index among the device's
        // instances (the hit's obj; instances of empty meshes have none)
        const InstanceRecHost &ih = s->instances[cd.mi_index];
        const MeshRec &m = s->meshes[ih.mesh];
        GeoCam &g = J.geo;
        g.on = 1;
        g.tri0 = m.tris_index;
        g.ntri = m.tris_count;
        g.uv = cd.uv_index;
        g.obj = 0;
        for (uint32_t q = 0; q < cd.mi_index; q++) g.obj += s->meshes[s->instances[q].mesh].tris_count ? 1u : 0u;
        for (int row = 0; row < 3; row++)
            for (int col = 0; col < 4; col++) g.xf[row * 4 + col] = ih.xform[col * 4 + row];
        for (int row = 0; row < 3; row++)
            for (int col = 0; col < 3; col++) g.inv[row * 3 + col] = ih.inv_xform[row * 4 + col];
    }
    J.halton = static_cast<const float *>(r->d_halton.p);
    J.temp = static_cast<float4 *>(r->d_temp.p);
    J.clean = static_cast<float4 *>(r->d_clean.p);
    J.fin = static_cast<float4 *>(r->d_final.p);
    J.temp_sh = sh ? static_cast<SHData *>(r->d_temp_sh.p) : nullptr;
    J.clean_sh = sh ? static_cast<SHData *>(r->d_clean_sh.p) : nullptr;
    // accumulation and tone (RendererRef.cpp:292-324)
    J.mix_k = 1.0f / it;
    J.gamma = cd.gamma;
    J.srgb = cd.dtype == 1 ? 1 : 0;
    J.clamp = cd.clamp != 0 ? 1 : 0;
    J.bounces = (pi.flags & PASS_SKIP_INDIRECT) ? 0 : pi.max_total_depth;
    J.samples = samples;
    J.pixel_base = 0;
    // the ray hash grid (RendererRef.cpp:48-77): the scene's box in 255 cells per axis
    for (int k = 0; k < 3; k++) {
        J.root_min[k] = s->world_min[k];
        J.cell[k] = (s->world_max[k] - s->world_min[k]) / 255;
    }
    r->pixels_on_host = r->sh_on_host = false;
    return RAY_OK;
}

// The wavefront over the jobs in d_jobs (host copies in jobs): ray generation,
// per bounce a closest-hit trace and a shading launch over the rays of all
// jobs, then the accumulation. Buffers and counters are rb's. sample: offset
// from each job's first iteration. ev (may be null): stats events.
// FNV-1a over the values a captured launch sequence depends on.
struct GraphKey {
    uint64_t h = 1469598103934665603ull;
    template <typename T>
    GraphKey &add(const T &v) {
        const unsigned char *p = reinterpret_cast<const unsigned char *>(&v);
        for (size_t i = 0; i < sizeof(T); i++) h = (h ^ p[i]) * 1099511628211ull;
        return *this;
    }
};

// Enqueues a launch sequence through a cached CUDA graph: the first call with
// a new key runs it directly (its buffers get allocated then), the second
// captures and instantiates it, later ones replay it. A capture that fails
// falls back to running the sequence directly.
// RAY_GRAPHS=0 in the environment turns graph replay off (every call enqueues directly).
bool graphs_enabled() {
    static const int on = [] {
        const char *v = std::getenv("RAY_GRAPHS");
        return (v && v[0] == '0') ? 0 : 1;
    }();
    return on != 0;
}

template <typename F>
int graph_run(GraphSlot &g, uint64_t key, cudaStream_t st, F &&enqueue) {
    if (!graphs_enabled()) return enqueue();
    if (g.key != key) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
        g.key = key;
        g.runs = 0;
    }
    if (g.exec) {
        RG_CUDA_TRY(cudaGraphLaunch(g.exec, st));
        return RAY_OK;
    }
    if (g.runs++ == 0 || g.failed) return enqueue();
    cudaGraph_t graph = nullptr;
    const cudaError_t eb = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    const int rc = eb == cudaSuccess ? enqueue() : RAY_ERR_CUDA;
    const cudaError_t ee = eb == cudaSuccess ? cudaStreamEndCapture(st, &graph) : eb;
    cudaError_t ei = cudaErrorUnknown;
    if (rc == RAY_OK && ee == cudaSuccess && graph) ei = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (ei == cudaSuccess) {
        RG_CUDA_TRY(cudaGraphLaunch(g.exec, st));
        return RAY_OK;
    }
    if (std::getenv("RAY_GRAPH_DEBUG"))
        fprintf(stderr, "graph capture failed: begin %d, enqueue %d (%s), end %d, instantiate %d\n", (int)eb, rc, ray_last_error(), (int)ee,
                (int)ei);
    g.exec = nullptr;
    g.failed = true;
    cudaGetLastError(); // the capture's error, if any, is not the caller's
    return enqueue();
}

// The adjoint's replay (adj in run_wavefront): its arguments and per-ray state buffers.
struct AdjointRun {
    AdjArgs args;
    AdjState *state[2];
    AdjShadowRec *recs;
};

int run_wavefront(ray_renderer *rb, const FrameJob *d_jobs, const std::vector<FrameJob> &jobs, const std::vector<const ray_scene *> &scn,
                  uint32_t total, int sample0, uint32_t sort_mask, cudaStream_t st, cudaEvent_t *ev, int &nb, bool resolve = true,
                  const AdjointRun *adj = nullptr, int samples = 1, GraphSlot *gs = nullptr, int trace_var = 0) {
    nb = 0;
    if (adj) sort_mask = 0; // the replay keeps the forward pass's order
    int rc = ensure_ray_buffers(rb, std::max<size_t>(total, 1));
    if (rc != RAY_OK) return rc;
    if (sort_mask) RG_CUDA_TRY(rb->d_loop_sort.ensure(loop_sort_scratch_bytes(std::max<size_t>(total, 1), (int)jobs.size())));
    // light samples of RAY_MAT_PRINCIPLED vertices wait in d_shadow (count in counter [8])
    // for their shadow rays; the reference's own lights are traced inside the shading
    bool ref_lights = false, nee = false, principled_only = true;
    for (const FrameJob &J : jobs) {
        ref_lights = ref_lights || J.sc.n_lights > 0;
        nee = nee || J.sc.n_area_lights > 0;
        principled_only = principled_only && J.sc.principled_only;
    }
    ShadowQueue shadow{nullptr, nullptr, nullptr, nullptr};
    if (nee || adj) {
        if (!adj) RG_CUDA_TRY(rb->d_shadow.ensure(std::max<size_t>(total, 1) * sizeof(ShadowRec)));
        RG_CUDA_TRY(rb->d_shadow_rays.ensure(std::max<size_t>(total, 1) * 2 * sizeof(float4)));
        RG_CUDA_TRY(rb->d_shadow_job.ensure(std::max<size_t>(total, 1) * sizeof(uint32_t)));
        shadow.recs = adj ? static_cast<void *>(adj->recs) : rb->d_shadow.p;
        shadow.rays = static_cast<float4 *>(rb->d_shadow_rays.p);
        shadow.job = static_cast<uint32_t *>(rb->d_shadow_job.p);
    }
    for (int k = 0; k < 2; k++) RG_CUDA_TRY(rb->d_job[k].ensure(std::max<size_t>(total, 1) * sizeof(uint32_t)));
    uint32_t *cnt = static_cast<uint32_t *>(rb->d_counters.p);
    unsigned long long *ray_stats = reinterpret_cast<unsigned long long *>(cnt + 4);
    uint32_t *err = cnt + 3;
    uint32_t *shadow_cnt = cnt + 8;
    shadow.count = shadow_cnt;
    float4 *rays[2] = {static_cast<float4 *>(rb->d_rays[0].p), static_cast<float4 *>(rb->d_rays[1].p)};
    RayPayload *pay[2] = {static_cast<RayPayload *>(rb->d_pay[0].p), static_cast<RayPayload *>(rb->d_pay[1].p)};
    uint32_t *job[2] = {static_cast<uint32_t *>(rb->d_job[0].p), static_cast<uint32_t *>(rb->d_job[1].p)};
    float4 *hits = static_cast<float4 *>(rb->d_hits.p);
    int32_t *obj = static_cast<int32_t *>(rb->d_obj.p);
    const int n_jobs = (int)jobs.size();
    int bounces = 0;
    TraceParams tp;
    tp.persistent = scn[0]->tuning.kernel >= 2;
    tp.refill_min = scn[0]->tuning.refill_min;
    for (int j = 0; j < n_jobs; j++) {
        bounces = std::max(bounces, jobs[j].bounces);
        tp.max_depth = std::max(tp.max_depth, scn[j]->tuning.deep_stack ? 0xffffffffu : scn[j]->max_depth);
        if (scn[j]->tlas.nodes) tp.tlas = true; // the kernels that can walk an instance tree
    }
    tp.block = scn[0]->tuning.block;
    tp.smem_stack = scn[0]->tuning.smem_stack;
    bool one_any = false; // shadow-ray traces: one triangle test per step
    if (trace_var > 0 && trace_var < N_TRACE_VARIANTS) { // the frame tuner's trace settings
        tp.refill_min = TRACE_VARIANTS[trace_var].refill;
        tp.block = TRACE_VARIANTS[trace_var].block;
        tp.smem_stack = TRACE_VARIANTS[trace_var].stack;
        tp.one_tri = (TRACE_VARIANTS[trace_var].one & 1) != 0;
        one_any = (TRACE_VARIANTS[trace_var].one & 2) != 0;
    }
    tp.next_ray = cnt + 2;
    if (n_jobs > 1) { // each ray traced in its job's scene
        tp.views = reinterpret_cast<const uint8_t *>(d_jobs) + offsetof(FrameJob, sc) + offsetof(RenderScene, sv);
        tp.view_stride = (uint32_t)sizeof(FrameJob);
    }
    // Geo (lightmap) jobs take their primary hits from the UV-space sampling
    bool persp = false;
    uint32_t geo_tris = 0;
    for (const FrameJob &J : jobs) {
        if (J.geo.on) geo_tris = std::max(geo_tris, std::max(J.geo.ntri, 1u));
        else persp = true;
    }
    uint32_t *geo_best = nullptr;
    if (geo_tris) {
        RG_CUDA_TRY(rb->d_geo_best.ensure(std::max<size_t>(total, 1) * sizeof(uint32_t)));
        geo_best = static_cast<uint32_t *>(rb->d_geo_best.p);
    }
    const SceneView &sv = jobs[0].sc.sv;
    auto enqueue_sample = [&](int sample) -> int {
        // primary rays (GeneratePrimaryRays, CoreRef.cpp:427-505)
        RG_CUDA_TRY(cudaMemsetAsync(cnt, 0, 2 * sizeof(uint32_t), st));
        RG_CUDA_TRY(launch_raygen_jobs(d_jobs, n_jobs, total, sample, rays[0], pay[0], job[0], cnt + 0, st));
        if (ev) RG_CUDA_TRY(cudaEventRecord(ev[1], st));
        tp.count = cnt + 0;
        tp.ray_job = job[0];
        if (persp) RG_CUDA_TRY(launch_trace_closest(sv, rays[0], total, hits, obj, err, nullptr, false, st, tp));
        if (geo_tris) {
            // SampleMeshInTextureSpace (RendererRef.cpp:142-146): rays and hits of the Geo jobs' texels
            RG_CUDA_TRY(cudaMemsetAsync(geo_best, 0xff, (size_t)total * sizeof(uint32_t), st));
            RG_CUDA_TRY(launch_geo_cover(d_jobs, n_jobs, geo_tris, sample, geo_best, st));
            RG_CUDA_TRY(launch_geo_rays(d_jobs, n_jobs, total, sample, geo_best, rays[0], pay[0], hits, obj, st));
        }
        if (ev) RG_CUDA_TRY(cudaEventRecord(ev[2], st));
        // shadow rays of the light samples: the persistent kernel in any-hit mode (the hits buffer is free again)
        TraceParams tps = tp;
        tps.any = true;
        tps.one_tri = one_any;
        tps.count = shadow_cnt;
        tps.ray_job = shadow.job;
        // shading of the rays in buffer `in` (bounce b), continuation rays to `out`, then the light samples'
        // shadow rays and the colour of the unblocked ones
        auto shade = [&](int b, int in, int out) -> cudaError_t {
            cudaError_t e = cudaSuccess;
            if (nee || adj) e = cudaMemsetAsync(shadow_cnt, 0, sizeof(uint32_t), st);
            if (e != cudaSuccess) return e;
            if (adj)
                e = launch_adjoint_shade(d_jobs, b, rays[in], pay[in], job[in], adj->state[in], hits, obj, cnt + in, total, rays[out], pay[out],
                                         job[out], adj->state[out], cnt + out, shadow, adj->args, err, st, ref_lights, principled_only);
            else
                e = launch_shade_jobs(d_jobs, sample, b, rays[in], pay[in], job[in], hits, obj, cnt + in, total, rays[out], pay[out], job[out],
                                      cnt + out, shadow, ref_lights, principled_only, err, ray_stats, st);
            if (e != cudaSuccess || !(nee || adj)) return e;
            e = launch_trace_closest(sv, shadow.rays, total, hits, nullptr, err, nullptr, false, st, tps);
            if (e != cudaSuccess) return e;
            if (adj) return launch_adjoint_shadow_apply(d_jobs, b, shadow, hits, total, adj->state[out], adj->args, err, st);
            return launch_shadow_apply(d_jobs, sample, b, shadow, hits, total, err, ray_stats, st);
        };
        RG_CUDA_TRY(shade(2, 0, 1));
        if (ev) RG_CUDA_TRY(cudaEventRecord(ev[3], st));
        // bounces (RendererRef.cpp:183-278); ray counts stay on the device
        int cur = 1;
        for (int bounce = 0; bounce < bounces; bounce++) {
            if ((sort_mask >> bounce) & 1u) {
                // SortRays_CPU before each bounce (RendererRef.cpp:200-203): the rays move to the other buffer in hash order
                const int dst = cur ^ 1;
                RG_CUDA_TRY(launch_loop_sort(d_jobs, (int)jobs.size(), rays[cur], pay[cur], job[cur], cnt + cur, total, rays[dst], pay[dst], job[dst],
                                             cnt + dst, rb->d_loop_sort.p, st, err));
                cur = dst;
            }
            if (ev) RG_CUDA_TRY(cudaEventRecord(ev[ev_sorted(bounce)], st));
            const int nxt = cur ^ 1;
            RG_CUDA_TRY(cudaMemsetAsync(cnt + nxt, 0, sizeof(uint32_t), st));
            tp.count = cnt + cur;
            tp.ray_job = job[cur];
            RG_CUDA_TRY(launch_trace_closest(sv, rays[cur], total, hits, obj, err, nullptr, false, st, tp));
            if (ev) RG_CUDA_TRY(cudaEventRecord(ev[ev_traced(bounce)], st));
            RG_CUDA_TRY(shade(bounce + 3, cur, nxt));
            if (ev) RG_CUDA_TRY(cudaEventRecord(ev[ev_shaded(bounce)], st));
            cur = nxt;
        }
        // accumulate and tone (RendererRef.cpp:292-324)
        if (resolve) RG_CUDA_TRY(launch_resolve_jobs(d_jobs, n_jobs, total, sample, st));
        return RAY_OK;
    };
    // the samples one after another (each a whole wavefront)
    auto enqueue = [&]() -> int {
        for (int k = 0; k < samples; k++) {
            const int rc2 = enqueue_sample(sample0 + k);
            if (rc2 != RAY_OK) return rc2;
        }
        return RAY_OK;
    };
    nb = bounces;
    if (!gs) return enqueue();
    // everything the launches take by value or point at: the graph is replayed while all of it is unchanged
    GraphKey key;
    key.add(d_jobs).add(n_jobs).add(total).add(sample0).add(samples).add(sort_mask).add(bounces).add(resolve).add(adj).add(st);
    for (int q = 0; q < 2; q++) key.add(rays[q]).add(pay[q]).add(job[q]);
    key.add(hits).add(obj).add(cnt).add(shadow.recs).add(shadow.rays).add(shadow.job).add(rb->d_loop_sort.p).add(nee).add(ref_lights).add(principled_only);
    key.add(sv.nodes).add(sv.leaf_tris).add(sv.inst).add(sv.n_inst).add(tp.persistent).add(tp.refill_min).add(tp.max_depth).add(tp.views);
    key.add(sv.tlas).add(tp.tlas).add(tp.block).add(tp.smem_stack).add(tp.one_tri);
    key.add(ev).add(geo_best).add(geo_tris).add(persp);
    return graph_run(*gs, key.h, st, enqueue);
}

// The jobs of a differentiable render: sample k (iteration first + k) as job k,
// each summing into its own w x h slice of d_diff_temp; the whole frame.
int diff_jobs(ray_renderer *r, ray_scene *s, int first_iteration, int samples, std::vector<FrameJob> &jobs, uint32_t &n_pix) {
    if (!r || !s) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (first_iteration < 1 || samples < 1 || samples > HALTON_SEQ_LEN ||
        table_base(first_iteration) != table_base(first_iteration + samples - 1)) {
        set_error("the samples' iterations (from 1) must lie in one block of 256");
        return RAY_ERR_INVALID_ARG;
    }
    ray_region reg{{0, 0, 0, 0}, first_iteration - 1};
    FrameJob J;
    ray_rect rect;
    int rc = prepare_job(r, s, &reg, J, rect, 1);
    if (rc == PREPARE_NOTHING) {
        set_error("the scene belongs to another device");
        return RAY_ERR_INVALID_ARG;
    }
    if (rc != RAY_OK) return rc;
    n_pix = (uint32_t)r->w * (uint32_t)r->h;
    if ((uint64_t)n_pix * samples > 0xffffffffull) {
        set_error("too many pixels x samples");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(r->d_diff_temp.ensure((size_t)n_pix * samples * sizeof(float4)));
    jobs.assign(samples, J);
    for (int k = 0; k < samples; k++) {
        FrameJob &Jk = jobs[k];
        Jk.pi.iteration = first_iteration + k;
        Jk.temp = static_cast<float4 *>(r->d_diff_temp.p) + (size_t)k * n_pix;
        Jk.temp_sh = Jk.clean_sh = nullptr;
        Jk.pixel_base = (uint32_t)k * n_pix;
    }
    RG_CUDA_TRY(r->d_jobs.ensure(jobs.size() * sizeof(FrameJob)));
    RG_CUDA_TRY(cudaMemcpyAsync(r->d_jobs.p, jobs.data(), jobs.size() * sizeof(FrameJob), cudaMemcpyHostToDevice, r->stream));
    return RAY_OK;
}

} // namespace

ray_renderer::~ray_renderer() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (int s = 0; s < 2; s++)
        for (int e = 0; e < N_EVENTS; e++)
            if (ev_sets[s][e]) cudaEventDestroy(ev_sets[s][e]);
    if (ev_sync) cudaEventDestroy(ev_sync);
    for (int e = 0; e < 2; e++)
        if (ev_batch[e]) cudaEventDestroy(ev_batch[e]);
    if (batch_graph.exec) cudaGraphExecDestroy(batch_graph.exec);
    if (own_stream) cudaStreamDestroy(own_stream);
}

extern "C" {

int ray_sort_rays(ray_renderer *r, const float *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                  uint32_t *perm_out, float *rays_out, void *stream) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || !root_min || !cell_size || (n && (!rays || !perm_out))) {
        set_error("ray_sort_rays: null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (n > RS_MAX_ITEMS) {
        set_error("ray_sort_rays: at most 2^30 - 1 rays per call");
        return RAY_ERR_INVALID_ARG;
    }
    if (n == 0) return RAY_OK;
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(r->d_sort_scratch.ensure(sort_rays_scratch_bytes(n)));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : r->stream;
    RG_CUDA_TRY(sort_rays(reinterpret_cast<const float4 *>(rays), n, root_min, cell_size, keys_out, perm_out,
                          reinterpret_cast<float4 *>(rays_out), r->d_sort_scratch.p, st));
    return RAY_OK;
}

int ray_resize(ray_renderer *r, int w, int h) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || w <= 0 || h <= 0 || w > 32768 || h > 32768) {
        set_error("invalid size");
        return RAY_ERR_INVALID_ARG;
    }
    if (w == r->w && h == r->h) return RAY_OK;
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(wait_stream(r->stream));
    // Framebuffer::Resize (FramebufferRef.cpp:10-27): the pixel array keeps
    // its leading elements and the new ones are zero
    const size_t n_old = (size_t)r->w * r->h, n_new = (size_t)w * h;
    DeviceBuf *bufs[3] = {&r->d_temp, &r->d_clean, &r->d_final};
    for (DeviceBuf *b : bufs) {
        if (!b->p) continue;
        DeviceBuf nb;
        RG_CUDA_TRY(nb.ensure(n_new * sizeof(float4)));
        RG_CUDA_TRY(cudaMemset(nb.p, 0, n_new * sizeof(float4)));
        RG_CUDA_TRY(cudaMemcpy(nb.p, b->p, std::min(n_old, n_new) * sizeof(float4), cudaMemcpyDeviceToDevice));
        std::swap(b->p, nb.p);
        std::swap(b->bytes, nb.bytes);
    }
    r->d_temp_sh.release();
    r->d_clean_sh.release();
    r->w = w;
    r->h = h;
    r->pixels_on_host = r->sh_on_host = false;
    return RAY_OK;
}

int ray_clear(ray_renderer *r, const ray_pixel *c) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r) {
        set_error("null renderer");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    int rc = ensure_frame_buffers(r, false);
    if (rc != RAY_OK) return rc;
    // RendererRef::Clear (RendererRef.h:78-80): the accumulation buffer only
    const ray_pixel v = c ? *c : ray_pixel{0.0f, 0.0f, 0.0f, 0.0f};
    RG_CUDA_TRY(launch_fill(static_cast<float4 *>(r->d_clean.p), (size_t)r->w * r->h, make_float4(v.r, v.g, v.b, v.a), r->stream));
    if (r->d_clean_sh.p) RG_CUDA_TRY(launch_fill_sh(static_cast<SHData *>(r->d_clean_sh.p), (size_t)r->w * r->h, r->stream));
    return RAY_OK;
}

int ray_render(ray_renderer *r, ray_scene *s, ray_region *region) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    try {
        FrameJob J;
        ray_rect rect;
        int rc = prepare_job(r, s, region, J, rect);
        if (rc == PREPARE_NOTHING) return RAY_OK;
        if (rc != RAY_OK) return rc;
        cudaStream_t st = r->stream;
        const size_t n_pix = (size_t)rect.w * rect.h;

        // stats of the frame two calls back are complete by now or soon
        const int set = (int)(r->frame & 1);
        rc = resolve_stats(r, set);
        if (rc != RAY_OK) return rc;
        cudaEvent_t *ev = r->ev_sets[set];
        const FramePlan plan =
            plan_frame(r, s, s->total_tris, (uint32_t)(s->lights.size() + s->area_lights.size()), (uint32_t)n_pix, J.bounces, J.geo.on != 0);
        const int kern = plan.kernel;

        uint32_t *cnt = static_cast<uint32_t *>(r->d_counters.p);
        // [0], [1] ray counts of the two buffers, [2] trace / path work counter,
        // [3] error flags, [4..7] two uint64: rays traced, shadow segments
        RG_CUDA_TRY(cudaMemsetAsync(cnt, 0, 8 * sizeof(uint32_t), st));
        unsigned long long *ray_stats = reinterpret_cast<unsigned long long *>(cnt + 4);
        uint32_t *err = cnt + 3;
        RG_CUDA_TRY(cudaEventRecord(ev[0], st));
        int nb = 0;
        RG_CUDA_TRY(r->d_jobs.ensure(sizeof(FrameJob)));
        RG_CUDA_TRY(cudaMemcpyAsync(r->d_jobs.p, &J, sizeof(FrameJob), cudaMemcpyHostToDevice, st));
        const FrameJob *d_jobs = static_cast<const FrameJob *>(r->d_jobs.p);
        if (kern == 2) {
            // the whole frame in one launch; its time counts as primary trace in the stats
            RG_CUDA_TRY(cudaEventRecord(ev[1], st));
            RG_CUDA_TRY(launch_render_paths(d_jobs, 1, (uint32_t)n_pix, cnt + 2, err, ray_stats, st));
            RG_CUDA_TRY(cudaEventRecord(ev[2], st));
            RG_CUDA_TRY(cudaEventRecord(ev[3], st));
        } else {
            // launched directly: its phase events feed the stats and the kernel and sort choice
            rc = run_wavefront(r, d_jobs, std::vector<FrameJob>{J}, std::vector<const ray_scene *>{s}, (uint32_t)n_pix, 0, plan.sort_mask, st,
                               ev, nb, true, nullptr, 1, nullptr, plan.trace_var);
            if (rc != RAY_OK) return rc;
        }
        RG_CUDA_TRY(cudaEventRecord(ev[N_EVENTS - 1], st));
        RG_CUDA_TRY(note_use(s, st));
        r->ev_bounces[set] = nb;
        r->ev_tune[set] = plan.tune_entry;
        r->ev_kernel[set] = kern;
        r->ev_variant[set] = plan.variant;
        if (plan.tune_entry >= 0) r->tune[plan.tune_entry].pending[plan.variant]++;
        r->ev_frame_pending[set] = true;
        r->last_kernel = kern;
        r->last_sort_mask = kern == 1 ? plan.sort_mask : 0u;
        r->last_trace_var = kern == 1 ? plan.trace_var : 0;
        r->frame++;
        return RAY_OK;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return RAY_ERR_OUT_OF_MEMORY;
    }
}

int ray_render_batch(ray_renderer *const *renderers, ray_scene *const *scenes, ray_region *const *regions, int count, int samples) {
    RG_API_LOCK;
    if (count < 0 || samples < 1 || (count > 0 && (!renderers || !scenes || !regions))) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (count == 0) return RAY_OK;
    try {
        ray_renderer *r0 = renderers[0];
        for (int i = 0; i < count; i++) {
            if (renderers[i] && scenes[i] && (!live_renderer(renderers[i]) || !live_scene(scenes[i]))) {
                set_error("unknown or destroyed renderer or scene handle");
                return RAY_ERR_INVALID_ARG;
            }
            if (!renderers[i] || !scenes[i] || !regions[i]) {
                set_error("null argument");
                return RAY_ERR_INVALID_ARG;
            }
            if (renderers[i]->device != r0->device) {
                set_error("a batch runs on one device: all renderers must share it");
                return RAY_ERR_INVALID_ARG;
            }
            for (int j = 0; j < i; j++) {
                if (regions[j] == regions[i]) {
                    set_error("a region appears twice in the batch");
                    return RAY_ERR_INVALID_ARG;
                }
                // one sample table per renderer and launch: its regions advance in step
                if (renderers[j] == renderers[i] && regions[j]->iteration != regions[i]->iteration) {
                    set_error("regions of one renderer in one batch must be at the same iteration");
                    return RAY_ERR_INVALID_ARG;
                }
            }
        }
        RG_CUDA_TRY(cudaSetDevice(r0->device));
        int rc = ensure_frame_state(r0);
        if (rc != RAY_OK) return rc;
        cudaStream_t st = r0->stream;
        // kernel: the first renderer's setting; by default per batch configuration the
        // faster of the two, timed (blocking) on the configuration's first calls
        uint64_t px_all = 0, tris_all = 0;
        for (int i = 0; i < count; i++) {
            const ray_rect &q = regions[i]->rect;
            px_all += (q.w == 0 || q.h == 0) ? (uint64_t)renderers[i]->w * renderers[i]->h : (uint64_t)q.w * q.h;
            tris_all += scenes[i]->total_tris;
        }
        // kernel and sort: the first renderer's settings; what they leave open is
        // chosen per batch configuration by timing (blocking) its first calls
        bool any_geo = false;
        for (int i = 0; i < count; i++) {
            const ray_scene *q = scenes[i];
            any_geo = any_geo || (q->current_cam < q->cameras.size() && q->cameras[q->current_cam].desc.type == RAY_CAM_GEO);
        }
        const FramePlan plan = plan_frame(r0, scenes[0], (uint32_t)tris_all, (uint32_t)count, (uint32_t)px_all, -samples, any_geo);
        const int kern = plan.kernel, tune_entry = plan.tune_entry;
        if (tune_entry >= 0) RG_CUDA_TRY(cudaEventRecord(r0->ev_batch[0], st));
        for (int done = 0; done < samples;) {
            // a run of iterations that keeps every region within one block of 256 (one sample table each)
            int run = samples - done;
            for (int i = 0; i < count; i++) run = std::min(run, HALTON_SEQ_LEN - ((regions[i]->iteration + 1) & (HALTON_SEQ_LEN - 1)));
            std::vector<FrameJob> jobs;
            std::vector<const ray_scene *> jscn;
            jobs.reserve(count);
            uint64_t total = 0;
            for (int i = 0; i < count; i++) {
                FrameJob J;
                ray_rect rect;
                rc = prepare_job(renderers[i], scenes[i], regions[i], J, rect, run);
                if (rc == PREPARE_NOTHING) continue;
                if (rc != RAY_OK) return rc;
                J.pixel_base = (uint32_t)total;
                total += (uint64_t)rect.w * rect.h;
                if (total > 0xffffffffull) {
                    set_error("too many pixels in one batch");
                    return RAY_ERR_INVALID_ARG;
                }
                jobs.push_back(J);
                jscn.push_back(scenes[i]);
            }
            // the batch runs on the first renderer's stream, after each renderer's own work
            for (int i = 0; i < count; i++) {
                ray_renderer *r = renderers[i];
                if (r->stream == st) continue;
                RG_CUDA_TRY(cudaEventRecord(r->ev_sync, r->stream));
                RG_CUDA_TRY(cudaStreamWaitEvent(st, r->ev_sync, 0));
            }
            uint32_t *cnt = static_cast<uint32_t *>(r0->d_counters.p);
            RG_CUDA_TRY(cudaMemsetAsync(cnt, 0, 8 * sizeof(uint32_t), st));
            if (!jobs.empty()) {
                RG_CUDA_TRY(r0->d_jobs.ensure(jobs.size() * sizeof(FrameJob)));
                RG_CUDA_TRY(cudaMemcpyAsync(r0->d_jobs.p, jobs.data(), jobs.size() * sizeof(FrameJob), cudaMemcpyHostToDevice, st));
                const FrameJob *d_jobs = static_cast<const FrameJob *>(r0->d_jobs.p);
                if (kern == 2) {
                    RG_CUDA_TRY(launch_render_paths(d_jobs, (int)jobs.size(), (uint32_t)total, cnt + 2, cnt + 3,
                                                    reinterpret_cast<unsigned long long *>(cnt + 4), st));
                } else {
                    // one wavefront per sample over the rays of all jobs, the run as one CUDA graph
                    int nb = 0;
                    rc = run_wavefront(r0, d_jobs, jobs, jscn, (uint32_t)total, 0, plan.sort_mask, st, nullptr, nb, true, nullptr, run,
                                       &r0->batch_graph, plan.trace_var);
                    if (rc != RAY_OK) return rc;
                }
            }
            // and each renderer's later work (reads of its pixels, its next frames) after the batch
            for (int i = 0; i < count; i++)
                if (scenes[i]->device == r0->device) RG_CUDA_TRY(note_use(scenes[i], st));
            RG_CUDA_TRY(cudaEventRecord(r0->ev_sync, st));
            for (int i = 0; i < count; i++) {
                ray_renderer *r = renderers[i];
                if (r->stream != st) RG_CUDA_TRY(cudaStreamWaitEvent(r->stream, r0->ev_sync, 0));
                r->last_kernel = kern;
                r->last_sort_mask = kern == 1 ? plan.sort_mask : 0u;
                r->last_trace_var = kern == 1 ? plan.trace_var : 0;
        r->last_trace_var = kern == 1 ? plan.trace_var : 0;
            }
            done += run;
        }
        if (tune_entry >= 0) { // a timed call of the kernel choice
            RG_CUDA_TRY(cudaEventRecord(r0->ev_batch[1], st));
            RG_CUDA_TRY(wait_event(r0->ev_batch[1]));
            float ms = 0.0f;
            RG_CUDA_TRY(cudaEventElapsedTime(&ms, r0->ev_batch[0], r0->ev_batch[1]));
            ray_renderer::TuneEntry &e = r0->tune[tune_entry];
            e.best[plan.variant] = std::min(e.best[plan.variant], ms);
            e.n[plan.variant]++;
            finish_tune(e); // no per-bounce times here: the sort runs before every bounce or none
        }
        return RAY_OK;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return RAY_ERR_OUT_OF_MEMORY;
    }
}

int ray_renderer_set_trace_variant(ray_renderer *r, int variant) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || variant < -1 || variant >= N_TRACE_VARIANTS) {
        set_error("trace variant must be -1 (chosen by timing) or an index of the tuner's trace settings");
        return RAY_ERR_INVALID_ARG;
    }
    r->trace_policy = variant;
    return RAY_OK;
}

int ray_renderer_set_kernel(ray_renderer *r, int kernel) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || kernel < 0 || kernel > 2) {
        set_error("kernel must be 0 (chosen by timing), 1 (wavefront) or 2 (path kernel)");
        return RAY_ERR_INVALID_ARG;
    }
    r->kernel = kernel;
    return RAY_OK;
}

int ray_render_diff(ray_renderer *r, ray_scene *s, int first_iteration, int samples, float *image_rgb, float *sample_rgb) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    try {
        if (!image_rgb || !sample_rgb) {
            set_error("null output buffer");
            return RAY_ERR_INVALID_ARG;
        }
        std::vector<FrameJob> jobs;
        uint32_t n_pix = 0;
        int rc = diff_jobs(r, s, first_iteration, samples, jobs, n_pix);
        if (rc != RAY_OK) return rc;
        cudaStream_t st = r->stream;
        uint32_t *cnt = static_cast<uint32_t *>(r->d_counters.p);
        RG_CUDA_TRY(cudaMemsetAsync(cnt, 0, 16 * sizeof(uint32_t), st));
        const FrameJob *d_jobs = static_cast<const FrameJob *>(r->d_jobs.p);
        int nb = 0;
        rc = run_wavefront(r, d_jobs, jobs, std::vector<const ray_scene *>(jobs.size(), s), n_pix * (uint32_t)samples, 0, 0u, st, nullptr, nb,
                           false);
        if (rc != RAY_OK) return rc;
        RG_CUDA_TRY(launch_diff_collect(d_jobs, samples, n_pix, image_rgb, sample_rgb, st));
        RG_CUDA_TRY(note_use(s, st));
        r->last_kernel = 1;
        r->last_sort_mask = 0;
        return RAY_OK;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return RAY_ERR_OUT_OF_MEMORY;
    }
}

int ray_render_adjoint(ray_renderer *r, ray_scene *s, int first_iteration, int samples, const float *sample_rgb, const float *d_image,
                       float *grad_albedo, float *grad_roughness) {
    return ray_render_adjoint_color(r, s, first_iteration, samples, sample_rgb, d_image, grad_albedo, grad_roughness, nullptr);
}

int ray_render_adjoint_color(ray_renderer *r, ray_scene *s, int first_iteration, int samples, const float *sample_rgb,
                             const float *d_image, float *grad_albedo, float *grad_roughness, float *grad_color) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    RG_CHECK(!s || live_scene(s), "unknown or destroyed scene handle");
    try {
        if (!r || !s || !sample_rgb || !d_image || !grad_roughness) {
            set_error("null argument");
            return RAY_ERR_INVALID_ARG;
        }
        if (!s->diff_rough) {
            set_error("the scene has no differentiable parameters (ray_scene_set_diff_params)");
            return RAY_ERR_INVALID_ARG;
        }
        if (s->diff_albedo && !grad_albedo) {
            set_error("the scene has an albedo texture: grad_albedo is required");
            return RAY_ERR_INVALID_ARG;
        }
        for (const MaterialRec &m : s->materials)
            if (m.type != (uint32_t)RAY_MAT_PRINCIPLED && m.type != (uint32_t)RAY_MAT_DIFFUSE && m.type != (uint32_t)RAY_MAT_EMISSIVE) {
                set_error("the adjoint takes scenes of RAY_MAT_PRINCIPLED, RAY_MAT_DIFFUSE and RAY_MAT_EMISSIVE materials only");
                return RAY_ERR_UNSUPPORTED;
            }
        std::vector<FrameJob> jobs;
        uint32_t n_pix = 0;
        int rc = diff_jobs(r, s, first_iteration, samples, jobs, n_pix);
        if (rc != RAY_OK) return rc;
        const uint32_t total = n_pix * (uint32_t)samples;
        for (int k = 0; k < 2; k++) RG_CUDA_TRY(r->d_adj[k].ensure(std::max<size_t>(total, 1) * sizeof(AdjState)));
        RG_CUDA_TRY(r->d_adj_shadow.ensure(std::max<size_t>(total, 1) * sizeof(AdjShadowRec)));
        AdjointRun adj;
        adj.args.sample_rgb = sample_rgb;
        adj.args.d_image = d_image;
        adj.args.grad_albedo = grad_albedo;
        adj.args.grad_rough = grad_roughness;
        adj.args.grad_color = grad_color;
        adj.args.inv_spp = 1.0f / (float)samples;
        adj.state[0] = static_cast<AdjState *>(r->d_adj[0].p);
        adj.state[1] = static_cast<AdjState *>(r->d_adj[1].p);
        adj.recs = static_cast<AdjShadowRec *>(r->d_adj_shadow.p);
        cudaStream_t st = r->stream;
        uint32_t *cnt = static_cast<uint32_t *>(r->d_counters.p);
        RG_CUDA_TRY(cudaMemsetAsync(cnt, 0, 16 * sizeof(uint32_t), st));
        int nb = 0;
        rc = run_wavefront(r, static_cast<const FrameJob *>(r->d_jobs.p), jobs, std::vector<const ray_scene *>(jobs.size(), s), total, 0, 0u, st,
                           nullptr, nb, false, &adj);
        if (rc != RAY_OK) return rc;
        RG_CUDA_TRY(note_use(s, st));
        return RAY_OK;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return RAY_ERR_OUT_OF_MEMORY;
    }
}

int ray_renderer_set_ray_sort(ray_renderer *r, int policy) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || policy < -1 || policy > (int)SORT_ALL) {
        set_error("ray sort policy must be RAY_SORT_AUTO (-1), 0 or a mask of bounces within RAY_SORT_ALL");
        return RAY_ERR_INVALID_ARG;
    }
    r->sort_policy = policy;
    return RAY_OK;
}

int ray_get_pixels(ray_renderer *r, const ray_pixel **out, int on_device) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || !out) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    int rc = ensure_frame_buffers(r, false);
    if (rc != RAY_OK) return rc;
    RG_CUDA_TRY(wait_stream_unlocked(r->stream));
    RG_CHECK(live_renderer(r), "renderer destroyed while the call waited for its GPU work");
    RG_CUDA_TRY(cudaSetDevice(r->device));
    rc = ensure_frame_buffers(r, false);
    if (rc != RAY_OK) return rc;
    RG_CUDA_TRY(wait_stream(r->stream)); // work another thread enqueued meanwhile
    if (on_device) {
        *out = static_cast<const ray_pixel *>(r->d_final.p);
        return RAY_OK;
    }
    const size_t n = (size_t)r->w * r->h;
    if (!r->pixels_on_host || r->host_pixels.size() != n) {
        r->host_pixels.resize(n);
        RG_CUDA_TRY(cudaMemcpy(r->host_pixels.data(), r->d_final.p, n * sizeof(ray_pixel), cudaMemcpyDeviceToHost));
        r->pixels_on_host = true;
    }
    *out = r->host_pixels.data();
    return RAY_OK;
}

int ray_get_sh_data(ray_renderer *r, const ray_shl1 **out) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || !out) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (!r->d_clean_sh.p) {
        *out = nullptr; // as the reference: no data until a camera asks for it
        return RAY_OK;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(wait_stream_unlocked(r->stream));
    RG_CHECK(live_renderer(r), "renderer destroyed while the call waited for its GPU work");
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(wait_stream(r->stream)); // work another thread enqueued meanwhile
    if (!r->d_clean_sh.p) {
        *out = nullptr;
        return RAY_OK;
    }
    const size_t n = (size_t)r->w * r->h;
    if (!r->sh_on_host || r->host_sh.size() != n) {
        r->host_sh.resize(n);
        RG_CUDA_TRY(cudaMemcpy(r->host_sh.data(), r->d_clean_sh.p, n * sizeof(ray_shl1), cudaMemcpyDeviceToHost));
        r->sh_on_host = true;
    }
    *out = r->host_sh.data();
    return RAY_OK;
}

int ray_renderer_debug_read(ray_renderer *r, int what, void *dst, uint64_t bytes, uint64_t *out_bytes) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || !out_bytes || (bytes && !dst) || what < 0 || what > 3) {
        set_error("invalid argument");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(wait_stream(r->stream));
    const DeviceBuf *b = what == 0 ? &r->d_rays[0] : (what == 1 ? &r->d_pay[0] : (what == 2 ? &r->d_halton : &r->d_temp));
    const uint64_t size = what == 2 ? (b->p ? HALTON_COUNT * HALTON_SEQ_LEN * sizeof(float) : 0) : b->bytes;
    *out_bytes = size;
    const uint64_t n = std::min<uint64_t>(bytes, size);
    if (n) RG_CUDA_TRY(cudaMemcpy(dst, b->p, n, cudaMemcpyDeviceToHost));
    return RAY_OK;
}

int ray_renderer_set_stream(ray_renderer *r, void *stream) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r) {
        set_error("null renderer");
        return RAY_ERR_INVALID_ARG;
    }
    cudaStream_t next = stream ? static_cast<cudaStream_t>(stream) : r->own_stream;
    if (next == r->stream) return RAY_OK;
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(wait_stream(r->stream)); // work on the old stream finishes first
    r->stream = next;
    return RAY_OK;
}

int ray_renderer_frame_info(ray_renderer *r, ray_frame_info *out) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || !out) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    *out = ray_frame_info{};
    if (!r->d_counters.p) return RAY_OK;
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(wait_stream(r->stream));
    uint32_t c[8];
    RG_CUDA_TRY(cudaMemcpy(c, r->d_counters.p, sizeof(c), cudaMemcpyDeviceToHost));
    out->error_flags = c[3];
    out->kernel = r->last_kernel;
    out->sort_mask = r->last_sort_mask;
    out->trace_variant = r->last_trace_var;
    const TraceVariant &tv = TRACE_VARIANTS[r->last_trace_var];
    out->trace_refill = tv.refill;
    out->trace_block = tv.block;
    out->trace_stack = tv.stack;
    out->trace_one_tri = (uint32_t)tv.one;
    memcpy(&out->rays, c + 4, 8);
    memcpy(&out->shadow_rays, c + 6, 8);
    return RAY_OK;
}

int ray_get_stats(ray_renderer *r, ray_stats *out) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r || !out) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (r->ev_sets[0][0]) {
        RG_CUDA_TRY(cudaSetDevice(r->device));
        for (int s = 0; s < 2; s++) {
            const int rc = resolve_stats(r, s);
            if (rc != RAY_OK) return rc;
        }
    }
    *out = r->stats;
    return RAY_OK;
}

int ray_reset_stats(ray_renderer *r) {
    RG_API_LOCK;
    RG_CHECK(!r || live_renderer(r), "unknown or destroyed renderer handle");
    if (!r) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (r->ev_sets[0][0]) {
        for (int s = 0; s < 2; s++) {
            const int rc = resolve_stats(r, s);
            if (rc != RAY_OK) return rc;
        }
    }
    r->stats = ray_stats{};
    return RAY_OK;
}

} // extern "C"
