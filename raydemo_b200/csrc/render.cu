// Render-loop entry points of the C ABI: RendererBase::RenderScene as a
// wavefront on one stream (ray generation, then per bounce a closest-hit
// trace and a shading kernel that appends the continuation rays), the
// framebuffer accessors, Resize/Clear and the stats.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <random>

#include "../../include/raygpu.h"
#include "scene.hpp"
#include "sort.cuh"

using namespace rg;

namespace {

constexpr int MAX_BOUNCES = 10; // Core.h:53
constexpr int N_EVENTS = ray_renderer::N_EVENTS; // 4 + 2 * MAX_BOUNCES + 1
static_assert(N_EVENTS == 5 + 2 * MAX_BOUNCES, "one event per phase");

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

int ensure_ray_buffers(ray_renderer *r, size_t n) {
    for (int k = 0; k < 2; k++) {
        RG_CUDA_TRY(r->d_rays[k].ensure(n * 2 * sizeof(float4)));
        RG_CUDA_TRY(r->d_pay[k].ensure(n * sizeof(RayPayload)));
    }
    RG_CUDA_TRY(r->d_hits.ensure(n * sizeof(float4)));
    RG_CUDA_TRY(r->d_obj.ensure(n * sizeof(int32_t)));
    RG_CUDA_TRY(r->d_counters.ensure(8 * sizeof(uint32_t)));
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
    }
    return RAY_OK;
}

// Adds the phase times of a finished frame to the stats (stats_t, RendererBase.h:93-100).
int resolve_stats(ray_renderer *r, int set) {
    if (!r->ev_frame_pending[set]) return RAY_OK;
    cudaEvent_t *e = r->ev_sets[set];
    const int nb = r->ev_bounces[set];
    RG_CUDA_TRY(cudaEventSynchronize(e[N_EVENTS - 1]));
    auto us = [&](int a, int b) -> unsigned long long {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e[a], e[b]);
        return (unsigned long long)(ms * 1000.0f);
    };
    r->stats.time_primary_ray_gen_us += us(0, 1);
    r->stats.time_primary_trace_us += us(1, 2);
    r->stats.time_primary_shade_us += us(2, 3);
    for (int b = 0; b < nb; b++) {
        r->stats.time_secondary_trace_us += us(3 + 2 * b, 4 + 2 * b);
        r->stats.time_secondary_shade_us += us(4 + 2 * b, 5 + 2 * b);
    }
    r->ev_frame_pending[set] = false;
    return RAY_OK;
}

} // namespace

ray_renderer::~ray_renderer() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (int s = 0; s < 2; s++)
        for (int e = 0; e < N_EVENTS; e++)
            if (ev_sets[s][e]) cudaEventDestroy(ev_sets[s][e]);
    if (own_stream) cudaStreamDestroy(own_stream);
}

extern "C" {

int ray_sort_rays(ray_renderer *r, const float *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                  uint32_t *perm_out, float *rays_out, void *stream) {
    if (!r || !root_min || !cell_size || (n && (!rays || !perm_out))) {
        set_error("ray_sort_rays: null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (n > 0xffffffffull) {
        set_error("ray_sort_rays: at most 2^32 - 1 rays per call");
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
    if (!r || w <= 0 || h <= 0 || w > 32768 || h > 32768) {
        set_error("invalid size");
        return RAY_ERR_INVALID_ARG;
    }
    if (w == r->w && h == r->h) return RAY_OK;
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(cudaStreamSynchronize(r->stream));
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
    if (!r || !s || !region) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (s->device != r->device) return RAY_OK; // a scene of another renderer: a no-op, as the reference's failed cast
    if (s->current_cam >= s->cameras.size() || !s->cameras[s->current_cam].alive) {
        set_error("the scene has no current camera");
        return RAY_ERR_INVALID_ARG;
    }
    const CameraRec &cam = s->cameras[s->current_cam];
    const ray_camera_desc &cd = cam.desc;
    if (cd.type != 0) {
        set_error("only perspective cameras are rendered");
        return RAY_ERR_UNSUPPORTED;
    }
    try {
        RG_CUDA_TRY(cudaSetDevice(r->device));
        int rc = commit(s);
        if (rc != RAY_OK) return rc;
        const int w = r->w, h = r->h;
        ray_rect rect = region->rect;
        if (rect.w == 0 || rect.h == 0) rect = ray_rect{0, 0, w, h};
        if (rect.x < 0 || rect.y < 0 || rect.w < 0 || rect.h < 0 || rect.x + rect.w > w || rect.y + rect.h > h) {
            set_error("region outside the framebuffer");
            return RAY_ERR_INVALID_ARG;
        }
        const bool sh = cd.output_sh != 0;
        rc = ensure_frame_buffers(r, sh);
        if (rc != RAY_OK) return rc;
        const size_t n_pix = (size_t)rect.w * rect.h;
        rc = ensure_ray_buffers(r, std::max<size_t>(n_pix, 1));
        if (rc != RAY_OK) return rc;
        cudaStream_t st = r->stream;

        // stats of the frame two calls back are complete by now or soon
        const int set = (int)(r->frame & 1);
        rc = resolve_stats(r, set);
        if (rc != RAY_OK) return rc;
        cudaEvent_t *ev = r->ev_sets[set];

        // RegionContext: iteration++, and the sample table regenerated every
        // 256 iterations (RendererRef.cpp:85-89). For a region that starts at
        // iteration 0 the table's base is 1 until iteration 255, then the
        // iteration rounded down to a multiple of 256.
        region->iteration++;
        const int it = region->iteration;
        const int base = it < HALTON_SEQ_LEN ? 1 : (it & ~(HALTON_SEQ_LEN - 1));
        RG_CUDA_TRY(cudaEventRecord(ev[0], st));
        if (base != r->halton_base) {
            RG_CUDA_TRY(launch_halton_table(static_cast<const uint16_t *>(r->d_perms.p), base, static_cast<float *>(r->d_halton.p), st));
            r->halton_base = base;
        }
        const float *halton = static_cast<const float *>(r->d_halton.p);

        PassInfo pi{};
        pi.iteration = it;
        pi.bounce = 2;
        pi.flags = (cd.lighting_only ? PASS_LIGHTING_ONLY : 0u) | (cd.skip_direct_lighting ? PASS_SKIP_DIRECT : 0u) |
                   (cd.skip_indirect_lighting ? PASS_SKIP_INDIRECT : 0u) | (cd.no_background ? PASS_NO_BACKGROUND : 0u) |
                   (cd.clamp ? PASS_CLAMP : 0u) | (cd.output_sh ? PASS_OUTPUT_SH : 0u) |
                   (cd.use_coherent_sampling ? PASS_COHERENT : 0u);
        // pass_settings_t holds uint8 depths (Types.h:47-55)
        pi.max_diff_depth = (uint8_t)cd.max_diff_depth;
        pi.max_glossy_depth = (uint8_t)cd.max_glossy_depth;
        pi.max_refr_depth = (uint8_t)cd.max_refr_depth;
        pi.max_transp_depth = (uint8_t)cd.max_transp_depth;
        pi.max_total_depth = std::min((int)(uint8_t)cd.max_total_depth, MAX_BOUNCES);
        pi.termination_start_depth = (uint8_t)cd.termination_start_depth;
        pi.w = w;

        // primary rays (GeneratePrimaryRays, CoreRef.cpp:427-505); the camera
        // constants are computed here as on the CPU
        CameraDev cdev{};
        cdev.filter = cd.filter;
        cdev.fov = cd.fov;
        cdev.focus_distance = cd.focus_distance;
        cdev.focus_factor = cd.focus_factor;
        for (int k = 0; k < 3; k++) {
            cdev.origin[k] = cam.origin[k];
            cdev.fwd[k] = cam.fwd[k];
            cdev.side[k] = cam.side[k];
            cdev.up[k] = cam.up[k];
        }
        const float PI = 3.141592653589793238463f;
        const float kx = float(w) / h;
        const float fov_k = std::tan(0.5f * cd.fov * PI / 180.0f) * cd.focus_distance;
        uint32_t *cnt = static_cast<uint32_t *>(r->d_counters.p);
        // [0], [1] ray counts of the two buffers, [2] trace work counter,
        // [3] error flags, [4..7] two uint64: rays traced, shadow segments
        RG_CUDA_TRY(cudaMemsetAsync(cnt, 0, 8 * sizeof(uint32_t), st));
        unsigned long long *ray_stats = reinterpret_cast<unsigned long long *>(cnt + 4);
        float4 *rays[2] = {static_cast<float4 *>(r->d_rays[0].p), static_cast<float4 *>(r->d_rays[1].p)};
        RayPayload *pay[2] = {static_cast<RayPayload *>(r->d_pay[0].p), static_cast<RayPayload *>(r->d_pay[1].p)};
        RG_CUDA_TRY(launch_raygen(cdev, kx, fov_k, it, rect.x, rect.y, rect.w, rect.h, w, h, halton, rays[0], pay[0], cnt + 0, st));
        RG_CUDA_TRY(cudaEventRecord(ev[1], st));

        const RenderScene sc = render_scene_view(s);
        TraceParams tp;
        tp.persistent = s->tuning.kernel == 2;
        tp.refill_min = s->tuning.refill_min;
        tp.max_depth = s->tuning.deep_stack ? 0xffffffffu : s->max_depth;
        tp.next_ray = cnt + 2;
        float4 *hits = static_cast<float4 *>(r->d_hits.p);
        int32_t *obj = static_cast<int32_t *>(r->d_obj.p);
        uint32_t *err = cnt + 3;
        const uint32_t max_rays = (uint32_t)n_pix;

        tp.count = cnt + 0;
        RG_CUDA_TRY(launch_trace_closest(sc.sv, rays[0], max_rays, hits, obj, err, nullptr, false, st, tp));
        RG_CUDA_TRY(cudaEventRecord(ev[2], st));
        RG_CUDA_TRY(launch_shade(sc, pi, halton, rays[0], pay[0], hits, obj, cnt + 0, max_rays, rays[1], pay[1], cnt + 1,
                                 static_cast<float4 *>(r->d_temp.p), sh ? static_cast<SHData *>(r->d_temp_sh.p) : nullptr, true, err,
                                 ray_stats, st));
        RG_CUDA_TRY(cudaEventRecord(ev[3], st));

        // bounces (RendererRef.cpp:183-278); ray counts stay on the device
        int nb = 0;
        if (!(pi.flags & PASS_SKIP_INDIRECT)) {
            int cur = 1;
            for (int bounce = 0; bounce < pi.max_total_depth; bounce++) {
                const int nxt = cur ^ 1;
                RG_CUDA_TRY(cudaMemsetAsync(cnt + nxt, 0, sizeof(uint32_t), st));
                tp.count = cnt + cur;
                RG_CUDA_TRY(launch_trace_closest(sc.sv, rays[cur], max_rays, hits, obj, err, nullptr, false, st, tp));
                RG_CUDA_TRY(cudaEventRecord(ev[4 + 2 * bounce], st));
                pi.bounce = bounce + 3;
                RG_CUDA_TRY(launch_shade(sc, pi, halton, rays[cur], pay[cur], hits, obj, cnt + cur, max_rays, rays[nxt], pay[nxt],
                                         cnt + nxt, static_cast<float4 *>(r->d_temp.p), nullptr, false, err, ray_stats, st));
                RG_CUDA_TRY(cudaEventRecord(ev[5 + 2 * bounce], st));
                cur = nxt;
                nb++;
            }
        }

        // accumulate and tone (RendererRef.cpp:292-324)
        const float mix_factor = 1.0f / it;
        RG_CUDA_TRY(launch_resolve(static_cast<const float4 *>(r->d_temp.p), static_cast<float4 *>(r->d_clean.p),
                                   static_cast<float4 *>(r->d_final.p), sh ? static_cast<SHData *>(r->d_temp_sh.p) : nullptr,
                                   sh ? static_cast<SHData *>(r->d_clean_sh.p) : nullptr, rect.x, rect.y, rect.w, rect.h, w, mix_factor,
                                   cd.dtype == 1 ? 1 : 0, cd.gamma, cd.clamp != 0, sh, st));
        RG_CUDA_TRY(cudaEventRecord(ev[N_EVENTS - 1], st));
        r->ev_bounces[set] = nb;
        r->ev_frame_pending[set] = true;
        r->frame++;
        r->pixels_on_host = r->sh_on_host = false;
        return RAY_OK;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return RAY_ERR_OUT_OF_MEMORY;
    }
}

int ray_get_pixels(ray_renderer *r, const ray_pixel **out, int on_device) {
    if (!r || !out) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    int rc = ensure_frame_buffers(r, false);
    if (rc != RAY_OK) return rc;
    RG_CUDA_TRY(cudaStreamSynchronize(r->stream));
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
    if (!r || !out) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    if (!r->d_clean_sh.p) {
        *out = nullptr; // as the reference: no data until a camera asks for it
        return RAY_OK;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(cudaStreamSynchronize(r->stream));
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
    if (!r || !out_bytes || (bytes && !dst) || what < 0 || what > 3) {
        set_error("invalid argument");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(cudaStreamSynchronize(r->stream));
    const DeviceBuf *b = what == 0 ? &r->d_rays[0] : (what == 1 ? &r->d_pay[0] : (what == 2 ? &r->d_halton : &r->d_temp));
    const uint64_t size = what == 2 ? (b->p ? HALTON_COUNT * HALTON_SEQ_LEN * sizeof(float) : 0) : b->bytes;
    *out_bytes = size;
    const uint64_t n = std::min<uint64_t>(bytes, size);
    if (n) RG_CUDA_TRY(cudaMemcpy(dst, b->p, n, cudaMemcpyDeviceToHost));
    return RAY_OK;
}

int ray_renderer_set_stream(ray_renderer *r, void *stream) {
    if (!r) {
        set_error("null renderer");
        return RAY_ERR_INVALID_ARG;
    }
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(cudaStreamSynchronize(r->stream)); // work on the old stream finishes first
    r->stream = stream ? static_cast<cudaStream_t>(stream) : r->own_stream;
    return RAY_OK;
}

int ray_renderer_frame_info(ray_renderer *r, ray_frame_info *out) {
    if (!r || !out) {
        set_error("null argument");
        return RAY_ERR_INVALID_ARG;
    }
    *out = ray_frame_info{};
    if (!r->d_counters.p) return RAY_OK;
    RG_CUDA_TRY(cudaSetDevice(r->device));
    RG_CUDA_TRY(cudaStreamSynchronize(r->stream));
    uint32_t c[8];
    RG_CUDA_TRY(cudaMemcpy(c, r->d_counters.p, sizeof(c), cudaMemcpyDeviceToHost));
    out->error_flags = c[3];
    memcpy(&out->rays, c + 4, 8);
    memcpy(&out->shadow_rays, c + 6, 8);
    return RAY_OK;
}

int ray_get_stats(ray_renderer *r, ray_stats *out) {
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
