// Device-side data of the renderer (the Ref backend's render loop,
// src/Ray/internal/RendererRef.cpp:19-325) and its kernel launchers.
#pragma once

#include "../../include/raygpu.h"
#include "common.cuh"
#include "trace.cuh"

namespace rg {

// material_t (src/Ray/internal/Core.h:121-131): textures[] = normal map,
// main texture, and for mix materials the two mixed materials. The padding
// word holds the metallic parameter of RAY_MAT_PRINCIPLED.
struct MaterialRec {
    uint32_t textures[4];
    float main_color[3], metallic;
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

// vertex_t (src/Ray/internal/Core.h:219-222) padded to 64 bytes: four 16-byte loads.
struct alignas(16) VertexRec {
    float p[3], n[3], b[3], t[2][2];
    float pad[3];
};
static_assert(sizeof(VertexRec) == 64, "VertexRec must stay 64 bytes");

constexpr int NUM_MIP_LEVELS = 14;

// One mip level as stored on the device: a (w + 2) x (h + 2) block of RGBA8
// texels (with the wrap border) at texel offset `off`; (px, py) is where the
// reference's atlas places the level, which fixes the rounding of its
// sampling coordinates.
struct TexLevel {
    uint32_t off;
    uint16_t px, py;
    uint16_t pitch, rows;
};
static_assert(sizeof(TexLevel) == 12, "TexLevel must stay 12 bytes");

// texture_t (Core.h:103-108) as the device samples it. Levels past the last
// generated one repeat it, as in the reference (SceneRef.cpp:104-109).
struct TexDev {
    uint32_t width; // bit 15: sRGB
    uint32_t height;
    TexLevel lv[NUM_MIP_LEVELS];
};

// A quad or sun light of RAY_MAT_PRINCIPLED's next-event estimation (80 bytes).
// Quad: p0 + s u + t v, unit normal n = u x v / |u x v|, area, radiance L.
// Sun: n = unit direction towards the sun, cos_max = cosine of the cone's
// half angle, L = irradiance.
struct AreaLight {
    float p0[3];
    uint32_t type; // RAY_LIGHT_QUAD or RAY_LIGHT_SUN
    float u[3], area;
    float v[3], cos_max;
    float n[3], pad0;
    float L[3], pad1;
};
static_assert(sizeof(AreaLight) == 80, "AreaLight must stay 80 bytes");

// Everything a shading kernel reads of the scene.
struct RenderScene {
    SceneView sv;                  // BVH, leaf triangles and instances (shadow rays)
    const TriRec *tris;            // triangles in insertion order (materials, plane normal)
    const uint32_t *vtx_indices;   // 3 per triangle
    const VertexRec *vertices;
    const MaterialRec *materials;
    const TexDev *textures;
    const uint32_t *texels;
    const LightRec *lights;
    const AreaLight *area_lights;
    uint32_t n_tris, n_materials, n_textures, n_lights, n_area_lights;
    uint32_t principled_only; // every material is RAY_MAT_PRINCIPLED (host-side choice of the shading kernel)
    float env_col[3], env_clamp;
    uint32_t env_map;
    // differentiable parameters (ray_scene_set_diff_params): a float RGB
    // albedo texture (h x w x 3) and roughness slots; a RAY_MAT_PRINCIPLED
    // material whose textures[2] holds a slot takes its base colour from the
    // texture (times main_color) and its roughness from the slot
    const float *diff_albedo;
    const float *diff_rough;
    const float *diff_rough_sampling; // null: sampling and pdfs take diff_rough too
    uint32_t diff_aw, diff_ah, n_diff_rough;
    // a RAY_MAT_DIFFUSE material whose textures[2] holds a slot takes its
    // Oren-Nayar roughness from diff_rough and, when diff_color is set, its
    // main colour from diff_color (3 floats per slot)
    const float *diff_color;
};

// pass_settings_t flags (src/Ray/Types.h:39-45)
enum : uint32_t {
    PASS_SKIP_DIRECT = 1u << 0,
    PASS_SKIP_INDIRECT = 1u << 1,
    PASS_LIGHTING_ONLY = 1u << 2,
    PASS_NO_BACKGROUND = 1u << 3,
    PASS_CLAMP = 1u << 4,
    PASS_OUTPUT_SH = 1u << 5,
    PASS_COHERENT = 1u << 6,
};

// pass_info_t (Core.h:269-292) minus the per-ray index
struct PassInfo {
    int iteration, bounce;
    uint32_t flags;
    int max_diff_depth, max_glossy_depth, max_refr_depth, max_transp_depth, max_total_depth, termination_start_depth;
    int w; // framebuffer width (pixel index = y * w + x)
};

// camera_t (Types.h:59-71) fields ray generation needs
struct CameraDev {
    int filter; // 0 box, 1 tent
    float fov, focus_distance, focus_factor;
    float origin[3], fwd[3], side[3], up[3];
};

// A Geo (lightmap) camera, camera_t::mi_index / uv_index (Types.h:69): the
// instance's mesh sampled in its UV layer `uv` (SampleMeshInTextureSpace,
// CoreRef.cpp:507-603). xf: the instance transform's first three rows
// (TransformPoint's operand order), inv: its inverse's upper 3x3 in the
// layout transform_normal reads.
struct GeoCam {
    int on;
    uint32_t tri0, ntri; // the mesh's global triangle range
    uint32_t obj, uv;
    float xf[12], inv[9];
};

// Ray payload beside the 32-byte trace record (o, tmax | d, xy): the rest of
// ray_packet_t (CoreRef.h:34-45), 80 bytes.
struct alignas(16) RayPayload {
    float c[3], ior;
    float do_dx[3], dd_dx[3], do_dy[3], dd_dy[3];
    int32_t ray_depth;
    uint32_t pad[3];
};
static_assert(sizeof(RayPayload) == 80, "RayPayload must stay 80 bytes");

// shl1_data_t (Types.h:25-28)
struct SHData {
    float coeff_r[4], coeff_g[4], coeff_b[4];
};

constexpr int HALTON_COUNT = 24;
constexpr int HALTON_SEQ_LEN = 256;
// table entries plus a guard band: the reference's deepest bounce reads two
// entries past row 255 (RendererRef.cpp:327-358 with MAX_BOUNCES 10)
constexpr int HALTON_TABLE_FLOATS = HALTON_COUNT * HALTON_SEQ_LEN + 64;

// One (renderer, scene, region) of a frame, read by both kernels: the
// wavefront (a launch per phase over the rays of all jobs) and the path
// kernel (one thread follows one pixel's path through all its bounces). The
// jobs of a launch cover consecutive global pixel ranges from pixel_base.
struct FrameJob {
    RenderScene sc;
    PassInfo pi;       // bounce is set per bounce
    CameraDev cam;
    float k, fov_k;    // aspect ratio and tan(fov / 2) * focus distance
    int rx, ry, rw, rh, w, h;
    const float *halton;
    float4 *temp, *clean, *fin;
    SHData *temp_sh, *clean_sh; // null unless the camera outputs SH data
    float mix_k, gamma;
    int srgb, clamp;
    int bounces;       // continuation rays traced: max_total_depth, or 0 with skip_indirect_lighting
    int samples;       // consecutive iterations pi.iteration .. + samples - 1, one after another per pixel
    uint32_t pixel_base;
    float root_min[3], cell[3]; // the ray hash grid: the scene's box split into 255 cells per axis
    GeoCam geo;                 // geo.on: primary hits come from the UV-space sampling, not from rays
};

// A RAY_MAT_PRINCIPLED light sample waiting for its shadow ray (48 bytes):
// the segment o -> p2, the colour it adds to temp[index] of job `job` when
// unblocked, and the pixel's sampling index.
struct ShadowRec {
    float o[3], p2[3], c[3];
    uint32_t index, job, rand_index;
};
static_assert(sizeof(ShadowRec) == 48, "shadow record layout");

// Where a shading launch appends its light samples: the records (ShadowRec
// or AdjShadowRec), their shadow rays (o, tmax = segment length; d) for the
// any-hit trace, the rays' jobs, and the device count.
struct ShadowQueue {
    void *recs;
    float4 *rays;
    uint32_t *job;
    uint32_t *count;
};

// ---- the path-replay adjoint (differentiable parameters of RAY_MAT_PRINCIPLED)
constexpr int ADJ_MAX_SLOTS = 64; // roughness slots

// Per ray of the adjoint wavefront (48 bytes): the path's colour summed
// through its previous vertex (in the order the sample buffer sums it) and
// what the previous vertex's continuation contributes to the gradient:
// per channel d(f cos)/d(albedo) / (f cos) times main_color, and
// d(f cos)/d(roughness) / (f cos), at its texture coordinates and slot.
struct AdjState {
    float a[3];
    float u, v;
    uint32_t slot; // RAY_INVALID_INDEX: no differentiable previous vertex
    float ga[3], gr[3];
};
static_assert(sizeof(AdjState) == 48, "AdjState layout");

// A light sample of the adjoint wavefront (80 bytes): the segment, its colour
// (added to the continuation's sum when unblocked), its gradient factors
// (albedo per channel with d_image folded in, roughness) and where they go.
struct AdjShadowRec {
    float o[3], p2[3], nee[3], ga[3];
    float gr, u, v;
    uint32_t slot, cont, job, rand_index, index;
};
static_assert(sizeof(AdjShadowRec) == 80, "AdjShadowRec layout");

// The adjoint's inputs and outputs. Job k of the launch is sample k: its
// radiance per pixel at sample_rgb[(k * w * h + pixel) * 3]; d_image: dLoss /
// d(mean image) per pixel (RGB); gradients accumulate into grad_albedo
// (diff_ah x diff_aw x 3) and grad_rough (n_diff_rough).
struct AdjArgs {
    const float *sample_rgb, *d_image;
    float *grad_albedo, *grad_rough;
    float *grad_color; // RAY_MAT_DIFFUSE slots' main colours (3 per slot), may be null
    float inv_spp;
};
// AdjState::slot / AdjShadowRec::slot: a RAY_MAT_DIFFUSE vertex's slot
// carries this flag (its colour gradient goes to grad_color, not to texels).
constexpr uint32_t ADJ_DIFFUSE_SLOT = 0x40000000u;

// Launchers (render_kernels.cu). All stream-ordered; counts live on the device.
cudaError_t launch_halton_table(const uint16_t *perms, int base_iteration, float *table, cudaStream_t st);
// The wavefront over the jobs of a launch (rays of several scenes together).
// Ray generation: one ray per pixel of every job, ray_job[i] = job of ray i,
// *count = total. Iterations are pi.iteration + sample.
cudaError_t launch_raygen_jobs(const FrameJob *jobs, int n_jobs, uint32_t total, int sample, float4 *rays, RayPayload *pay,
                               uint32_t *ray_job, uint32_t *count, cudaStream_t st);
// Geo cameras: the smallest covering triangle per texel into best (all ones
// beforehand), then the texels' camera rays and hits into rays / pay / hits / obj.
cudaError_t launch_geo_cover(const FrameJob *jobs, int n_jobs, uint32_t max_tris, int sample, uint32_t *best, cudaStream_t st);
cudaError_t launch_geo_rays(const FrameJob *jobs, int n_jobs, uint32_t total, int sample, const uint32_t *best, float4 *rays, RayPayload *pay,
                            float4 *hits, int32_t *obj, cudaStream_t st);
// Shades the hits of *in_count rays (bounce: pass_info_t::bounce, 2 for the
// primary rays: SetPixel, else AddPixel with alpha 0), appends the rays that
// go on to out (count *out_count) and the light samples of RAY_MAT_PRINCIPLED
// vertices to shadow (count *shadow_count, zeroed beforehand). ref_lights:
// some job's scene has the reference's lights (traced inside the shading).
cudaError_t launch_shade_jobs(const FrameJob *jobs, int sample, int bounce, const float4 *rays, const RayPayload *pay, const uint32_t *ray_job,
                              const float4 *hits, const int32_t *obj, const uint32_t *in_count, uint32_t max_rays, float4 *out_rays,
                              RayPayload *out_pay, uint32_t *out_job, uint32_t *out_count, const ShadowQueue &shadow, bool ref_lights,
                              bool principled_only, uint32_t *err, unsigned long long *ray_stats, cudaStream_t st);
// After the any-hit trace of a shading launch's shadow rays (hits): adds the
// colour of each unblocked light sample to its pixel. A ray whose first hit
// is on a non-solid triangle takes the full visibility walk through the
// transparent layers (ComputeVisibility) instead.
cudaError_t launch_shadow_apply(const FrameJob *jobs, int sample, int bounce, const ShadowQueue &shadow, const float4 *hits, uint32_t max_recs,
                                uint32_t *err, unsigned long long *ray_stats, cudaStream_t st);
// clean += (temp - clean) / iteration over every job's rect, then final = tone(clean)
cudaError_t launch_resolve_jobs(const FrameJob *jobs, int n_jobs, uint32_t total, int sample, cudaStream_t st);
// The whole frame of every job in one launch (ray generation, all bounces,
// accumulation and tone): jobs in device memory, *work zeroed beforehand.
cudaError_t launch_render_paths(const FrameJob *jobs, int n_jobs, uint32_t total_pixels, uint32_t *work, uint32_t *err,
                                unsigned long long *ray_stats, cudaStream_t st);
// Ray sorting between bounces (sort.cu): the *count rays of a wavefront
// buffer in the order of a stable sort on (job, get_ray_hash of the ray in
// its job's grid), written to the other buffer with *count_out = *count.
// capacity: the buffers' size; only the min(*count, capacity) live rays are
// hashed, sorted and copied (the count is read on the device). err gets
// SORT_ERR_LOOKBACK if the sort's bounded wait ran out.
size_t loop_sort_scratch_bytes(uint64_t capacity, int n_jobs);
cudaError_t launch_loop_sort(const FrameJob *jobs, int n_jobs, const float4 *rays, const RayPayload *pay, const uint32_t *ray_job,
                             const uint32_t *count, uint32_t capacity, float4 *rays_out, RayPayload *pay_out, uint32_t *job_out,
                             uint32_t *count_out, void *scratch, cudaStream_t st, uint32_t *err);
// Differentiable forward: per pixel, image = (sum over the jobs k of temp_k) / n_jobs
// and sample_rgb[k] = temp_k (RGB); temp_k = jobs[k].temp, all w x h.
cudaError_t launch_diff_collect(const FrameJob *jobs, int n_jobs, uint32_t n_pix, float *image, float *sample_rgb, cudaStream_t st);
// The adjoint's shading (replays the forward shading of each ray and adds the
// gradient of its previous vertex's continuation) and its light samples.
cudaError_t launch_adjoint_shade(const FrameJob *jobs, int bounce, const float4 *rays, const RayPayload *pay, const uint32_t *ray_job,
                                 const AdjState *adj_in, const float4 *hits, const int32_t *obj, const uint32_t *in_count, uint32_t max_rays,
                                 float4 *out_rays, RayPayload *out_pay, uint32_t *out_job, AdjState *adj_out, uint32_t *out_count,
                                 const ShadowQueue &shadow, const AdjArgs &args, uint32_t *err, cudaStream_t st, bool ref_lights,
                                 bool principled_only);
cudaError_t launch_adjoint_shadow_apply(const FrameJob *jobs, int bounce, const ShadowQueue &shadow, const float4 *hits, uint32_t max_recs,
                                        AdjState *adj_cont, const AdjArgs &args, uint32_t *err, cudaStream_t st);
cudaError_t launch_fill(float4 *buf, size_t n, float4 v, cudaStream_t st);
cudaError_t launch_fill_sh(SHData *buf, size_t n, cudaStream_t st);

} // namespace rg
