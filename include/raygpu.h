/*
 * raygpu -- C ABI of the B200 wavefront path tracer.
 *
 * A drop-in for the renderer/scene interface of the Ray library embedded in
 * SerhiiY-94/RayDemo (src/Ray). Every entry point returns an int status
 * (RAY_OK or a negative RAY_ERR_* code); ray_last_error() gives a message for
 * the calling thread. Descriptors are borrowed for the call only: all data is
 * copied, as the reference does (src/Ray/SceneBase.h).
 *
 * Struct layouts: plain C PODs. The 16-byte ray_pixel matches pixel_color_t
 * (src/Ray/Types.h:14-18); the descriptor structs carry the fields of the
 * reference descriptors in the same order, with C types (ints for bools and
 * enums, uint64_t for size_t).
 */
#ifndef RAYGPU_H
#define RAYGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RAY_OK 0
#define RAY_ERR_INVALID_ARG (-1)
#define RAY_ERR_CUDA (-2)
#define RAY_ERR_OUT_OF_MEMORY (-3)
#define RAY_ERR_NOT_FOUND (-4)
#define RAY_ERR_STACK_OVERFLOW (-5)
#define RAY_ERR_TIMEOUT (-6)
#define RAY_ERR_UNSUPPORTED (-7)

#define RAY_INVALID_INDEX 0xffffffffu

/* Memory space of the buffers handed to the batch entry points. */
#define RAY_MEM_HOST 0
#define RAY_MEM_DEVICE 1

typedef struct ray_renderer ray_renderer;
typedef struct ray_scene ray_scene;

/* Ray::eRendererType (RendererBase.h:15-22); this library reports its own bit. */
#define RAY_RENDERER_CUDA_SM100 (1 << 6)

/* settings_t (RendererBase.h:25-31); device selects the CUDA device. */
typedef struct ray_settings {
    int w, h;
    int use_wide_bvh; /* accepted for compatibility; the GPU always builds its own wide BVH */
    int device;
} ray_settings;

typedef struct ray_rect { int x, y, w, h; } ray_rect;     /* rect_t, Types.h:31 */
typedef struct ray_pixel { float r, g, b, a; } ray_pixel; /* pixel_color_t, Types.h:14-18 */
typedef struct ray_shl1 { float coeff_r[4], coeff_g[4], coeff_b[4]; } ray_shl1; /* shl1_data_t, Types.h:25-28 */

/* RegionContext (RendererBase.h:35-51): the caller owns it; ray_render
 * increments `iteration` and regenerates the sample table itself. */
typedef struct ray_region {
    ray_rect rect; /* w == 0 or h == 0: whole image */
    int iteration;
} ray_region;

/* stats_t (RendererBase.h:93-100), microseconds, cumulative. */
typedef struct ray_stats {
    unsigned long long time_primary_ray_gen_us, time_primary_trace_us, time_primary_shade_us;
    unsigned long long time_secondary_sort_us, time_secondary_trace_us, time_secondary_shade_us;
} ray_stats;

/* eMaterialType (SceneBase.h:45-52) */
enum { RAY_MAT_DIFFUSE = 0, RAY_MAT_GLOSSY, RAY_MAT_REFRACTIVE, RAY_MAT_EMISSIVE, RAY_MAT_MIX, RAY_MAT_TRANSPARENT };
/* Extension with no counterpart in the reference: a metallic-roughness
 * material (Lambert diffuse + GGX microfacet specular, Smith height-correlated
 * shadowing, Schlick Fresnel with F0 = 0.04 for the dielectric part). Base
 * colour = main_color x main_texture (bilinear, level 0; RAY_INVALID_INDEX:
 * white; the normal map is not used), roughness (alpha =
 * roughness^2), metallic in ray_mat_desc::metallic. It takes direct light by
 * next-event estimation from RAY_LIGHT_QUAD and RAY_LIGHT_SUN lights (quad
 * lights also by its sampled rays, combined by multiple importance sampling),
 * and indirect light from emissive surfaces and the environment; the
 * reference's point, spot and directional lights light only the reference's
 * materials. Its random numbers come from a padded 2D Sobol sequence with
 * hash-based Owen scrambling per pixel (the reference's materials keep the
 * reference's Halton table). */
#define RAY_MAT_PRINCIPLED 6
/* eVertexLayout (SceneBase.h:27-32) */
enum { RAY_LAYOUT_PNT = 0, RAY_LAYOUT_PNTT, RAY_LAYOUT_PNBT, RAY_LAYOUT_PNBTT };
/* eCamType (Types.h:34). GEO: a lightmap camera -- the framebuffer is the
 * UV layer uv_index of instance mi_index's mesh, each texel's surface point
 * shaded as a camera-ray hit (RendererRef.cpp:142-149). ORTHO is not rendered
 * (RAY_ERR_UNSUPPORTED): the reference constructs no orthographic camera
 * (Core.cpp:883-885). */
enum { RAY_CAM_PERSP = 0, RAY_CAM_ORTHO, RAY_CAM_GEO };
/* eLightType (SceneBase.h:108-112) */
enum { RAY_LIGHT_POINT = 0, RAY_LIGHT_SPOT, RAY_LIGHT_DIRECTIONAL };
/* Extensions with no counterpart in the reference, used by RAY_MAT_PRINCIPLED:
 * QUAD: a one-sided rectangle p = position + s * edge_u + t * edge_v
 * (s, t in [0, 1], edges perpendicular) emitting radiance `color` towards
 * edge_u x edge_v; not part of the geometry (rays pass through it). SUN: light
 * arriving from -direction within a cone of `angle` degrees (full angle),
 * irradiance `color` on a surface facing it. */
#define RAY_LIGHT_QUAD 3
#define RAY_LIGHT_SUN 4

/* mat_desc_t (SceneBase.h:55-67) */
typedef struct ray_mat_desc {
    int type;
    float main_color[3];
    uint32_t main_texture, normal_map, mix_materials[2];
    float roughness, strength, fresnel, int_ior, ext_ior;
    float metallic; /* RAY_MAT_PRINCIPLED only (not in the reference's mat_desc_t) */
} ray_mat_desc;

/* shape_desc_t (SceneBase.h:70-81) */
typedef struct ray_shape_desc {
    uint32_t mat_index, back_mat_index;
    uint64_t vtx_start, vtx_count;
} ray_shape_desc;

/* mesh_desc_t (SceneBase.h:84-95) */
typedef struct ray_mesh_desc {
    int prim_type; /* 0: indexed triangle list */
    int layout;
    const float *vtx_attrs;
    uint64_t vtx_attrs_count; /* number of vertices */
    const uint32_t *vtx_indices;
    uint64_t vtx_indices_count;
    int base_vertex;
    const ray_shape_desc *shapes;
    uint64_t shapes_count;
    int allow_spatial_splits, use_fast_bvh_build;
} ray_mesh_desc;

/* tex_desc_t (SceneBase.h:98-104); data: w*h RGBA8 pixels */
typedef struct ray_tex_desc {
    const uint8_t *data;
    int w, h;
    int is_srgb, generate_mipmaps;
} ray_tex_desc;

/* light_desc_t (SceneBase.h:114-119) */
typedef struct ray_light_desc {
    int type;
    float position[3], radius;
    float color[3];
    float direction[3], angle;
    float edge_u[3], edge_v[3]; /* RAY_LIGHT_QUAD only (not in the reference's light_desc_t) */
} ray_light_desc;

/* camera_desc_t (SceneBase.h:122-145) */
typedef struct ray_camera_desc {
    int type, filter, dtype; /* eCamType, eFilterType, eDeviceType (Types.h:33-37) */
    float origin[3], fwd[3], up[3];
    float fov, gamma, focus_distance, focus_factor;
    uint32_t mi_index, uv_index;
    int lighting_only, skip_direct_lighting, skip_indirect_lighting, no_background, clamp, output_sh, use_coherent_sampling;
    int max_diff_depth, max_glossy_depth, max_refr_depth, max_transp_depth, max_total_depth, termination_start_depth;
} ray_camera_desc;

/* environment_desc_t (SceneBase.h:148-152) */
typedef struct ray_environment_desc {
    float env_col[3];
    float env_clamp;
    uint32_t env_map;
} ray_environment_desc;

/* One closest hit. prim: global triangle index in scene insertion order
 * (the reference's tris_ index), -1 on a miss; t, u, v as computed by the
 * reference's intersection (CoreRef.cpp:11-42). */
typedef struct ray_hit {
    int32_t prim;
    float t, u, v;
} ray_hit;

const char *ray_last_error(void);
int ray_version(void);

/* ---- renderer (RendererBase.h:55-103, RendererFactory.h:19) */
/* Ray::CreateRenderer: the flags argument of the reference picks a CPU or
 * OpenCL backend; there is one backend here, so it takes none. */
int ray_create_renderer(const ray_settings *s, ray_renderer **out);
int ray_destroy_renderer(ray_renderer *r);
int ray_renderer_type(const ray_renderer *r, int *out_type);           /* RendererBase::type */
int ray_renderer_size(const ray_renderer *r, int *w, int *h);          /* RendererBase::size */
int ray_resize(ray_renderer *r, int w, int h);                        /* RendererBase::Resize */
int ray_clear(ray_renderer *r, const ray_pixel *c);                   /* RendererBase::Clear (NULL: black) */
int ray_create_scene(ray_renderer *r, ray_scene **out);               /* RendererBase::CreateScene */
int ray_destroy_scene(ray_scene *s);
/* RendererBase::RenderScene: one sample per pixel over region->rect. */
int ray_render(ray_renderer *r, ray_scene *s, ray_region *region);
/* RendererBase::get_pixels_ref: RGBA f32 row-major w*h; host pointer valid
 * until the next render/resize/clear (on_device != 0: device pointer). */
int ray_get_pixels(ray_renderer *r, const ray_pixel **out, int on_device);
int ray_get_sh_data(ray_renderer *r, const ray_shl1 **out); /* get_sh_data_ref */
int ray_get_stats(ray_renderer *r, ray_stats *out);          /* GetStats */
int ray_reset_stats(ray_renderer *r);                        /* ResetStats */

/* ---- scene (SceneBase.h:157-285) */
int ray_scene_get_environment(ray_scene *s, ray_environment_desc *out);
int ray_scene_set_environment(ray_scene *s, const ray_environment_desc *env);
int ray_scene_add_texture(ray_scene *s, const ray_tex_desc *t, uint32_t *out_index);
int ray_scene_remove_texture(ray_scene *s, uint32_t i);
int ray_scene_add_material(ray_scene *s, const ray_mat_desc *m, uint32_t *out_index);
int ray_scene_remove_material(ray_scene *s, uint32_t i);
int ray_scene_add_mesh(ray_scene *s, const ray_mesh_desc *m, uint32_t *out_index);
int ray_scene_remove_mesh(ray_scene *s, uint32_t i);
int ray_scene_add_light(ray_scene *s, const ray_light_desc *l, uint32_t *out_index);
int ray_scene_remove_light(ray_scene *s, uint32_t i);
int ray_scene_add_mesh_instance(ray_scene *s, uint32_t mesh_index, const float xform[16], uint32_t *out_index);
int ray_scene_set_mesh_instance_transform(ray_scene *s, uint32_t mi_index, const float xform[16]);
int ray_scene_remove_mesh_instance(ray_scene *s, uint32_t mi_index);
int ray_scene_add_camera(ray_scene *s, const ray_camera_desc *c, uint32_t *out_index);     /* SceneBase::AddCamera */
int ray_scene_get_camera(ray_scene *s, uint32_t i, ray_camera_desc *out);                 /* SceneBase::GetCamera */
int ray_scene_set_camera(ray_scene *s, uint32_t i, const ray_camera_desc *c);             /* SceneBase::SetCamera */
int ray_scene_remove_camera(ray_scene *s, uint32_t i);                                    /* SceneBase::RemoveCamera */
/* No counterpart in the reference: sets camera i's constructed side and up
 * axes (camera_t::side / up, Types.h:59-71) as given, in place of those
 * ray_scene_add_camera / ray_scene_set_camera construct. An adapter that holds
 * the reference's already constructed camera_t (SceneBase's camera store)
 * hands its axes on unchanged, so the primary rays stay bit-identical. */
int ray_scene_set_camera_axes(ray_scene *s, uint32_t i, const float side[3], const float up[3]);
int ray_scene_current_cam(ray_scene *s, uint32_t *out);
int ray_scene_set_current_cam(ray_scene *s, uint32_t i);
int ray_scene_triangle_count(ray_scene *s, uint32_t *out);
int ray_scene_node_count(ray_scene *s, uint32_t *out);
/* Uploads pending changes and builds the BVHs on the GPU (done implicitly by
 * ray_render and the trace entry points). */
int ray_scene_commit(ray_scene *s);

/* ---- batch closest hit: Traverse_MacroTree_WithStack_ClosestHit over a batch
 * (CoreRef.cpp:1133-1222). rays: n records of 8 floats
 * (ox, oy, oz, tmax, dx, dy, dz, unused); hits: n ray_hit; obj (optional, may be
 * NULL): n mesh-instance indices (-1 on a miss). mem: RAY_MEM_HOST or
 * RAY_MEM_DEVICE for all three buffers. stream: a cudaStream_t or NULL. */
int ray_scene_trace_closest(ray_scene *s, const float *rays, uint64_t n, ray_hit *hits, int32_t *obj, int mem, void *stream);

/* ---- ray sorting: SortRays_CPU (CoreRef.cpp:615-657) on device buffers.
 * rays: n records of 8 floats (as for ray_scene_trace_closest). root_min,
 * cell_size: the origin grid of get_ray_hash (CoreRef.cpp:316-333); the
 * reference renderer uses the scene's root box and (max - min) / 255
 * (RendererRef.cpp:48-77). keys_out (may be NULL): the hash of every input
 * ray, bit-exact; perm_out: perm_out[k] = input index of the ray that lands at
 * position k (a stable sort on the hash, the order SortRays_CPU produces);
 * rays_out (may be NULL): the rays in that order. Device memory only;
 * stream-ordered (stream: a cudaStream_t or NULL for the renderer's stream).
 * The sort's scratch memory belongs to the renderer. At most 2^30 - 1 rays. */
int ray_sort_rays(ray_renderer *r, const float *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                  uint32_t *perm_out, float *rays_out, void *stream);

/* Allocation-free variant of ray_sort_rays; it has no counterpart in the
 * reference. For callers that cannot call cudaMalloc: hosts whose GPU memory
 * belongs to their own allocator and budget, and frame loops that must not
 * stall on cudaMalloc's implicit device-wide synchronisation. Same inputs,
 * outputs and results as ray_sort_rays, without a renderer: the scratch
 * memory is a fixed array of 13,640,192 bytes (13.01 MiB) that every GPU
 * loading this library holds until the process exits, so n is limited to
 * RAY_SORT_NOALLOC_MAX_RAYS (larger n: RAY_ERR_INVALID_ARG). The first call on
 * a device looks the array up on the current device and keeps its address for
 * the life of the process: make that first call before any stream capture
 * begins, and do not reset the device (cudaDeviceReset) while the library is
 * in use. All calls share the array: calls that overlap on the GPU (other
 * streams, other host threads) race. Like every entry point, its host side
 * takes the library's process-wide lock. stream: a cudaStream_t, or NULL for
 * the default stream. */
#define RAY_SORT_NOALLOC_MAX_RAYS (1u << 20)
int ray_sort_rays_noalloc(const float *rays, uint64_t n, const float root_min[3], const float cell_size[3], uint32_t *keys_out,
                          uint32_t *perm_out, float *rays_out, void *stream);

/* Statistics of the last trace call on this scene: error flags OR-ed over rays
 * (bit 0: a ray's traversal stack overflowed), node and triangle visit totals
 * (counted only when counting was enabled with ray_scene_set_counting). */
typedef struct ray_trace_info {
    uint32_t error_flags;
    uint64_t node_visits, tri_tests;
} ray_trace_info;
int ray_scene_set_counting(ray_scene *s, int enable);
int ray_scene_last_trace_info(ray_scene *s, ray_trace_info *out);

/* Traversal kernel choice for this scene (no counterpart in the reference,
 * which has one CPU loop): kernel 1 = one thread per ray, 2 = resident grid
 * whose lanes take new rays as theirs finish (refill once at least
 * refill_min lanes of a warp are idle, 1..32) and test the triangles of a
 * node step at once, 3 (the default, with refill_min 8) = the same grid
 * testing one triangle per lane and step (a lane takes its next node once the
 * last one's triangles are done), the warp meeting again after each phase.
 * kernel 0 or refill_min <= 0 keep the current setting. deep_stack: 0 = size the traversal stack by the
 * BVH depth (shared memory only unless a tree is deeper than it holds),
 * 1 = always continue it in local memory. reorder: 0 = trace the rays in
 * their input order; 1 = first sort them (stably) by the reference's ray hash
 * (get_ray_hash, CoreRef.cpp:316-333: direction sector above the origin's
 * Morton cell, over the scene's box in 255 cells per axis, as SortRays_CPU
 * keys them) and trace them in that order; 2 = the same with the origin cell
 * above the direction sector. The hits are written at each ray's input
 * position either way, and do not depend on the order. reorder_bits: how many
 * of the key's top bits the sort uses (8..32; 0 = 32). Calls of fewer than
 * 65,536 rays are not reordered. block (64, 128, 256; 0 = 64) and smem_stack
 * (16, 24, 32 entries per thread; 0 = 16; not 32 with 256 threads): threads
 * per block of the persistent kernel and the depth of its shared-memory stack
 * (a deeper tree continues in local memory). stream_hint: 1 = the persistent
 * kernel reads rays and writes hits with the streaming (evict-first) cache
 * hint. l2_persist: 1 = the scene's wide nodes, 2 = its leaf triangles, are
 * marked persisting in L2 for the trace (an access-policy window on the
 * trace's streams, removed after it; the first such call sets this CUDA
 * context's persisting-L2 limit, which lasts as long as the context).
 * instance_tree: 0 = traces walk an instance tree (a BVH over the instances'
 * world boxes, built on the GPU at commit, refitted when only transforms
 * changed; the reference's macro tree, SceneRef.cpp:492-516) from 32
 * instances on and test the instance boxes in turn below that; 1 = the tree
 * from 2 instances on; -1 = never. */
typedef struct ray_trace_tuning {
    int kernel, refill_min, deep_stack, reorder, reorder_bits, block, smem_stack, stream_hint, l2_persist, instance_tree;
} ray_trace_tuning;
int ray_scene_set_trace_tuning(ray_scene *s, const ray_trace_tuning *t);
int ray_scene_get_trace_tuning(ray_scene *s, ray_trace_tuning *out);

/* BVH summary of one mesh (for tests and the roofline): node count, leaf
 * triangle records, maximum wide depth. */
typedef struct ray_bvh_info {
    uint32_t nodes, tris, depth, root;
    float bbox_min[3], bbox_max[3];
} ray_bvh_info;
int ray_scene_mesh_bvh_info(ray_scene *s, uint32_t mesh, ray_bvh_info *out);

/* The instance tree after the last commit: instances it covers (0: none,
 * the traversal tests the instance boxes in turn), host milliseconds the
 * last commit spent building or refitting it (device work included), and
 * whether that was a refit (1) or a build (0). */
typedef struct ray_instance_tree_info {
    uint32_t instances;
    int refit;
    double ms;
} ray_instance_tree_info;
int ray_scene_instance_tree_info(ray_scene *s, ray_instance_tree_info *out);

/* Diagnostics: copies one of the scene's device arrays to host memory (after
 * committing). what: 0 wide nodes (80 bytes each), 1 leaf-ordered triangles
 * (48 bytes each), 2 instance records (96 bytes each). Copies at most `bytes`
 * bytes; *out_bytes receives the array size. */
int ray_scene_debug_read(ray_scene *s, int what, void *dst, uint64_t bytes, uint64_t *out_bytes);

/* Failure detection (no counterpart in the reference, whose OpenCL backend
 * returns silently on any error, RendererOCL.cpp:474-632), for tests that make
 * failures happen on the host:
 * ray_scene_debug_write overwrites bytes of the committed wide nodes (what 0)
 * or leaf triangles (what 1) from host memory, as a corrupt structure would
 * hold them; the traversal bounds-checks every node and triangle index it
 * reads and bounds its steps, so a trace of such a scene ends every ray and
 * reports RAY_ERR_CUDA (corrupt structure) or RAY_ERR_STACK_OVERFLOW instead
 * of reading out of bounds. Scene edits that rebuild the BVH restore it.
 * ray_debug_fail_device_alloc: the after-th next device allocation the
 * library makes fails as a full device would (0: the next one; -1: none);
 * the failing call returns RAY_ERR_OUT_OF_MEMORY and keeps nothing it had
 * allocated for itself beyond what the handle owns (freed with the handle).
 * ray_set_wait_timeout_ms: the bound on every host wait of the library
 * (default 300,000 ms; <= 0 restores it): a wait that runs out returns
 * RAY_ERR_TIMEOUT without stopping the GPU work it waited for. */
int ray_scene_debug_write(ray_scene *s, int what, uint64_t offset, const void *src, uint64_t bytes);
int ray_debug_fail_device_alloc(int64_t after);
int ray_set_wait_timeout_ms(int64_t ms);

/* Trace tuner (no counterpart in the reference): times the traversal
 * settings of ray_trace_tuning on the caller's rays (n rays in device memory;
 * hits: an n-entry device buffer the candidates write) and keeps the fastest
 * for this scene: one setting at a time from the current ones (kernel, L2
 * residency, cache hint, refill threshold, block size with stack depth, trace
 * order), each candidate the best of two timed traces after one untimed.
 * Every candidate gives the same hits. The choice is cached per scene
 * signature (triangle, node and instance counts, BVH depth, ray count rounded
 * to a power of two); a later call with a cached signature applies it without
 * timing unless flags bit 0 is set. out (may be NULL): the choice. report (may
 * be NULL): "name=ms;..." of the candidates timed, NUL-terminated within
 * report_cap bytes. Synchronous. */
int ray_scene_tune_trace(ray_scene *s, const float *rays, uint64_t n, ray_hit *hits, int flags, void *stream, ray_trace_tuning *out,
                         char *report, uint64_t report_cap);

/* Diagnostics: copies one of the renderer's device arrays to host memory after
 * the last ray_render. what: 0 the first ray buffer (32 bytes per ray: ox, oy,
 * oz, tmax, dx, dy, dz, pixel as (x << 16) | y), 1 its payloads (80 bytes per
 * ray: c[3], ior, do_dx[3], dd_dx[3], do_dy[3], dd_dy[3], ray_depth, 3 unused),
 * 2 the sample table (6144 floats, RendererRef.cpp:327-358), 3 the frame's
 * sample buffer (16 bytes per pixel). The first ray buffer holds the primary
 * rays when the frame traced no bounce (skip_indirect_lighting). Copies at most
 * `bytes` bytes; *out_bytes receives the array size. */
int ray_renderer_debug_read(ray_renderer *r, int what, void *dst, uint64_t bytes, uint64_t *out_bytes);

/* Counts of the last ray_render (no counterpart in the reference): rays traced
 * for closest hits (primary and continuation rays), shadow-ray segments traced
 * (one per surface a light's visibility ray passes), and error flags OR-ed over
 * the frame's kernels (1 traversal stack overflow, 2 corrupt BVH index,
 * 4 traversal step limit, 8 a material/texture/instance index out of range,
 * 16 mix materials nested deeper than 32, 32 more than 256 transparent layers
 * on a shadow ray). Waits for the frame to finish. */
typedef struct ray_frame_info {
    uint32_t error_flags;
    int32_t kernel; /* the kernel that rendered it: 1 wavefront, 2 path kernel */
    uint64_t rays, shadow_rays;
    uint32_t sort_mask; /* wavefront: bounces whose rays were sorted first (bit b: secondary bounce b) */
    uint32_t trace_one_tri; /* wavefront: one triangle test per lane and step in its closest-hit traces (bit 0), shadow-ray traces (bit 1) */
    /* wavefront: the trace settings it ran with (ray_renderer_set_trace_variant):
     * their index, refill threshold, threads per block and shared stack entries
     * (0 for each of the three: the scene's own settings) */
    int32_t trace_variant, trace_refill, trace_block, trace_stack;
} ray_frame_info;
int ray_renderer_frame_info(ray_renderer *r, ray_frame_info *out);

/* The wavefront's trace settings (no counterpart in the reference): -1 (the
 * default) = the frame tuner times them with the kernel and the sort mask on
 * the first frames of each frame configuration -- index 0 is the scene's own
 * refill threshold, threads per block and shared stack entries with a node's
 * triangles tested at once, 1..3 are (8, 128, 24), (16, 128, 24), (8, 64, 24)
 * the same way, 4..5 are (4, 64, 16), (8, 128, 16) with one triangle test per
 * lane and step -- and keeps the fastest; the choice is also kept per frame
 * signature (triangle and light counts, pixels, bounces, settings) for every
 * renderer of the process; 0..5 = that setting. Every setting renders the
 * same image. */
int ray_renderer_set_trace_variant(ray_renderer *r, int variant);

/* Ray sorting in the wavefront (the reference's Ref renderer sorts the
 * continuation rays before every bounce by get_ray_hash, RendererRef.cpp:
 * 200-203; the image does not depend on it). policy: RAY_SORT_AUTO (the
 * default) sorts per bounce where timing the configuration's first frames
 * showed it faster (chosen together with the kernel), 0 never, else a mask of
 * the bounces to sort before (bit b: secondary bounce b; RAY_SORT_ALL every
 * bounce). The sort is stable on the key (job, hash): rays of one scene of a
 * batch stay together. */
#define RAY_SORT_AUTO (-1)
#define RAY_SORT_ALL 0x3FF
int ray_renderer_set_ray_sort(ray_renderer *r, int policy);

/* Kernel choice for ray_render (no counterpart in the reference, whose CPU
 * renderers have one loop): 1 = wavefront (a launch per bounce for ray
 * generation, closest hit and shading; ray counts on the device), 2 = path
 * kernel (one launch per frame, one thread per pixel through all bounces),
 * 0 = chosen per frame configuration (scene, rect size, bounces) by timing
 * both on its first frames. Both give the same image. Default 0. */
int ray_renderer_set_kernel(ray_renderer *r, int kernel);

/* Batched form (no counterpart in the reference): `samples` samples over each
 * region of `count` (renderer, scene, region) triples, as if ray_render were
 * called `samples` times for each in turn, with the scenes rendered together:
 * the path kernel renders every region's samples in one launch; the wavefront
 * runs each phase (ray generation, closest hit, shading, accumulation) as one
 * launch over the rays of all scenes. The first renderer's kernel setting
 * (ray_renderer_set_kernel) picks one; by default both are timed on the first
 * calls of a batch configuration and the faster is kept. A region's samples
 * are split where its iterations cross a multiple of 256 (its sample table
 * changes there). Renderers may repeat: regions of one framebuffer must not
 * overlap and must be at the same iteration. All renderers must be on one
 * device. The work goes on the first renderer's stream, ordered after the work
 * already on every renderer's stream and before the work enqueued there later;
 * the first renderer's ray_renderer_frame_info reports the last sample's
 * launches. Batched frames are not timed into the stats. */
int ray_render_batch(ray_renderer *const *renderers, ray_scene *const *scenes, ray_region *const *regions, int count, int samples);

/* ---- differentiable rendering (no counterpart in the reference).
 * Parameters of RAY_MAT_PRINCIPLED materials held in caller-owned device
 * memory: a float RGB albedo texture (albedo_h x albedo_w x 3, linear, read
 * bilinearly with wrap-around, texel centres at (i + 0.5) / w) and roughness
 * slots. material_slot (host, one entry per material of the scene, or NULL
 * for none) gives each material's slot, or -1: a material with a slot takes
 * its base colour from the texture (times main_color) and its roughness from
 * the slot. The arrays are read by every later render; NULL p detaches them.
 * At most 64 slots. roughness_sampling (device, n_roughness; may be NULL):
 * the roughness that direction sampling, pdfs and MIS weights take instead
 * of `roughness` -- frozen sampling, under which the rendered estimator is a
 * smooth function of the roughness and its derivative is exactly what the
 * adjoint computes (for checking it by finite differences).
 * The reference's RAY_MAT_DIFFUSE materials may have slots too: such a
 * material takes its Oren-Nayar roughness (sigma) from the slot and, when
 * color (device, n_roughness x 3; may be NULL) is given, its main colour from
 * color[3 * slot ..] (its main texture stays as it is). With no
 * RAY_MAT_PRINCIPLED material in a slot the albedo texture may be NULL. */
typedef struct ray_diff_params {
    const float *albedo;
    int albedo_w, albedo_h;
    const float *roughness;
    int n_roughness;
    const int32_t *material_slot;
    int n_materials;
    const float *roughness_sampling;
    const float *color;
} ray_diff_params;
int ray_scene_set_diff_params(ray_scene *s, const ray_diff_params *p);
/* Forward pass: samples iterations first_iteration .. first_iteration +
 * samples - 1 (from 1, within one block of 256) of the whole frame through
 * the current camera, without touching the renderer's accumulation.
 * image_rgb (device, h x w x 3) = mean of the samples; sample_rgb (device,
 * samples x h x w x 3) = each sample's radiance, which the adjoint needs. */
int ray_render_diff(ray_renderer *r, ray_scene *s, int first_iteration, int samples, float *image_rgb, float *sample_rgb);
/* Adjoint pass (path replay backpropagation): replays the paths of the
 * ray_render_diff call with the same first_iteration and samples and adds
 * dLoss/dalbedo to grad_albedo (device, albedo_h x albedo_w x 3) and
 * dLoss/droughness to grad_roughness (device, n_roughness), given d_image
 * (device, h x w x 3) = dLoss/dimage_rgb. Sampling is detached (pdfs and MIS
 * weights held constant). Scenes: RAY_MAT_PRINCIPLED, RAY_MAT_DIFFUSE and
 * RAY_MAT_EMISSIVE materials; quad and sun lights, and the reference's point,
 * spot and directional lights (their shadow rays traced again in the
 * adjoint); RAY_ERR_UNSUPPORTED otherwise. grad_albedo may be NULL when the
 * scene has no albedo texture. Russian roulette is not differentiated: give
 * the camera a termination depth at or past its bounce limit for exact
 * gradients. */
int ray_render_adjoint(ray_renderer *r, ray_scene *s, int first_iteration, int samples, const float *sample_rgb, const float *d_image,
                       float *grad_albedo, float *grad_roughness);
/* The same, also adding dLoss/d(main colour) of the RAY_MAT_DIFFUSE slots to
 * grad_color (device, n_roughness x 3; may be NULL) -- the colours that
 * ray_diff_params::color supplies. */
int ray_render_adjoint_color(ray_renderer *r, ray_scene *s, int first_iteration, int samples, const float *sample_rgb,
                             const float *d_image, float *grad_albedo, float *grad_roughness, float *grad_color);

/* The CUDA stream the renderer enqueues its work on from now on (a
 * cudaStream_t; NULL: the renderer's own stream). No counterpart in the
 * reference, whose renderers run on the calling thread. Waits for the work
 * already enqueued on the previous stream. */
int ray_renderer_set_stream(ray_renderer *r, void *stream);

#ifdef __cplusplus
}
#endif
#endif
