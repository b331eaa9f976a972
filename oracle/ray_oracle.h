/*
 * CPU oracle for the wavefront path tracer: a plain-C restatement of the Ray
 * library's hot-path arithmetic (SerhiiY-94/RayDemo, src/Ray). It is test
 * infrastructure only: tests, the smoke check and the CPU-baseline leg of the
 * benchmark may call it as a checker; the product never links or runs it.
 *
 * Build with -ffp-contract=off: the reference results depend on products and
 * sums being rounded separately (no FMA contraction).
 */
#ifndef RAY_ORACLE_H
#define RAY_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same 48-byte layout as tri_accel_t (src/Ray/internal/Core.h:27-36). */
typedef struct orc_tri {
    float nu, nv, np, pu, pv;
    int32_t ci;
    float e0u, e0v, e1u, e1v;
    uint32_t mi, back_mi;
} orc_tri;

/* One closest hit: prim = -1 on a miss (t then holds the input tmax). */
typedef struct orc_hit {
    int32_t prim;
    float t, u, v;
} orc_hit;

/* Same field order as Ref::ray_packet_t (src/Ray/internal/CoreRef.h:34-45). */
typedef struct orc_ray_packet {
    float o[3], d[3], c[3], ior;
    float do_dx[3], dd_dx[3], do_dy[3], dd_dy[3];
    int32_t xy;
    int32_t ray_depth;
} orc_ray_packet;

typedef struct orc_camera {
    int filter; /* 0 Box, 1 Tent (Types.h eFilterType) */
    float fov, gamma, focus_distance, focus_factor;
    float origin[3], fwd[3], side[3], up[3];
} orc_camera;

/* PreprocessTri (src/Ray/internal/Core.cpp:162-214) for an indexed mesh.
 * pos: vertex positions with `stride` floats between vertices. Returns the
 * number of degenerate triangles (written as the reference's InvalidTriangle). */
int64_t orc_preprocess_tris(const float *pos, int64_t stride, const uint32_t *idx, int64_t ntris, orc_tri *out);

/* Closest hit over all triangles with _IntersectTri arithmetic
 * (src/Ray/internal/CoreRef.cpp:11-42). rays: 8 floats per ray
 * (ox, oy, oz, tmax, dx, dy, dz, unused). Ties on t keep the lowest index.
 * world_box (6 floats, min then max; may be NULL): the box of the single mesh
 * instance, tested first as the reference's macro traversal does
 * (bbox_test with safe_invert, CoreRef.cpp:64-86, 272-294, 1133-1222). */
void orc_closest_hit_brute(const orc_tri *tris, int64_t ntris, const float *rays, int64_t nrays, orc_hit *hits, int nthreads,
                           const float *world_box);

/* Same result through an oracle-owned binary BVH (conservative boxes, so the
 * result equals the brute-force one). aabbs: 6 floats per triangle. */
typedef struct orc_bvh orc_bvh;
orc_bvh *orc_bvh_build(const float *aabbs, int64_t ntris);
void orc_bvh_free(orc_bvh *b);
void orc_closest_hit_bvh(const orc_bvh *b, const orc_tri *tris, const float *rays, int64_t nrays, orc_hit *hits, int nthreads,
                         const float *world_box);

/* get_ray_hash (src/Ray/internal/CoreRef.cpp:316-333) for rays given as
 * 8 floats (o, tmax, d, unused). */
void orc_ray_hash(const float *rays, int64_t nrays, const float root_min[3], const float cell_size[3], uint32_t *keys);
/* The permutation SortRays_CPU (CoreRef.cpp:615-657) applies: a stable sort
 * by 32-bit key. perm[i] = source index of the ray that lands at position i. */
void orc_sort_perm(const uint32_t *keys, int64_t n, uint32_t *perm);

/* ConstructCamera, perspective case (src/Ray/internal/Core.cpp:856-886). */
void orc_construct_camera(int filter, const float origin[3], const float fwd[3], const float up[3], float fov, float gamma,
                          float focus_distance, float focus_factor, orc_camera *cam);
/* GeneratePrimaryRays (src/Ray/internal/CoreRef.cpp:427-505). */
void orc_generate_primary_rays(const orc_camera *cam, int iteration, int rx, int ry, int rw, int rh, int w, int h,
                               const float *halton, orc_ray_packet *out);

/* Halton permutations (src/Ray/internal/Halton.h:7-43 with the generator of
 * RendererRef.cpp:10-13) and the 24 x 256 sample table
 * (RendererRef.cpp:327-358). perms: 1,002 entries. */
void orc_halton_perms(uint16_t *perms);
void orc_halton_table(int iteration, const uint16_t *perms, float *out);

/* Integer hash and [0,1) float construction used for per-pixel scrambling
 * (CoreRef.cpp:264-270, 359-368). */
int32_t orc_hash(int32_t x);
float orc_construct_float(uint32_t m);

/* ---- the metallic-roughness material (RAY_MAT_PRINCIPLED of the library's
 * C ABI; no counterpart in the reference): a CPU path tracer restating the
 * GPU renderer's frames for scenes of such materials lit by quad and sun
 * lights and the default (white) environment map times env_col. Meshes are
 * given in object space and placed by instances, intersected as the
 * reference's macro traversal does (instance box test, TransformRay), so the
 * hits are the GPU's bit for bit.
 *   tris       ntris records (orc_preprocess_tris of each mesh's positions),
 *              mesh after mesh
 *   aabbs      6 floats per triangle (for the oracle BVH of each mesh)
 *   normals    9 floats per triangle: the vertex normals
 *   uvs        6 floats per triangle
 *   mat        per triangle: front material index, back material index
 *              (-1: a back face is black)
 *   mesh_tris  2 per mesh: first triangle, triangle count
 *   inst_mesh  per instance: its mesh; inst_xform: 16 floats, column-major
 *   mats       8 floats per material: base rgb, roughness, metallic, texture
 *              index (-1: white), differentiable slot (-1: none), unused
 *   diff_*     the differentiable parameters (may be NULL): a float RGB
 *              albedo (diff_ah x diff_aw x 3) and roughness slots; a material
 *              with a slot takes base = rgb x albedo(uv), roughness = slot's;
 *              diff_rough_sampling (may be NULL): frozen roughness for
 *              sampling, pdfs and MIS weights
 *   texels     RGBA8 of every texture, one after another
 *   tex_info   4 ints per texture: texel offset, w, h, sRGB
 *   lights     20 floats per light, from orc_area_light
 * Renders `spp` iterations (1 .. spp) of the full w x h frame and returns the
 * accumulated mean in out (w * h * 4): the renderer's clean buffer
 * (clean += (sample - clean) / iteration), or with plain_mean the
 * differentiable forward pass's (sum of the samples) * (1 / spp). */
typedef struct orc_principled_scene {
    const orc_tri *tris;
    const float *aabbs, *normals, *uvs;
    const int32_t *mat;
    const int64_t *mesh_tris;
    const int32_t *inst_mesh;
    const float *inst_xform;
    const float *mats;
    const uint32_t *texels;
    const int32_t *tex_info;
    const float *lights;
    const float *diff_albedo, *diff_rough, *diff_rough_sampling;
    int64_t ntris;
    int nmeshes, ninst, nmats, ntex, nlights;
    int diff_aw, diff_ah, n_diff_rough;
    float env_col[3];
} orc_principled_scene;
void orc_render_principled(const orc_principled_scene *sc, const orc_camera *cam, int w, int h, int spp, int max_diff_depth,
                           int max_total_depth, int termination_start_depth, float *out, int nthreads, int plain_mean);
/* The 20-float light record of a quad (type 3: position, edge_u, edge_v,
 * radiance) or sun (type 4: direction, full cone angle in degrees,
 * irradiance) light. Returns 0, or -1 for an invalid light. */
int orc_area_light(int type, const float position[3], const float color[3], const float direction[3], float angle,
                   const float edge_u[3], const float edge_v[3], float out[20]);

#ifdef __cplusplus
}
#endif
#endif
