// Closest-hit traversal entry points (device side of the batch trace and of
// the render loop).
#pragma once

#include "common.cuh"

namespace rg {

struct SceneView {
    const WideNode *nodes;
    const TriRec *leaf_tris;
    const InstanceRec *inst;
    uint32_t n_inst;
    // the instance tree (n_inst - 1 nodes), or null: the traversal then tests
    // the instances' boxes one after another
    const TlasNode *tlas = nullptr;
};

// Instance counts from which traces walk the instance tree instead of
// testing every instance box in turn.
constexpr uint32_t TLAS_MIN_INSTANCES = 32;

// Error bits written (OR-ed) to *err by the traversal.
constexpr uint32_t TRACE_ERR_STACK = 1u;
constexpr uint32_t TRACE_ERR_BOUNDS = 2u; // a node or triangle index outside the mesh's arrays
constexpr uint32_t TRACE_ERR_LIMIT = 4u;  // more node visits than the mesh has nodes
// (8 is the radix sort's look-back bound, SORT_ERR_LOOKBACK)
constexpr uint32_t TRACE_ERR_TLAS = 16u;  // the instance tree's stack overflowed or an index was out of bounds

// Kernel choice and its knobs (picked by the tuner).
struct TraceParams {
    bool persistent = true; // resident grid with per-lane ray refill
    // persistent grid: one triangle test per lane and loop iteration (the next
    // node once the last one's triangles are done), else a node's triangles at
    // once; counting launches always take the latter
    bool one_tri = false;
    int refill_min = 8;     // refill a warp's idle lanes once at least this many are idle
    // closest-hit persistent kernel only: threads per block (64, 128, 256) and
    // shared-memory stack entries per thread (16, 24, 32; 256 x 32 exceeds the
    // block's static shared memory)
    int block = 128, smem_stack = 24;
    // closest-hit persistent kernel: rays read and hits written with the
    // streaming (evict-first) cache hint
    int stream_hint = 0;
    uint32_t max_depth = 0; // deepest wide BVH among the traced meshes (sizes the stack)
    uint32_t *next_ray = nullptr; // device work counter for the persistent kernel
    const uint32_t *count = nullptr; // device ray count: when set, min(n, *count) rays are traced
    // rays of several scenes (persistent kernel only): ray i is traced in the
    // SceneView at views + ray_job[i] * view_stride, and the sv argument is unused
    const uint8_t *views = nullptr;
    uint32_t view_stride = 0;
    const uint32_t *ray_job = nullptr;
    // some scene of the launch has an instance tree: the kernels that walk it
    // (the others test the instance boxes in turn and carry no tree stack)
    bool tlas = false;
    // trace order: the k-th ray taken is ray order[k] (its hit is written at
    // that index); null: input order
    const uint32_t *order = nullptr;
    // shadow rays (persistent kernel): a ray ends at its first accepted hit on
    // a solid triangle (that hit is returned); without one, the closest hit
    // on a non-solid triangle or a miss
    bool any = false;
};

// rays: n x 8 floats (ox, oy, oz, tmax, dx, dy, dz, unused).
// hits: n x {prim, t, u, v}; obj may be null. counters (may be null when
// count == false): [0] node visits, [1] triangle tests.
cudaError_t launch_trace_closest(const SceneView &sv, const float4 *rays, uint32_t n, float4 *hits, int32_t *obj, uint32_t *err,
                                 unsigned long long *counters, bool count, cudaStream_t st, const TraceParams &tp);

} // namespace rg
