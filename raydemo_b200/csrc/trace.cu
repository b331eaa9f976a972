// Closest-hit traversal (compiled with --fmad=false).
//
// World level: for every mesh instance, the reference's instance box test
// (bbox_test with safe_invert, CoreRef.cpp:64-86, 272-294) and TransformRay
// (CoreRef.cpp:1605-1617), both reproduced operation for operation. Mesh
// level: the compressed 8-wide BVH, traversed with node groups (a base index
// plus a hit mask of up to 8 children) on a per-thread stack, children in
// octant order, which is roughly front to back; the triangles of the leaf
// children a node step hits (up to 24) are tested at once. Triangles use the
// reference's intersection arithmetic (CoreRef.cpp:11-42) with every product
// and sum rounded on its own, so t, u, v are bit-exact; a tie on t goes to the
// lower triangle index, which makes the result independent of visiting order.
//
// The kernels share the traversal step:
//   k_trace_closest      one thread per ray (a grid over the rays)
//   k_trace_persistent   a resident grid; a lane whose ray is done takes the
//                        next one from a global counter (warp-aggregated), so
//                        more lanes do useful work per instruction on
//                        incoherent rays of very different lengths
//   k_trace_closest_one  its closest-hit, one-triangle-per-step form for
//                        scenes without an instance tree, register-bounded
// The stack holds one node group per tree level at most. It lives in shared
// memory; meshes deeper than that use the DEEP instances, which continue it
// in a local array.
#include "trace.cuh"
#include "traverse.cuh"

namespace rg {
namespace {

using namespace trav;


template <bool COUNT>
__device__ __forceinline__ void flush_counters(uint32_t err, uint32_t nvis, uint32_t ntri, uint32_t *err_out, unsigned long long *counters) {
    if (err) atomicOr(err_out, err);
    if (COUNT) {
        unsigned long long a = nvis, b = ntri;
        for (int off = 16; off; off >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, off);
            b += __shfl_xor_sync(0xffffffffu, b, off);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&counters[0], a);
            atomicAdd(&counters[1], b);
        }
    }
}

template <bool COUNT, bool DEEP, bool TLAS = false>
__global__ void __launch_bounds__(TRACE_BLOCK) k_trace_closest(SceneView sv, const float4 *__restrict__ rays, uint32_t n, float4 *__restrict__ hits,
                                                               int32_t *__restrict__ obj_out, uint32_t *__restrict__ err_out,
                                                               unsigned long long *__restrict__ counters, const uint32_t *__restrict__ n_dev,
                                                               const uint32_t *__restrict__ order) {
    __shared__ uint2 s_stack[SMEM_STACK * TRACE_BLOCK];
    Stack<DEEP> st;
    st.smem = s_stack + threadIdx.x;
    st.sp = 0;
    if (n_dev) n = min(n, *n_dev);
    const uint32_t k = blockIdx.x * TRACE_BLOCK + threadIdx.x;
    uint32_t err = 0, nvis = 0, ntri = 0;
    if (k < n) {
        const uint32_t i = order ? __ldg(order + k) : k;
        const float4 r0 = __ldg(rays + 2ull * i), r1 = __ldg(rays + 2ull * i + 1);
        Best best;
        best.t = r0.w;
        best.u = best.v = 0.0f;
        best.prim = -1;
        best.obj = -1;
        const float sx = safe_inv(r1.x), sy = safe_inv(r1.y), sz = safe_inv(r1.z);
        if (TLAS && sv.tlas) { // the instance tree
            uint32_t tstk[TLAS_STACK];
            int tsp = 1;
            tstk[0] = 0;
            for (int m; (m = tlas_next(sv, r0, sx, sy, sz, best.t, tstk, tsp, err)) >= 0;) {
                const InstanceRec *ir = sv.inst + m;
                trace_mesh<COUNT>(mesh_of(sv, ir, m), transform_ray(ir, r0, r1), best, st, err, nvis, ntri);
            }
        } else {
            for (uint32_t m = 0; m < sv.n_inst; m++) {
                const InstanceRec *ir = sv.inst + m;
                float bmin[3], bmax[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    bmin[k] = __ldg(&ir->bbox_min[k]);
                    bmax[k] = __ldg(&ir->bbox_max[k]);
                }
                if (!ref_bbox_test(r0.x, r0.y, r0.z, sx, sy, sz, best.t, bmin, bmax)) continue;
                trace_mesh<COUNT>(mesh_of(sv, ir, (int)m), transform_ray(ir, r0, r1), best, st, err, nvis, ntri);
            }
        }
        hits[i] = make_float4(__int_as_float(best.prim), best.t, best.prim >= 0 ? best.u : 0.0f, best.prim >= 0 ? best.v : 0.0f);
        if (obj_out) obj_out[i] = best.obj;
    }
    flush_counters<COUNT>(err, nvis, ntri, err_out, counters);
}

// Persistent variant. Per lane: the ray it owns (index ri), the next instance
// to try (mi) and, while a mesh is being traversed (in_mesh), the traversal
// state. Each loop iteration of a warp: refill lanes without a ray when
// enough of them are idle, advance lanes to their next instance (or finish
// their ray), then one node step plus the triangles it hit.
// MULTI: rays of several scenes in one launch; ray i belongs to the scene
// whose SceneView is at views + ray_job[i] * view_stride.
// ANY: shadow rays -- a ray ends at its first accepted hit on a solid
// triangle (Traverse_MacroTree_WithStack_AnyHit, CoreRef.cpp:1224-1368).
// ONE: a lane tests one triangle per loop iteration and takes its next node
// only when the triangles of the last one are done, so each iteration is at
// most one node step and one triangle test per lane; otherwise a lane tests
// all the triangles of its node step in the same iteration, and the warp's
// triangle loop runs as long as its longest list.
template <bool COUNT, bool DEEP, bool MULTI, bool ANY, int BLOCK, int SDEPTH, bool TLAS, bool ONE>
__device__ __forceinline__ void trace_persistent(SceneView sv, const float4 *__restrict__ rays, uint32_t n, float4 *__restrict__ hits,
                                                 int32_t *__restrict__ obj_out, uint32_t *__restrict__ err_out,
                                                 unsigned long long *__restrict__ counters, uint32_t *__restrict__ next_ray, int refill_min,
                                                 const uint32_t *__restrict__ n_dev, const uint8_t *__restrict__ views, uint32_t view_stride,
                                                 const uint32_t *__restrict__ ray_job, const uint32_t *__restrict__ order, int stream_hint) {
    if (n_dev) n = min(n, *n_dev);
    __shared__ uint2 s_stack[SDEPTH * BLOCK];
    Stack<DEEP, BLOCK, SDEPTH> st;
    st.smem = s_stack + threadIdx.x;
    st.sp = 0;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lanemask_lt = (1u << lane) - 1u;
    uint32_t err = 0, nvis = 0, ntri = 0;
    uint32_t ri = NO_RAY, mi = 0, visits = 0, steps = 0;
    uint32_t tstk[TLAS ? TLAS_STACK : 1]; // the ray's instance-tree stack (scenes with an instance tree)
    int tsp = 0;
    bool in_mesh = false;
    Best best;
    best.t = 0.0f;
    best.u = best.v = 0.0f;
    best.prim = best.obj = -1;
    LocalRay r = make_local_ray(0.0f, 0.0f, 0.0f, 1.0f, 1.0f, 1.0f);
    MeshRef mr{};
    uint32_t ng_base = 0, ng_bits = 0, tg_base = 0, tg_bits = 0;
    bool pool_empty = false;
    while (true) {
        // ---- refill lanes that have no ray
        const uint32_t need = __ballot_sync(0xffffffffu, ri == NO_RAY);
        if (!pool_empty && need != 0 && (__popc(need) >= refill_min || need == 0xffffffffu)) {
            const uint32_t leader = __ffs(need) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(next_ray, (uint32_t)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(need) >= n) pool_empty = true;
            if (ri == NO_RAY) {
                const uint32_t idx = base + __popc(need & lanemask_lt);
                if (idx < n) {
                    ri = order ? __ldg(order + idx) : idx;
                    mi = 0;
                    if (TLAS) {
                        tstk[0] = 0; // the tree's root, for a scene that has one
                        tsp = 1;
                    }
                    in_mesh = false;
                    best.t = __ldg(&rays[2ull * ri].w);
                    best.u = best.v = 0.0f;
                    best.prim = best.obj = -1;
                }
            }
        }
        if (pool_empty && __all_sync(0xffffffffu, ri == NO_RAY)) break;
        // A lane without work this iteration falls through to the next one;
        // with ONE the warp meets again (__syncwarp) after each phase, which
        // keeps lanes that took different branches from drifting into
        // different iterations (measured: 4.28 ms without, 3.7 ms with, per
        // 4M-ray launch of the microbench on B200)
        bool idle = ri == NO_RAY;
        if (!ONE && idle) continue;
        // ---- next instance whose box the ray enters, or the end of the ray
        // (a ray whose scene has no instance left is done without reading it
        // again; a multi-scene ray reads its scene view first)
        if (!idle && !in_mesh) {
          if (MULTI || (TLAS && sv.tlas ? tsp > 0 : mi < sv.n_inst)) {
            // streaming hint: the ray is read once per instance pass and the
            // hit written once, so they may leave L1/L2 first (evict-first),
            // which keeps more of the BVH resident
            const float4 r0 = stream_hint ? __ldcs(rays + 2ull * ri) : __ldg(rays + 2ull * ri);
            const float4 r1 = stream_hint ? __ldcs(rays + 2ull * ri + 1) : __ldg(rays + 2ull * ri + 1);
            const float sx = safe_inv(r1.x), sy = safe_inv(r1.y), sz = safe_inv(r1.z);
            SceneView job_sv;
            if (MULTI) job_sv = *reinterpret_cast<const SceneView *>(views + (size_t)__ldg(ray_job + ri) * view_stride);
            const SceneView &lsv = MULTI ? job_sv : sv;
            if (TLAS && lsv.tlas) {
                const int m = tlas_next(lsv, r0, sx, sy, sz, best.t, tstk, tsp, err);
                if (m >= 0) {
                    const InstanceRec *ir = lsv.inst + m;
                    mr = mesh_of(lsv, ir, m);
                    r = transform_ray(ir, r0, r1);
                    ng_base = 0;
                    ng_bits = (1u << (24 + r.oct)) | 1u;
                    tg_bits = 0;
                    st.sp = 0;
                    visits = 0;
                    steps = 0;
                    in_mesh = true;
                }
            }
            while ((!TLAS || !lsv.tlas) && mi < lsv.n_inst) {
                const InstanceRec *ir = lsv.inst + mi;
                float bmin[3], bmax[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    bmin[k] = __ldg(&ir->bbox_min[k]);
                    bmax[k] = __ldg(&ir->bbox_max[k]);
                }
                mi++;
                if (!ref_bbox_test(r0.x, r0.y, r0.z, sx, sy, sz, best.t, bmin, bmax)) continue;
                mr = mesh_of(lsv, ir, (int)mi - 1);
                r = transform_ray(ir, r0, r1);
                ng_base = 0;
                ng_bits = (1u << (24 + r.oct)) | 1u;
                tg_bits = 0;
                st.sp = 0;
                visits = 0;
                steps = 0;
                in_mesh = true;
                break;
            }
          }
            if (!in_mesh) {
                const float4 h = make_float4(__int_as_float(best.prim), best.t, best.prim >= 0 ? best.u : 0.0f, best.prim >= 0 ? best.v : 0.0f);
                if (stream_hint) __stcs(hits + ri, h);
                else hits[ri] = h;
                if (obj_out) obj_out[ri] = best.obj;
                ri = NO_RAY;
                idle = true;
                if (!ONE) continue;
            }
        }
        if (ONE) __syncwarp();
        // ---- one traversal step: a node visit and the triangles it hits. A
        // mesh takes at most node_count steps; more means a corrupt structure.
        // Every group pushed today has a node bit, so the else branch (a group
        // of triangles only, tested as such) does not run; keeping the node
        // step under this test measured 4.8 ms instead of 6.9 ms per 4M-ray
        // launch on B200, the compiler keeping the warp converged around it.
        if (!idle && (!ONE || tg_bits == 0)) {
            bool ok = ++steps <= mr.node_count + 8u;
            if (!ok) err |= TRACE_ERR_LIMIT;
            if (ok && ng_bits > 0x00FFFFFFu) {
                ok = node_step<COUNT>(mr, r, best.t, ng_base, ng_bits, tg_base, tg_bits, st, visits, err, nvis);
            } else if (ok) {
                tg_base = ng_base;
                tg_bits = ng_bits;
                ng_bits = 0;
            }
            if (!ok) {
                in_mesh = false;
                mi = 0xffffffffu; // abandon the ray; the error flag reports it
                tsp = 0;
                tg_bits = 0;
                idle = true;
                if (!ONE) continue;
            }
        }
        if (ONE) __syncwarp();
        bool stop = false;
        if (ONE) {
            if (!idle && tg_bits) {
                const uint32_t k = __ffs(tg_bits) - 1;
                tg_bits &= tg_bits - 1;
                if (ANY) {
                    if (tri_test<COUNT, true>(mr, r, tg_base + k, best, err, ntri)) {
                        stop = true;
                        tg_bits = 0;
                    }
                } else {
                    tri_test<COUNT>(mr, r, tg_base + k, best, err, ntri);
                }
            }
        } else {
            while (!idle && tg_bits) {
                const uint32_t k = __ffs(tg_bits) - 1;
                tg_bits &= tg_bits - 1;
                if (ANY) {
                    if (tri_test<COUNT, true>(mr, r, tg_base + k, best, err, ntri)) {
                        stop = true;
                        tg_bits = 0;
                    }
                } else {
                    tri_test<COUNT>(mr, r, tg_base + k, best, err, ntri);
                }
            }
        }
        if (ONE) __syncwarp();
        if (idle) continue;
        if (ANY && stop) { // a solid triangle blocks the ray: no further instance
            in_mesh = false;
            mi = 0xffffffffu;
            tsp = 0;
            continue;
        }
        if (tg_bits == 0 && ng_bits <= 0x00FFFFFFu) {
            if (st.sp == 0) {
                in_mesh = false;
            } else {
                const uint2 e = st.pop();
                ng_base = e.x;
                ng_bits = e.y;
            }
        }
    }
    flush_counters<COUNT>(err, nvis, ntri, err_out, counters);
}

template <bool COUNT, bool DEEP, bool MULTI = false, bool ANY = false, int BLOCK = TRACE_BLOCK, int SDEPTH = SMEM_STACK, bool TLAS = false,
          bool ONE = false>
__global__ void __launch_bounds__(BLOCK) k_trace_persistent(SceneView sv, const float4 *__restrict__ rays, uint32_t n,
                                                                  float4 *__restrict__ hits, int32_t *__restrict__ obj_out,
                                                                  uint32_t *__restrict__ err_out, unsigned long long *__restrict__ counters,
                                                                  uint32_t *__restrict__ next_ray, int refill_min,
                                                                  const uint32_t *__restrict__ n_dev, const uint8_t *__restrict__ views = nullptr,
                                                                  uint32_t view_stride = 0, const uint32_t *__restrict__ ray_job = nullptr,
                                                                  const uint32_t *__restrict__ order = nullptr, int stream_hint = 0) {
    trace_persistent<COUNT, DEEP, MULTI, ANY, BLOCK, SDEPTH, TLAS, ONE>(sv, rays, n, hits, obj_out, err_out, counters, next_ray, refill_min,
                                                                        n_dev, views, view_stride, ray_job, order, stream_hint);
}

// The closest-hit, one-triangle-per-step form for scenes without an
// instance tree whose BVHs fit the shared stack, with registers bounded so
// that 1024 threads per SM stay resident (64 registers; no spills, where the
// other instances of the kernel would spill at that bound): measured
// 3.23 ms per 4M-ray launch of the microbench on B200 against 3.33 ms at 72
// registers and 896 threads (64 threads per block, 16 stack entries).
template <int BLOCK, int SDEPTH>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) k_trace_closest_one(SceneView sv, const float4 *__restrict__ rays, uint32_t n,
                                                                          float4 *__restrict__ hits, int32_t *__restrict__ obj_out,
                                                                          uint32_t *__restrict__ err_out,
                                                                          unsigned long long *__restrict__ counters,
                                                                          uint32_t *__restrict__ next_ray, int refill_min,
                                                                          const uint32_t *__restrict__ n_dev,
                                                                          const uint32_t *__restrict__ order, int stream_hint) {
    trace_persistent<false, false, false, false, BLOCK, SDEPTH, false, true>(sv, rays, n, hits, obj_out, err_out, counters, next_ray,
                                                                              refill_min, n_dev, nullptr, 0, nullptr, order, stream_hint);
}

int g_persistent_blocks[2][2] = {{0, 0}, {0, 0}}; // [DEEP][TLAS]

// The closest-hit persistent kernel with a tuned block size and shared stack
// depth (one resident grid: the SM count times the blocks that fit per SM).
template <bool DEEP, bool TLAS, int BLOCK, int SDEPTH, bool ONE>
cudaError_t launch_tuned(const SceneView &sv, const float4 *rays, uint32_t n, float4 *hits, int32_t *obj, uint32_t *err,
                         unsigned long long *counters, cudaStream_t st, const TraceParams &tp) {
    static_assert(SDEPTH * BLOCK * 8 <= 48 * 1024, "static shared memory limit");
    // k_trace_closest_one: with 16 stack entries (at 24 per thread its 1024 threads
    // hold 192 KB of shared stack per SM, and it measured 4.12 ms against 3.38
    // for the unbounded kernel, which keeps more of the SM's L1)
    constexpr bool FAST = ONE && !DEEP && !TLAS && SDEPTH <= 16;
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) {
            if (FAST)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_closest_one<BLOCK, SDEPTH>, BLOCK, 0);
            else
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_persistent<false, DEEP, false, false, BLOCK, SDEPTH, TLAS, ONE>,
                                                                  BLOCK, 0);
        }
        if (e != cudaSuccess) return e;
        blocks = sms * (per_sm > 0 ? per_sm : 1);
    }
    cudaError_t e = cudaMemsetAsync(tp.next_ray, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    if (FAST)
        k_trace_closest_one<BLOCK, SDEPTH><<<blocks, BLOCK, 0, st>>>(sv, rays, n, hits, obj, err, counters, tp.next_ray, tp.refill_min, tp.count,
                                                                     tp.order, tp.stream_hint);
    else
        k_trace_persistent<false, DEEP, false, false, BLOCK, SDEPTH, TLAS, ONE><<<blocks, BLOCK, 0, st>>>(
            sv, rays, n, hits, obj, err, counters, tp.next_ray, tp.refill_min, tp.count, nullptr, 0, nullptr, tp.order, tp.stream_hint);
    return cudaGetLastError();
}

template <bool DEEP, bool TLAS>
cudaError_t launch_tuned_dispatch(const SceneView &sv, const float4 *rays, uint32_t n, float4 *hits, int32_t *obj, uint32_t *err,
                                  unsigned long long *counters, cudaStream_t st, const TraceParams &tp) {
#define RG_TUNED(B, D)                                                                                                                  \
    if (tp.block == B && tp.smem_stack == D)                                                                                            \
        return tp.one_tri ? launch_tuned<DEEP, TLAS, B, D, true>(sv, rays, n, hits, obj, err, counters, st, tp)                          \
                          : launch_tuned<DEEP, TLAS, B, D, false>(sv, rays, n, hits, obj, err, counters, st, tp);
    RG_TUNED(64, 16) RG_TUNED(64, 24) RG_TUNED(64, 32)
    RG_TUNED(128, 16) RG_TUNED(128, 24) RG_TUNED(128, 32)
    RG_TUNED(256, 16) RG_TUNED(256, 24)
#undef RG_TUNED
    return cudaErrorInvalidValue;
}

template <bool DEEP, bool TLAS>
cudaError_t launch_impl(const SceneView &sv, const float4 *rays, uint32_t n, float4 *hits, int32_t *obj, uint32_t *err,
                        unsigned long long *counters, bool count, cudaStream_t st, const TraceParams &tp) {
    constexpr int B = TRACE_BLOCK, D = SMEM_STACK;
    if (!tp.persistent && !tp.views && !tp.any) {
        const uint32_t grid = (n + TRACE_BLOCK - 1) / TRACE_BLOCK;
        if (count)
            k_trace_closest<true, DEEP, TLAS><<<grid, TRACE_BLOCK, 0, st>>>(sv, rays, n, hits, obj, err, counters, tp.count, tp.order);
        else
            k_trace_closest<false, DEEP, TLAS><<<grid, TRACE_BLOCK, 0, st>>>(sv, rays, n, hits, obj, err, counters, tp.count, tp.order);
        return cudaGetLastError();
    }
    if (!tp.next_ray) return cudaErrorInvalidValue;
    if (!count && !tp.views && !tp.any && (tp.one_tri || !(tp.block == TRACE_BLOCK && tp.smem_stack == SMEM_STACK)))
        return launch_tuned_dispatch<DEEP, TLAS>(sv, rays, n, hits, obj, err, counters, st, tp);
    int &blocks = g_persistent_blocks[DEEP ? 1 : 0][TLAS ? 1 : 0];
    if (blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_persistent<false, DEEP, false, false, B, D, TLAS>, TRACE_BLOCK, 0);
        if (e != cudaSuccess) return e;
        blocks = sms * (per_sm > 0 ? per_sm : 1);
    }
    cudaError_t e = cudaMemsetAsync(tp.next_ray, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    // shadow rays and rays of several scenes (no counting variants), with one
    // triangle test per step or a node's triangles at once
#define RG_LAUNCH_P(MULTI_, ANY_, ONE_)                                                                                                 \
    k_trace_persistent<false, DEEP, MULTI_, ANY_, B, D, TLAS, ONE_><<<blocks, TRACE_BLOCK, 0, st>>>(                                    \
        sv, rays, n, hits, obj, err, counters, tp.next_ray, tp.refill_min, tp.count, tp.views, tp.view_stride, tp.ray_job)
    if (tp.any) {
        if (tp.views) {
            if (tp.one_tri) RG_LAUNCH_P(true, true, true);
            else RG_LAUNCH_P(true, true, false);
        } else {
            if (tp.one_tri) RG_LAUNCH_P(false, true, true);
            else RG_LAUNCH_P(false, true, false);
        }
        return cudaGetLastError();
    }
    if (tp.views) {
        if (tp.one_tri) RG_LAUNCH_P(true, false, true);
        else RG_LAUNCH_P(true, false, false);
        return cudaGetLastError();
    }
#undef RG_LAUNCH_P
    if (count)
        k_trace_persistent<true, DEEP, false, false, B, D, TLAS><<<blocks, TRACE_BLOCK, 0, st>>>(
            sv, rays, n, hits, obj, err, counters, tp.next_ray, tp.refill_min, tp.count, nullptr, 0, nullptr, tp.order);
    else
        k_trace_persistent<false, DEEP, false, false, B, D, TLAS><<<blocks, TRACE_BLOCK, 0, st>>>(
            sv, rays, n, hits, obj, err, counters, tp.next_ray, tp.refill_min, tp.count, nullptr, 0, nullptr, tp.order, tp.stream_hint);
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_trace_closest(const SceneView &sv, const float4 *rays, uint32_t n, float4 *hits, int32_t *obj, uint32_t *err,
                                 unsigned long long *counters, bool count, cudaStream_t st, const TraceParams &tp) {
    if (n == 0) return cudaSuccess;
    // one group per level at most: the shared-memory stack suffices up to its
    // depth in levels (the tuned closest-hit kernel's depth where it applies)
    const bool tuned = tp.persistent && !count && !tp.views && !tp.any;
    const uint32_t sdepth = tuned ? (uint32_t)tp.smem_stack : (uint32_t)SMEM_STACK;
    if (tp.tlas) {
        if (tp.max_depth < sdepth) return launch_impl<false, true>(sv, rays, n, hits, obj, err, counters, count, st, tp);
        return launch_impl<true, true>(sv, rays, n, hits, obj, err, counters, count, st, tp);
    }
    if (tp.max_depth < sdepth) return launch_impl<false, false>(sv, rays, n, hits, obj, err, counters, count, st, tp);
    return launch_impl<true, false>(sv, rays, n, hits, obj, err, counters, count, st, tp);
}

} // namespace rg
