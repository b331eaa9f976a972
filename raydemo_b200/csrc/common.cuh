// Shared device-side types and helpers of the B200 path tracer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace rg {

// Precomputed triangle in the layout of tri_accel_t (src/Ray/internal/Core.h:27-36),
// 48 bytes = three 16-byte loads. In the leaf-ordered copy used by traversal
// the last two words hold the global triangle index instead of the materials.
struct alignas(16) TriRec {
    float nu, nv, np, pu;
    float pv;
    int32_t ci;
    float e0u, e0v;
    float e1u, e1v;
    uint32_t mi, back_mi; // leaf copy: mi = global triangle index, back_mi unused
};
static_assert(sizeof(TriRec) == 48, "TriRec must stay 48 bytes");

constexpr int TRI_W_BITS = 3;
constexpr int TRI_AXIS_ALIGNED_BIT = 4;
constexpr int TRI_INV_NORMAL_BIT = 8;
constexpr int TRI_SOLID_BIT = 16;
constexpr float HIT_EPS = 0.000001f;
constexpr float FLT_EPS_ = 0.0000001f;
constexpr float MAX_DIST = 3.402823466e+38F;

// Compressed 8-wide node (80 bytes). Child boxes are quantised to 8 bits per
// plane against a per-node origin p and per-axis power-of-two scale 2^(e-127).
// The build picks p and e so that every decoded plane p + q * 2^e is an exact
// float and lies outside the exact child box by at least one quantum, so the
// slab test on the decoded box never rejects what a test on the exact box
// accepts.
//
// meta[i] (slot i): 0 = empty. Internal child: 0b001 << 5 | (24 + i). Leaf:
// unary triangle count (0b001, 0b011, 0b111) << 5 | offset of its first
// triangle from tri_base (0..21). Internal children are stored contiguously
// from child_base in slot order.
struct alignas(16) WideNode {
    float p[3];
    uint8_t e[3];
    uint8_t imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
};
static_assert(sizeof(WideNode) == 80, "WideNode must stay 80 bytes");

// Mesh instance as the traversal sees it (96 bytes).
struct alignas(16) InstanceRec {
    // inverse transform, column-major 4x4 without its last row:
    // [0..2] column 0, [3..5] column 1, [6..8] column 2, [9..11] translation
    float inv_xform[12];
    float bbox_min[3];
    uint32_t node_base; // first wide node of the mesh BVH in the scene node array
    float bbox_max[3];
    uint32_t tri_base;  // first leaf triangle of the mesh in the scene leaf array
    uint32_t prim_base;  // global index of the mesh's first triangle
    uint32_t mesh;
    uint32_t node_count; // bounds for the traversal's index checks
    uint32_t tri_count;
};
static_assert(sizeof(InstanceRec) == 96, "InstanceRec must stay 96 bytes");

constexpr int LEAF_MAX_TRIS = 3;

// Instance tree node (binary, over the instances' world boxes): the boxes
// of both children and their ids; an id with TLAS_LEAF set is an instance
// index, else a node index (node 0 is the root).
constexpr uint32_t TLAS_LEAF = 0x80000000u;
struct TlasNode {
    float lo[2][3];
    float hi[2][3];
    uint32_t child[2];
    uint32_t pad[2];
};
static_assert(sizeof(TlasNode) == 64, "TlasNode must stay 64 bytes");

} // namespace rg

// Error helpers for host code.
namespace rg {
void set_error(const std::string &msg);
// Every device allocation of the library goes through device_alloc, so that
// a test can make the n-th next one fail on the host (ray_debug_fail_device_alloc).
cudaError_t device_alloc(void **p, size_t bytes);
// Host waits with a bound (ray_set_wait_timeout_ms; default 300 s): poll the
// event or stream until it completes, an error is reported, or the bound
// passes (cudaErrorTimeout; the GPU work itself is not stopped).
cudaError_t wait_event(cudaEvent_t e);
cudaError_t wait_stream(cudaStream_t s);
} // namespace rg

// Returns from the calling entry point with the RAY_ERR_* code of a failed
// CUDA call (a bounded wait that ran out: RAY_ERR_TIMEOUT; a failed
// allocation: RAY_ERR_OUT_OF_MEMORY; anything else: RAY_ERR_CUDA).
#define RG_CUDA_TRY(expr)                                                                                              \
    do {                                                                                                               \
        cudaError_t _e = (expr);                                                                                       \
        if (_e != cudaSuccess) {                                                                                       \
            ::rg::set_error(std::string(#expr " failed: ") + cudaGetErrorString(_e));                                 \
            return _e == cudaErrorTimeout ? RAY_ERR_TIMEOUT                                                            \
                                          : (_e == cudaErrorMemoryAllocation ? RAY_ERR_OUT_OF_MEMORY : RAY_ERR_CUDA); \
        }                                                                                                              \
    } while (0)
