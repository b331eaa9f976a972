// GPU BVH construction for one mesh.
#pragma once

#include "common.cuh"

namespace rg {

struct MeshBvh {
    WideNode *nodes = nullptr;  // node 0 is the root
    uint32_t node_count = 0;
    TriRec *leaf_tris = nullptr; // leaf order; .mi = triangle index within the mesh
    uint32_t tri_count = 0;
    uint32_t depth = 0;          // wide levels on the longest root-to-leaf path
    float bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
};

void free_mesh_bvh(MeshBvh &b);

// PreprocessTri (src/Ray/internal/Core.cpp:162-214) for n triangles given as
// 9 floats each (three vertex positions), plus their axis-aligned boxes.
// mat: 3 words per triangle (front material, back material, solid flag).
cudaError_t launch_preprocess_tris(const float *verts, const uint32_t *mat, uint32_t n, TriRec *tris_out, float *aabb_out,
                                   cudaStream_t st);

// Builds the wide BVH over n preprocessed triangles (Ref order) with boxes
// aabb (6 floats each): LBVH over 64-bit Morton keys, greedy collapse to
// 8-wide nodes, quantised child boxes. Allocates out.nodes / out.leaf_tris.
// Returns RAY_OK or a RAY_ERR_* code (message through set_error).
int build_mesh_bvh(const TriRec *tris_ref, const float *aabb, uint32_t n, MeshBvh &out, cudaStream_t st);

// The instance tree: an LBVH over the instances' world boxes (Morton codes
// of the box centres, the same radix sort and binary radix tree as a mesh's
// build), its node boxes computed bottom-up and packed into TlasNode
// records. A refit keeps the topology and recomputes only the boxes (after
// instances moved); a build is needed when the instance count changed.
struct InstTree {
    uint32_t n = 0;              // instances of the current topology (0: none built)
    float *aabb = nullptr;       // 6 floats per instance: world box
    uint32_t *sorted = nullptr;  // sorted position -> instance index
    uint32_t *left = nullptr, *right = nullptr, *parent = nullptr, *first = nullptr, *last = nullptr;
    float *nb = nullptr;         // node boxes (6 floats per internal node)
    uint32_t *flags = nullptr;   // arrival counters of the bottom-up passes
    TlasNode *nodes = nullptr;   // n - 1 packed nodes
};
void free_inst_tree(InstTree &t);
// boxes: n world boxes (6 floats each) in host memory. refit: keep the
// topology (requires t.n == n). Returns RAY_OK or a RAY_ERR_* code.
int build_inst_tree(const float *boxes, uint32_t n, bool refit, InstTree &t, cudaStream_t st);

} // namespace rg
