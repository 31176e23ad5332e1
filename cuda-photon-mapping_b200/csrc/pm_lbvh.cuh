// pm_lbvh.cuh -- device BVH builder (linear BVH over Morton codes).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace pm {

// Device scratch for lbvh_build over ntri triangles.
size_t lbvh_scratch_bytes(int ntri);

// Interior nodes the builder writes (node 0 is the root).
inline int64_t lbvh_node_count(int ntri) { return ntri > 1 ? (int64_t)ntri - 1 : 1; }

// BVH over ntri triangles (tri_pos: device, 9 floats per triangle) in the
// traversal's node format (pm_scene.cuh): nodes = lbvh_node_count(ntri) x 4
// float4, both children's padded boxes (box +- (pad + 1e-5 |coordinate|))
// with their refs; prim = ntri triangle indices (Morton order).  Subtrees of
// at most 4 triangles become leaves.  ntri < 2^23.
cudaError_t lbvh_build(const float* tri_pos, int ntri, float pad, float4* nodes, int* prim, void* scratch,
                       unsigned* status, int* launches, cudaStream_t st);

// Triangle records in leaf order, 4 float4 each: out[j] = the first three
// float4 of tri[prim[j]] and its fifth (the normal) with the triangle's index
// in w (the fourth, v0 - v2, is formed by the test).
cudaError_t bvh_leaf_records(const float4* tri, const int* prim, int ntri, float4* out, cudaStream_t st);

}  // namespace pm
