// On-device SAH BVH builder (bvh_build.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "scene.cuh"

namespace rumi {

struct BvhBuildInfo {
    int large_levels;      // breadth-first levels of the large-task phase
    int small_tasks;       // subtrees built by the warp-per-task phase
    int node_capacity;     // entries reserved in the node array
    int node_high_water;   // first unused index of the large-phase region
};

int bvh_node_capacity(int n_prims);
size_t bvh_scratch_bytes(int n_prims);
// d_prim_flags: n_rects + n_spheres ints -- per rect "emissive" (one-sided test off), then
// per sphere "image-based light" (far root from inside)
int bvh_build(const float *d_tri_v, int n_tris, const float4 *d_rects, const int *d_prim_flags, int n_rects,
              const float4 *d_spheres, int n_spheres, BvhNode *nodes, float4 *leaf_prims, void *scratch,
              cudaStream_t stream, BvhBuildInfo *info);

// Four-wide tree collapsed from the binary one (bvh4.cu).
int bvh4_node_capacity(int n_prims);
size_t bvh4_scratch_bytes(int n_prims);
int bvh4_collapse(const BvhNode *nodes2, int n_nodes2, Bvh4Node *nodes4, int cap4, void *scratch,
                  cudaStream_t stream);

// Compressed eight-wide tree collapsed from the binary one (bvh8.cu); prims8 receives the
// leaf primitives in its order.  Returns the node count, 0 without primitives, -1 on error.
int bvh8_node_capacity(int n_prims);
size_t bvh8_scratch_bytes(int n_prims);
int bvh8_collapse(const BvhNode *nodes2, int n_nodes2, const float4 *prims2, int n_prims, Bvh8Node *nodes8, int cap8,
                  float4 *prims8, void *scratch, cudaStream_t stream);

}  // namespace rumi
