/* rt_sah.h -- C ABI of the SAH and Hybrid BVH builds (sm_100a).
 *
 * Replaces CUDA_buildMeshTreeSAH (kernels/CUDA_buildMeshTreeSAH.cu:672-789) as
 * called by CUDAMeshTree::buildMeshTreeSAH (CUDAMeshTree.cpp:93-96) and, after
 * an LBVH build of `lbvh_depth` levels without leaf splitting or face reorder,
 * by CUDAMeshTree::buildMeshTreeHybrid (CUDAMeshTree.cpp:98-103).
 *
 * The tree is the one a serial execution of the reference's launches builds:
 * a node is split when it is popped from the reference's stack, depth first,
 * left child first, so the k-th split of a subtree whose root was popped when
 * the node counter stood at B gets children B + 2k and B + 2k + 1 (the
 * reference's concurrent blocks allocate ids in a racy order). Splits: 32
 * bins over the centroid bounds' longest axis, cost 2 * 1.0 + 0.125 * (area
 * ratios x counts); a node of <= 16 faces, or of < 224 faces whose best cost
 * exceeds 0.125 (count + 1), is a leaf. A node of >= 224 faces that no bin
 * boundary separates into two non-empty sides is also a leaf (the reference
 * never terminates there). Node records, indices and reordered faces have the
 * reference's layouts (rt_core.h); bits 3-31 of an internal node's first word
 * are zero (the reference leaves them unset). Boxes: min over -0/+0 is -0.
 */
#ifndef RT_SAH_H
#define RT_SAH_H

#include "rt_core.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rt_sah_desc {
  const float* vertices; /* float4 per vertex */
  uint32_t vertex_count;
  uint32_t face_count;
  const uint32_t* faces_in; /* uint4 per face */
  uint32_t* faces_out;      /* uint4 per face, position order; must not alias faces_in */
  const float* hitbox;      /* optional: 8 floats (min xyzw, max xyzw); NULL = the vertices' bounds */
  uint32_t lbvh_depth;      /* 0: SAH build; 1..32: Hybrid (LBVH of this depth, then SAH in every leaf) */
  float* boxes;             /* out: aabox per original face */
  uint32_t* indices;        /* out: original face id per position */
  uint32_t* nodes;          /* out: bvnode records */
  uint32_t max_nodes;       /* capacity of nodes (rt_sah_sizes) */
  float* tris;              /* optional out: {v0, e1, e2} per position (traversal triangle stream) */
  void* accel;              /* optional out: traversal blob (rt_lbvh_accel_bytes(face_count) bytes) */
  size_t accel_bytes;
  rt_build_info* info;      /* device memory: node_count, leaf_count, real_depth = levels processed, error;
                               overrun_visits = leaves of >= 224 faces that no bin boundary could split */
  void* scratch;
  size_t scratch_bytes;
} rt_sah_desc;

/* Scratch bytes and node capacity for a build of face_count faces. */
rt_status rt_sah_sizes(uint32_t face_count, uint32_t lbvh_depth, size_t* scratch_bytes, uint32_t* max_nodes);
/* Builds the tree. The call waits for the stream once per tree level (it reads
 * the level's node count), so it cannot be captured in a CUDA graph. */
rt_status rt_sah_build(const rt_sah_desc* d, rt_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* RT_SAH_H */
