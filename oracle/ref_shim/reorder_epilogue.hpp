// reorder_epilogue.hpp -- runs kernel_reorderMesh of kernels/CUDA_reorderMeshFaces.cu.
// TEST INFRASTRUCTURE ONLY.
REF_API void ref_reorder_faces(const uint* faces, const uint* indices, uint n, uint* faces_out) {
  tex_faces_id.ptr = indices;
  tex_faces.ptr = (const uint4*)faces;
  uint grid = (n + BLOCK_SIZE - 1) / BLOCK_SIZE;
  blockDim = {BLOCK_SIZE, 1, 1};
  for (uint b = 0; b < grid; ++b)
    for (uint t = 0; t < BLOCK_SIZE; ++t) { blockIdx = {b, 0, 0}; threadIdx = {t, 0, 0}; kernel_reorderMesh((uint4*)faces_out, (int)n); }
}
