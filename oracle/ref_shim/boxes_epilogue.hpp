// boxes_epilogue.hpp -- runs kernel_initIndices / kernel_calcBoxes of
// kernels/CUDA_calcMeshBoxes.cu one simulated thread at a time.
// TEST INFRASTRUCTURE ONLY.
template <typename F>
static void shim_launch1d(uint count, uint block, F&& body) {
  uint grid = (count + block - 1) / block;
  blockDim = {block, 1, 1};
  for (uint b = 0; b < grid; ++b)
    for (uint t = 0; t < block; ++t) { blockIdx = {b, 0, 0}; threadIdx = {t, 0, 0}; body(); }
}
REF_API void ref_mesh_boxes(const float* vertices, const uint* faces, uint n, float* boxes_out, uint* indices_out) {
  tex_faces.ptr = (const uint4*)faces;
  tex_vertices.ptr = (const float4*)vertices;
  shim_launch1d(n, BLOCK_SIZE, [&] { kernel_initIndices(indices_out, n); });
  shim_launch1d(n, BLOCK_SIZE, [&] { kernel_calcBoxes((aabox*)boxes_out, (int)n); });
}
