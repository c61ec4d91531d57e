// trace_epilogue.hpp -- runs the reference's per-ray kernel
// (kernels/CUDA_raytraceMeshTree.cu:111-219, the coherency=false path) one
// pixel at a time with the launch shape of :461-472 (8x4 blocks). Misses leave
// face id / coords unspecified, as in the reference; only depth is defined.
// TEST INFRASTRUCTURE ONLY.
REF_API void ref_trace(const float* nodes, const float* vertices, const uint* faces, const float* orig, const float* dir,
                       int width, int height, uint* faces_id, float* coords, float* depths) {
  tex_nodes.ptr = (const uint4*)nodes;
  tex_vertices.ptr = (const float4*)vertices;
  tex_faces.ptr = (const uint4*)faces;
  tex_rays_orig.ptr = (const float4*)orig;
  tex_rays_dir.ptr = (const float4*)dir;
  blockDim = {BLOCK_WIDTH, BLOCK_HEIGHT, 1};
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      blockIdx = {(uint)(x / BLOCK_WIDTH), (uint)(y / BLOCK_HEIGHT), 0};
      threadIdx = {(uint)(x % BLOCK_WIDTH), (uint)(y % BLOCK_HEIGHT), 0};
      kernel_raytraceMeshTree(faces_id, (float2*)coords, depths, width, height);
    }
}
