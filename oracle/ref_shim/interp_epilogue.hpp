// interp_epilogue.hpp -- runs kernel_interpolateData of
// kernels/CUDA_interpolateData.cu one pixel at a time (16x16 blocks, :233-248).
// TEST INFRASTRUCTURE ONLY.
REF_API void ref_interpolate(const uint* faces_id, const float* coords, int width, int height, const uint* faces, const float* vertices,
                             const float* normals, const float* colors, const float* texcoords, float* points, float* out_normals,
                             float* out_colors, float* out_texcoords, uint* materials) {
  tex_faces_id.ptr = faces_id;
  tex_coords.ptr = (const float2*)coords;
  tex_faces.ptr = (const uint4*)faces;
  tex_vertices.ptr = (const float4*)vertices;
  tex_normals.ptr = (const float4*)normals;
  tex_colors.ptr = (const float4*)colors;
  tex_texcoords.ptr = (const float2*)texcoords;
  blockDim = {BLOCK_WIDTH, BLOCK_HEIGHT, 1};
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      blockIdx = {(uint)(x / BLOCK_WIDTH), (uint)(y / BLOCK_HEIGHT), 0};
      threadIdx = {(uint)(x % BLOCK_WIDTH), (uint)(y % BLOCK_HEIGHT), 0};
      kernel_interpolateData((float4*)points, (float4*)out_normals, (float4*)out_colors, (float2*)out_texcoords, materials, width, height,
                             normals != nullptr, colors != nullptr, texcoords != nullptr);
    }
}
