// rays_tail.hpp -- closes ref_camera_rays: stores the basis and runs
// kernel_calcPrimaryRays (kernels/CUDA_calcPrimaryRays.cu:20-32) per pixel.
// TEST INFRASTRUCTURE ONLY.
  angle_out3[0] = cam.angle.x; angle_out3[1] = cam.angle.y; angle_out3[2] = cam.angle.z;
  memcpy(basis_out16 + 0, &rayOrig, 16); memcpy(basis_out16 + 4, &rayDir, 16);
  memcpy(basis_out16 + 8, &rayX, 16); memcpy(basis_out16 + 12, &rayY, 16);
  blockDim = {16, 16, 1};
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      blockIdx = {(uint)(x / 16), (uint)(y / 16), 0};
      threadIdx = {(uint)(x % 16), (uint)(y % 16), 0};
      kernel_calcPrimaryRays((float4*)orig_out, (float4*)dir_out, width, height, rayOrig, rayDir, rayX, rayY);
    }
}
