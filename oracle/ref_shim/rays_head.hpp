// rays_head.hpp -- opens the driver around the reference's host camera basis
// (kernels/CUDA_calcPrimaryRays.cu:43-55), which is inserted right after this.
// TEST INFRASTRUCTURE ONLY.
REF_API void ref_camera_rays(const float* center3, const float* target3, float fov_in, float ratio_in, int width, int height,
                             float* angle_out3, float* basis_out16, float* orig_out, float* dir_out) {
  CUDACamera cam;
  cam.fov = fov_in; cam.ratio = ratio_in;
  cam.center = make_float3(center3[0], center3[1], center3[2]);
  cam.angle = make_float3(PI * 0.5f, 0.0f, 0.0f);  // CUDACamera.cpp:41-43
  cam.dir = make_float3(0.0f, 0.0f, 1.0f);
  cam.lookAt(target3[0], target3[1], target3[2]);
  CUDACamera* camera = &cam;
