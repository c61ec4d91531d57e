// raster_epilogue.hpp -- host drivers: the camera's view / projection matrices
// from CUDACamera::update (compiled from CUDACamera.cpp), and the rasteriser
// kernel run as the reference launches it (2 x 2 blocks of 8 x 4 threads, one
// block after another, each block on 32 host threads). The matrix the
// reference passes is transpose(view * proj) (kernels/CUDA_rasterizeMeshTree.cu:261-263).
// TEST INFRASTRUCTURE ONLY.
REF_API void ref_raster_matrix(const float* center3, const float* dir3, const float* angle3, float fov, float ratio, float* out16) {
  renderkit::CUDACamera cam;
  cam.center = make_float3(center3[0], center3[1], center3[2]);
  cam.dir = make_float3(dir3[0], dir3[1], dir3[2]);
  cam.angle = make_float3(angle3[0], angle3[1], angle3[2]);
  cam.fov = fov;
  cam.ratio = ratio;
  cam.zNearPlane = 1.000f;   // CUDACamera.cpp:34
  cam.zFarPlane = 1999.999f; // CUDACamera.cpp:35
  cam.update();
  float4x4 m;
  matrixMultiply(m, cam.matView, cam.matProj);
  matrixTranspose(m);
  memcpy(out16, &m, 64);
}

REF_API void ref_rasterize(const float* vertices, const uint* faces, int face_count, const float* matrix16, int width, int height,
                           uint* faces_id, float* coords, float* depths) {
  tex_vertices.ptr = (const float4*)vertices;
  tex_faces.ptr = (const uint4*)faces;
  float4x4 m;
  memcpy(&m, matrix16, 64);
  ShimBlockPool pool(BLOCK_WIDTH);
  blockDim.x = BLOCK_WIDTH; blockDim.y = BLOCK_HEIGHT; blockDim.z = 1;
  for (unsigned by = 0; by < BLOCK_COUNT_Y; ++by)
    for (unsigned bx = 0; bx < BLOCK_COUNT_X; ++bx) {
      blockIdx.x = bx; blockIdx.y = by; blockIdx.z = 0;
      pool.run([&] { kernel_rasterizeMeshTree(faces_id, (float2*)coords, depths, m, face_count, width, height); });
    }
}
