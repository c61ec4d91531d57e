// rt_interp.cu -- per-ray attribute interpolation from (face, u, v).
//
// Replaces CUDA_interpolateData (kernels/CUDA_interpolateData.cu:45-138,216-256),
// the direct consumer of the traversal's hit buffers: hit point, normal (the
// interpolated vertex normal, or the face normal), color, texture coordinate
// and material of each ray's hit face. Weights are (1 - u - v, u, v) computed
// as the reference writes them, sums left to right, no FMA contraction; the
// reference normalizes with rsqrtf (an approximate instruction), this kernel
// with the IEEE 1 / sqrtf. A miss (id < 0) writes zeros, the values
// CUDABuffer::clearOutputSurfaces leaves in those surfaces (CUDABuffer.cpp:109-131);
// the reference instead reads a face through its uninitialised miss id.
#include "rt_common.cuh"

namespace rt {
namespace {

struct InterpArgs {
  const int32_t* hit_id;
  const float2* hit_uv;
  uint32_t count;
  const uint4* faces;
  const float4* verts;
  const float4* normals;
  const float4* colors;
  const float2* texcoords;
  float4* out_points;
  float4* out_normals;
  float4* out_colors;
  float2* out_texcoords;
  uint32_t* out_materials;
};

__device__ __forceinline__ float4 lerp3(float w0, float u, float v, float4 a, float4 b, float4 c) {
  return make_float4(w0 * a.x + u * b.x + v * c.x, w0 * a.y + u * b.y + v * c.y, w0 * a.z + u * b.z + v * c.z,
                     w0 * a.w + u * b.w + v * c.w);
}
// normalize(v) = v * (1 / sqrt(dot4(v, v)))
__device__ __forceinline__ float4 normalize4(float4 v) {
  const float inv = 1.0f / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w);
  return make_float4(v.x * inv, v.y * inv, v.z * inv, v.w * inv);
}

__global__ __launch_bounds__(256) void k_interpolate(InterpArgs A) {
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < A.count; l += gridDim.x * blockDim.x) {
    const int32_t id = A.hit_id[l];
    if (id < 0) {
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      if (A.out_points) A.out_points[l] = z;
      if (A.out_normals) A.out_normals[l] = z;
      if (A.out_colors) A.out_colors[l] = z;
      if (A.out_texcoords) A.out_texcoords[l] = make_float2(0.f, 0.f);
      if (A.out_materials) A.out_materials[l] = 0u;
      continue;
    }
    const float2 uv = A.hit_uv[l];
    const uint4 f = ldg4(A.faces + id);
    const float4 v0 = ldg4(A.verts + f.x), v1 = ldg4(A.verts + f.y), v2 = ldg4(A.verts + f.z);
    const float w0 = 1.0f - uv.x - uv.y;
    if (A.out_points) A.out_points[l] = lerp3(w0, uv.x, uv.y, v0, v1, v2);
    if (A.out_normals) {
      float4 n;
      if (A.normals) {
        n = normalize4(lerp3(w0, uv.x, uv.y, ldg4(A.normals + f.x), ldg4(A.normals + f.y), ldg4(A.normals + f.z)));
      } else {
        const float4 e1 = make_float4(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z, v1.w - v0.w);
        const float4 e2 = make_float4(v2.x - v0.x, v2.y - v0.y, v2.z - v0.z, v2.w - v0.w);
        n = normalize4(make_float4(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x, 0.0f));
      }
      A.out_normals[l] = n;
    }
    if (A.out_colors)
      A.out_colors[l] = A.colors ? lerp3(w0, uv.x, uv.y, ldg4(A.colors + f.x), ldg4(A.colors + f.y), ldg4(A.colors + f.z))
                                 : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    if (A.out_texcoords) {
      if (A.texcoords) {
        const float2 t0 = __ldg(A.texcoords + f.x), t1 = __ldg(A.texcoords + f.y), t2 = __ldg(A.texcoords + f.z);
        A.out_texcoords[l] = make_float2(w0 * t0.x + uv.x * t1.x + uv.y * t2.x, w0 * t0.y + uv.x * t1.y + uv.y * t2.y);
      } else {
        A.out_texcoords[l] = uv;
      }
    }
    if (A.out_materials) A.out_materials[l] = f.w;
  }
}

}  // namespace
}  // namespace rt

using namespace rt;

extern "C" rt_status rt_interpolate(const rt_interp_desc* d, rt_stream stream) {
  if (!d || !d->hit_id || !d->hit_uv || !d->faces || !d->vertices) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (d->count == 0) return RT_OK;
  InterpArgs A;
  A.hit_id = d->hit_id; A.hit_uv = (const float2*)d->hit_uv; A.count = d->count; A.faces = (const uint4*)d->faces;
  A.verts = (const float4*)d->vertices; A.normals = (const float4*)d->normals; A.colors = (const float4*)d->colors;
  A.texcoords = (const float2*)d->texcoords; A.out_points = (float4*)d->out_points; A.out_normals = (float4*)d->out_normals;
  A.out_colors = (float4*)d->out_colors; A.out_texcoords = (float2*)d->out_texcoords; A.out_materials = d->out_materials;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t blocks = (uint32_t)hmin<uint64_t>((d->count + 255) / 256, (uint64_t)sms * 16);
  k_interpolate<<<blocks, 256, 0, (cudaStream_t)stream>>>(A);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}
