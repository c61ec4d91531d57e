// rt_host.cpp -- host-side pieces of the C ABI: camera math and status strings.
//
// Compiled by the host compiler with -ffp-contract=off so that the camera
// basis is the same IEEE computation the reference performs on the host
// (CUDACamera.cpp:70-88,126-132 and kernels/CUDA_calcPrimaryRays.cu:43-55).
#include <math.h>
#include <atomic>
#include <string.h>

#include "../../include/rt_core.h"
#include "../../include/rt_raster.h"

namespace {

const float kPi = 3.14159265359f;  // CUDACommon.h:108

struct V4 { float x, y, z, w; };
V4 add(V4 a, V4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
V4 scale(V4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
float dot(V4 a, V4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
V4 cross(V4 a, V4 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0f}; }
// normalize with the host rsqrtf of the reference (1 / sqrtf)
V4 normalize(V4 v) { float inv = 1.0f / sqrtf(dot(v, v)); return scale(v, inv); }

}  // namespace

extern "C" rt_status rt_camera_look_at(rt_camera* cam, const float target[3]) {
  if (!cam || !target) return RT_ERR_INVALID_ARGUMENT;
  // CUDACamera::lookAt: dir = target - center, then angleFromDir
  float dx = target[0] - cam->center[0], dy = target[1] - cam->center[1], dz = target[2] - cam->center[2];
  float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
  dx = dx * inv; dy = dy * inv; dz = dz * inv;
  float ay = asinf(dy);
  if (ay < -kPi * 0.5f + 0.001f) ay = -kPi * 0.5f + 0.001f;
  if (ay > kPi * 0.5f - 0.001f) ay = kPi * 0.5f - 0.001f;
  float ax;
  if (dx > 0) ax = asinf(dz / cosf(ay));
  else if (dz > 0) ax = acosf(dx / cosf(ay));
  else ax = acosf(-dx / cosf(-ay)) + kPi;
  if (ax < 0.0f) ax += kPi * 2.0f;
  if (ax > kPi * 2.0f) ax -= kPi * 2.0f;
  cam->angle[0] = ax;
  cam->angle[1] = ay;
  return RT_OK;
}

extern "C" rt_status rt_camera_basis(const rt_camera* cam, uint32_t width, uint32_t height, float basis[16]) {
  if (!cam || !basis || width == 0 || height == 0) return RT_ERR_INVALID_ARGUMENT;
  float y = tanf(cam->fov * 0.5f);
  float x = y * cam->ratio;
  float p = cam->angle[0], yw = cam->angle[1], r = cam->angle[2];
  V4 camDir = {cosf(p) * cosf(yw), sinf(yw), sinf(p) * cosf(yw), 0.0f};
  V4 camUp = {cosf(p) * sinf(r), cosf(r), 0.0f, 0.0f};
  V4 right = normalize(cross(camDir, camUp));
  V4 up = normalize(cross(right, camDir));
  V4 rayOrig = {cam->center[0], cam->center[1], cam->center[2], 0.0f};
  V4 rayDir = add(add(scale(up, y), scale(right, x)), camDir);
  V4 rayX = scale(scale(right, 2.0f * x), 1.0f / (float)width);
  V4 rayY = scale(scale(up, 2.0f * y), 1.0f / (float)height);
  memcpy(basis + 0, &rayOrig, 16);
  memcpy(basis + 4, &rayDir, 16);
  memcpy(basis + 8, &rayX, 16);
  memcpy(basis + 12, &rayY, 16);
  return RT_OK;
}

// transpose(view * proj) of CUDACamera::update (CUDACamera.cpp:245-266) with the
// float4x4 helpers of types/_cuda_float4x4.h (rotation about an axis :323-350,
// perspective :398-410, lookAt :412-426, multiply :142-167): 4-wide dot
// products summed left to right, normalize = v * (1 / sqrtf(dot(v, v))).
extern "C" rt_status rt_camera_view_dir(const rt_camera* cam, const float target[3], float dir[3]) {
  if (!cam || !target || !dir) return RT_ERR_INVALID_ARGUMENT;
  const float dx = target[0] - cam->center[0], dy = target[1] - cam->center[1], dz = target[2] - cam->center[2];
  const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
  dir[0] = dx * inv; dir[1] = dy * inv; dir[2] = dz * inv;
  return RT_OK;
}

extern "C" rt_status rt_raster_matrix(const rt_camera* cam, const float dir[3], float m[16]) {
  if (!cam || !dir || !m) return RT_ERR_INVALID_ARGUMENT;
  const float dx = dir[0], dy = dir[1], dz = dir[2];
  const V4 eye = {cam->center[0], cam->center[1], cam->center[2], 0.0f};
  const V4 at = {cam->center[0] + dx * 4999.999f, cam->center[1] + dy * 4999.999f, cam->center[2] + dz * 4999.999f, 0.0f};
  float nx = dx, ny = 0.0f, nz = dy;  // the reference's roll axis (dir.x, 0, dir.y)
  const float ninv = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
  nx = nx * ninv; ny = ny * ninv; nz = nz * ninv;
  const float u = cosf(cam->angle[2]), v = sinf(cam->angle[2]), w = 1.0f - u;
  const V4 r0 = {w * nx * nx + u, w * nx * ny - v * nz, w * nx * nz + v * ny, 0.0f};
  const V4 r1 = {w * ny * nx + v * nz, w * ny * ny + u, w * ny * nz - v * nx, 0.0f};
  const V4 r2 = {w * nz * nx - v * ny, w * nz * ny + v * nx, w * nz * nz + u, 0.0f};
  const V4 r3 = {0.0f, 0.0f, 0.0f, 1.0f};
  const V4 up0 = {0.0f, 1.0f, 0.0f, 1.0f};
  const V4 up = {dot(r0, up0), dot(r1, up0), dot(r2, up0), dot(r3, up0)};
  const V4 za = normalize({at.x - eye.x, at.y - eye.y, at.z - eye.z, at.w - eye.w});
  const V4 xa = normalize(cross(up, za));
  const V4 ya = cross(za, xa);
  const V4 view[4] = {{xa.x, ya.x, za.x, 0.0f}, {xa.y, ya.y, za.y, 0.0f}, {xa.z, ya.z, za.z, 0.0f},
                      {-dot(xa, eye), -dot(ya, eye), -dot(za, eye), 1.0f}};
  const float zn = 1.000f, zf = 1999.999f;  // CUDACamera.cpp:34-35
  const float ys = 1.0f / tanf(cam->fov * 0.5f);
  const float xs = ys / cam->ratio;
  const float zfac = zf / (zf - zn);
  const float wfac = -zn * zfac;
  // columns of proj (rows of its transpose)
  const V4 pc[4] = {{xs, 0.0f, 0.0f, 0.0f}, {0.0f, ys, 0.0f, 0.0f}, {0.0f, 0.0f, zfac, wfac}, {0.0f, 0.0f, 1.0f, 0.0f}};
  // (view * proj)_ij = dot(view_i, proj column j); the kernel's matrix is its transpose
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) m[4 * j + i] = dot(view[i], pc[j]);
  return RT_OK;
}

extern "C" const char* rt_status_string(rt_status s) {
  switch (s) {
    case RT_OK: return "ok";
    case RT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case RT_ERR_NO_DEVICE: return "no CUDA device";
    case RT_ERR_CUDA: return "CUDA error";
    case RT_ERR_SCRATCH_TOO_SMALL: return "scratch buffer too small";
    case RT_ERR_CAPACITY: return "capacity exceeded";
    case RT_ERR_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

extern "C" uint32_t rt_version(void) { return 100u; }
extern "C" uint32_t rt_abi_version(void) { return RT_ABI_VERSION; }

namespace {
std::atomic<uint64_t> g_launches{0};
}
namespace rt {
void note_launch(uint32_t kernels) { g_launches.fetch_add(kernels, std::memory_order_relaxed); }
}  // namespace rt
extern "C" uint64_t rt_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
