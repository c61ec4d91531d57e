// prelude.hpp -- host-side stand-ins for the CUDA-1.x facilities that the
// reference's kernels use, so that selected functions of the reference source
// can be compiled with g++ and executed on the CPU, one simulated thread at a
// time. TEST INFRASTRUCTURE ONLY: used by oracle/build_ref.sh to build the
// checker libraries under oracle/_ref/. Nothing here is product code.
//
// What is emulated:
//  * texture<T,1,...> references bound to host arrays and tex1Dfetch;
//  * blockIdx / blockDim / threadIdx as globals set by the driver loops;
//  * __global__/__device__/__host__/__shared__ qualifiers (shared arrays become
//    function statics, which is exact for kernels without __syncthreads when
//    threads run one after another);
//  * atomicAdd (sequential);
//  * the vector helpers of the reference's types/ headers that the extracted
//    functions call (restated; the reference headers pull in unvendored files);
//  * bvnode / aabox with the field layout of CUDANode.h:20-50 / CUDABox.h:17-148;
//  * cudaMallocHost/cudaMemcpy/cudaFreeHost on host memory. Host allocations
//    are padded with 0xFFFFFFFF words so that a read past the end of the split
//    list (which the reference's recursion can do) sees "no split".
#pragma once
#include <math.h>
#include <algorithm>
#include <numeric>
#include <vector>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

// CUDA vector types (vector_types.h layout), defined here so that no CUDA
// runtime header is needed.
struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct __attribute__((aligned(16))) float4 { float x, y, z, w; };
struct __attribute__((aligned(16))) uint4 { unsigned x, y, z, w; };
static inline float2 make_float2(float x, float y) { return {x, y}; }
static inline float3 make_float3(float x, float y, float z) { return {x, y, z}; }
static inline float4 make_float4(float x, float y, float z, float w) { return {x, y, z, w}; }

typedef unsigned int uint;

#define __global__
#define __device__
#define __host__
#define __shared__ static
#ifndef __inline__
#define __inline__ inline
#endif
#define CUDART_NORM_HUGE_F 3.402823466e+38f

struct ShimDim3 { unsigned x, y, z; };
#ifdef SHIM_THREADED
// kernels with __syncthreads run their 32 threads as real host threads
// (sah_shim.hpp); each has its own threadIdx
static ShimDim3 blockIdx, blockDim;
static thread_local ShimDim3 threadIdx;
#else
static ShimDim3 blockIdx, blockDim, threadIdx;
#endif

enum cudaTextureReadMode { cudaReadModeElementType = 0 };
template <typename T, int dim, int mode>
struct texture { const T* ptr = nullptr; };
template <typename T, int dim, int mode>
static inline T tex1Dfetch(const texture<T, dim, mode>& t, int i) { return t.ptr[i]; }

static inline uint atomicAdd(uint* p, uint v) { uint old = *p; *p = old + v; return old; }

enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3 };
static const size_t kShimPadWords = 1u << 16;
static inline int cudaMallocHost(void** p, size_t bytes) {
  size_t total = bytes + kShimPadWords * 4;
  *p = malloc(total);
  memset(*p, 0xFF, total);
  return 0;
}
static inline int cudaFreeHost(void* p) { free(p); return 0; }
static inline int cudaMemcpy(void* d, const void* s, size_t b, cudaMemcpyKind) { memmove(d, s, b); return 0; }

// ---- vector helpers (semantics of types/_cuda_float*.h; host rsqrtf = 1/sqrtf,
// device fminf/fmaxf = IEEE minNum/maxNum as C's fminf/fmaxf)
static inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
static inline float3 make_float3(float s) { return make_float3(s, s, s); }
static inline float3 make_float3(float4 a) { return make_float3(a.x, a.y, a.z); }
static inline float4 make_float4(float s) { return make_float4(s, s, s, s); }
static inline float4 make_float4(float3 a) { return make_float4(a.x, a.y, a.z, 0.0f); }
static inline float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline float4 operator-(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
static inline float4 operator*(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
static inline float4 operator*(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
static inline float4 operator*(float s, float4 a) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
static inline float4 operator/(float4 a, float s) { float inv = 1.0f / s; return a * inv; }
static inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
static inline float4 normalize(float4 v) { float inv_len = rsqrtf(dot(v, v)); return v * inv_len; }
static inline float4 cross(float4 a, float4 b) {
  float4 r;
  r.x = a.y * b.z - a.z * b.y; r.y = a.z * b.x - a.x * b.z; r.z = a.x * b.y - a.y * b.x; r.w = 0.0f;
  return r;
}
static inline float4 fminf(float4 a, float4 b) { return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w)); }
static inline float4 fmaxf(float4 a, float4 b) { return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w)); }
static inline float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
static inline float2 operator*(float s, float2 a) { return make_float2(a.x * s, a.y * s); }
static inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
static inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float3 normalize(float3 v) { float inv_len = rsqrtf(dot(v, v)); return v * inv_len; }
static inline float3 fminf(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
static inline float3 fmaxf(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

// Mixed float4 / float3 min and max: the float4 keeps its w (types/_cuda_float4.h),
// the float3 result drops the other's w (types/_cuda_float3.h).
static inline float4 fminf(float4 a, float3 b) { return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), a.w); }
static inline float4 fmaxf(float4 a, float3 b) { return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), a.w); }
static inline float3 fminf(float3 a, float4 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
static inline float3 fmaxf(float3 a, float4 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

namespace renderkit {
// bvnode: same members and bit layout as CUDANode.h:20-50.
struct __attribute__((aligned(16))) bvnode {
  union {
    int raw_data0;
    int raw_data1;
    struct { uint type : 1; uint axis : 2; uint child_id; } node;
    struct { uint type : 1; uint obj_count : 31; uint obj_id; } leaf;
  };
  float3 box_min;
  float3 box_max;
};
static inline bool isLeaf(const bvnode& b) { return b.leaf.type == 1; }
static inline bool isNode(const bvnode& b) { return b.node.type == 0; }
static inline void getObjects(const bvnode& b, int& id, int& count) { id = b.leaf.obj_id; count = b.leaf.obj_count; }
static inline void getChildren(const bvnode& b, const float4& dir, int& near_id, int& far_id) {
  int axis = (int)b.node.axis;
  bool neg = axis == 0 ? (dir.x < 0.f) : (axis == 1 ? (dir.y < 0.f) : (dir.z < 0.f));
  if (neg) { near_id = b.node.child_id + 1; far_id = b.node.child_id; }
  else { near_id = b.node.child_id; far_id = b.node.child_id + 1; }
}
// aabox: CUDABox.h:17-148 (the members used by the extracted kernels).
struct __attribute__((aligned(16))) aabox {
  float4 min, max;
  float getArea() const {
    float4 v = max - min;
    return 2.f * (v.x * v.y + v.x * v.z + v.y * v.z);
  }
  void reset() { min = make_float4(+CUDART_NORM_HUGE_F); max = make_float4(-CUDART_NORM_HUGE_F); }
  void reset(const float4& v) { min = v; max = v; }
  void reset(const float4& a, const float4& b) { min = a; max = b; }
  void reset(const float3& a, const float3& b) { min = make_float4(a); max = make_float4(b); }
  void merge(const aabox& b) { min = fminf(min, b.min); max = fmaxf(max, b.max); }
  void merge(const float4& v) { min = fminf(min, v); max = fmaxf(max, v); }
  void merge(const float4& a, const float4& b) { min = fminf(min, a); max = fmaxf(max, b); }
  void merge(const float3& a, const float3& b) { min = fminf(min, a); max = fmaxf(max, b); }
};
}  // namespace renderkit
using namespace renderkit;

static_assert(sizeof(renderkit::bvnode) == 32, "bvnode layout");

#define REF_API extern "C" __attribute__((visibility("default")))
