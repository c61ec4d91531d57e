// raster_shim.hpp -- the pieces the reference's rasteriser and camera update
// (kernels/CUDA_rasterizeMeshTree.cu:77-225, CUDACamera.cpp:245-266) use that
// the prelude does not provide: int2, float2 helpers, make_float4(float3,
// float), and a CUDACamera with the members update() reads and writes.
// TEST INFRASTRUCTURE ONLY.
#pragma once
struct int2 { int x, y; };
static inline int2 make_int2(int x, int y) { return {x, y}; }
static inline float2 make_float2(int2 a) { return make_float2((float)a.x, (float)a.y); }
static inline float2 make_float2(float s) { return make_float2(s, s); }
static inline float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
static inline float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
static inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline void operator*=(float4& a, float s) { a.x *= s; a.y *= s; a.z *= s; a.w *= s; }
using std::max;
using std::min;
