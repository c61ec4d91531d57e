// rt_trace.cu -- primary rays, closest-hit traversal and diffuse bounce rays.
//
// Replaces CUDA_calcPrimaryRays (kernels/CUDA_calcPrimaryRays.cu:20-69) and
// CUDA_raytraceMeshTree (kernels/CUDA_raytraceMeshTree.cu:434-480).
//
// The traversal result is the closest (t, position) over every triangle that
// the reference's Moller-Trumbore test (:57-89, arithmetic pinned: no FMA
// contraction, IEEE division, 4-wide dot products) accepts with t < tmax. The
// result does not depend on the tree or on the visiting order because the box
// test is conservative: each box is padded by 2^-13 of its largest coordinate
// magnitude and a node is culled only when its entry distance exceeds
// 1.000122 x the best t. Node records are the reference's 32-byte bvnodes,
// loaded as two 128-bit read-only loads; triangles are read from the build's
// position-ordered {v0, e1, e2} stream (48 bytes, three 128-bit loads), so a
// leaf's triangles are contiguous.
#include "rt_common.cuh"

namespace rt {
namespace {

constexpr int kStack = 64;
constexpr float kBoxPad = 1.220703125e-4f;      // 2^-13
constexpr float kCullSlack = 1.0001220703125f;  // 1 + 2^-13

struct TraceArgs {
  const uint4* nodes;
  const float4* tris;
  const float4* verts;
  const uint4* faces;
  const uint32_t* indices;
  const float4* orig;
  const float4* dir;
  const float* tmax;
  uint32_t ray_count;
  uint32_t id_mode;
  int32_t* hit_id;
  float* hit_t;
  float2* hit_uv;
  uint32_t* visits;
  uint32_t* tests;
  uint32_t* err;
};

__device__ __forceinline__ float fix_dir(float c) { return fabsf(c) < 1e-20f ? copysignf(1e-20f, c) : c; }

// Moller-Trumbore of kernels/CUDA_raytraceMeshTree.cu:57-89; zu / zv are the
// (ray.w * 0) products of the 4-wide dot products (they only fix the sign of a
// zero sum).
__device__ __forceinline__ bool mt_test(const float4& o, const float4& d, float zu, float zv, const float4& v0, const float4& e1,
                                        const float4& e2, float& t, float& u, float& v) {
  const float px = d.y * e2.z - d.z * e2.y;
  const float py = d.z * e2.x - d.x * e2.z;
  const float pz = d.x * e2.y - d.y * e2.x;
  const float det = ((e1.x * px + e1.y * py) + e1.z * pz) + 0.0f;
  if (det > -0.000001f && det < 0.000001f) return false;
  const float inv = 1.0f / det;
  const float tx = o.x - v0.x, ty = o.y - v0.y, tz = o.z - v0.z;
  u = (((tx * px + ty * py) + tz * pz) + zu) * inv;
  if (u < 0.0f || u > 1.0f) return false;
  const float qx = ty * e1.z - tz * e1.y;
  const float qy = tz * e1.x - tx * e1.z;
  const float qz = tx * e1.y - ty * e1.x;
  v = (((d.x * qx + d.y * qy) + d.z * qz) + zv) * inv;
  if (v < 0.0f || u + v > 1.0f) return false;
  t = (((e2.x * qx + e2.y * qy) + e2.z * qz) + 0.0f) * inv;
  return t >= 0.0f;
}

__device__ __forceinline__ bool box_test(float bx0, float by0, float bz0, float bx1, float by1, float bz1, const float4& o,
                                         float ix, float iy, float iz, float tbest) {
  float px = fmax_sel(fabsf(bx0), fabsf(bx1)) * kBoxPad;
  float py = fmax_sel(fabsf(by0), fabsf(by1)) * kBoxPad;
  float pz = fmax_sel(fabsf(bz0), fabsf(bz1)) * kBoxPad;
  float t0x = ((bx0 - px) - o.x) * ix, t1x = ((bx1 + px) - o.x) * ix;
  float t0y = ((by0 - py) - o.y) * iy, t1y = ((by1 + py) - o.y) * iy;
  float t0z = ((bz0 - pz) - o.z) * iz, t1z = ((bz1 + pz) - o.z) * iz;
  float tn = fmax_sel(fmax_sel(fmin_sel(t0x, t1x), fmin_sel(t0y, t1y)), fmin_sel(t0z, t1z));
  float tf = fmin_sel(fmin_sel(fmax_sel(t0x, t1x), fmax_sel(t0y, t1y)), fmax_sel(t0z, t1z));
  return tn <= tf && tf >= 0.0f && tn <= tbest * kCullSlack;
}

template <bool kTris, bool kCount>
__global__ __launch_bounds__(128) void k_trace(TraceArgs A) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.ray_count) return;
  const float4 o = ldg4(A.orig + r), d = ldg4(A.dir + r);
  const float tmax0 = A.tmax ? __ldg(A.tmax + r) : kHuge;
  int32_t best = -1;
  float bt = tmax0, bu = 0.0f, bv = 0.0f;
  uint32_t visits = 0, tests = 0;
  if (tmax0 > 0.0f) {
    const float ix = 1.0f / fix_dir(d.x), iy = 1.0f / fix_dir(d.y), iz = 1.0f / fix_dir(d.z);
    const float zu = o.w * 0.0f, zv = d.w * 0.0f;
    uint32_t stack[kStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const uint32_t nid = stack[--sp];
      const uint4 q0 = ldg4(A.nodes + 2 * (size_t)nid);
      const uint4 q1 = ldg4(A.nodes + 2 * (size_t)nid + 1);
      if (kCount) ++visits;
      if (q0.x & 1u) {
        const uint32_t first = q0.y, cnt = q0.x >> 1;
        for (uint32_t k = 0; k < cnt; ++k) {
          const uint32_t pos = first + k;
          float4 v0, e1, e2;
          if (kTris) {
            v0 = ldg4(A.tris + 3 * (size_t)pos);
            e1 = ldg4(A.tris + 3 * (size_t)pos + 1);
            e2 = ldg4(A.tris + 3 * (size_t)pos + 2);
          } else {
            const uint4 f = ldg4(A.faces + pos);
            v0 = ldg4(A.verts + f.x);
            const float4 v1 = ldg4(A.verts + f.y), v2 = ldg4(A.verts + f.z);
            e1 = make_float4(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z, 0.0f);
            e2 = make_float4(v2.x - v0.x, v2.y - v0.y, v2.z - v0.z, 0.0f);
          }
          if (kCount) ++tests;
          float t, u, v;
          if (!mt_test(o, d, zu, zv, v0, e1, e2, t, u, v)) continue;
          if (t < bt || (best >= 0 && t == bt && (int32_t)pos < best)) {
            best = (int32_t)pos; bt = t; bu = u; bv = v;
          }
        }
      } else {
        const float bx0 = __uint_as_float(q0.z), by0 = __uint_as_float(q0.w), bz0 = __uint_as_float(q1.x);
        const float bx1 = __uint_as_float(q1.y), by1 = __uint_as_float(q1.z), bz1 = __uint_as_float(q1.w);
        if (box_test(bx0, by0, bz0, bx1, by1, bz1, o, ix, iy, iz, bt)) {
          const uint32_t axis = (q0.x >> 1) & 3u;
          const float da = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
          const uint32_t c = q0.y;
          if (sp + 2 <= kStack) {
            stack[sp++] = da < 0.f ? c : c + 1;  // far
            stack[sp++] = da < 0.f ? c + 1 : c;  // near
          } else if (A.err) {
            atomicOr(A.err, (uint32_t)RT_DEVERR_STACK_OVERFLOW);
          }
        }
      }
    }
  }
  if (best >= 0) {
    A.hit_id[r] = A.id_mode == 1 ? (int32_t)__ldg(A.indices + best) : best;
    A.hit_t[r] = bt;
    A.hit_uv[r] = make_float2(bu, bv);
  } else {
    A.hit_id[r] = -1;
    A.hit_t[r] = tmax0;
    A.hit_uv[r] = make_float2(0.0f, 0.0f);
  }
  if (kCount) {
    if (A.visits) A.visits[r] = visits;
    if (A.tests) A.tests[r] = tests;
  }
}

// ----------------------------------------------------------------------------
// Traversal over the build's blob: two-child records (both children's padded
// boxes tested together, the nearer child first, the farther pushed with its
// entry distance so that it is dropped on pop once the best hit is closer),
// then inside a leaf one padded box per 8 consecutive triangles. Same
// conservative test and the same (t, position) rule as k_trace, so the hits
// are identical; only the work differs.
// Counters: visits = 32-byte box records read (a two-child record counts 2,
// a group box 1, a leaf-table entry 1), tests = triangles tested.
// ----------------------------------------------------------------------------
struct AccelArgs {
  const float4* tnodes;
  const uint4* leaves;
  const float4* groups;
  const uint32_t* hdr;
};

__device__ __forceinline__ bool slab2(const float4& mn, const float4& mx, const float4& o, float ix, float iy, float iz, float tbest,
                                      float& tn) {
  const float t0x = (mn.x - o.x) * ix, t1x = (mx.x - o.x) * ix;
  const float t0y = (mn.y - o.y) * iy, t1y = (mx.y - o.y) * iy;
  const float t0z = (mn.z - o.z) * iz, t1z = (mx.z - o.z) * iz;
  tn = fmax_sel(fmax_sel(fmin_sel(t0x, t1x), fmin_sel(t0y, t1y)), fmin_sel(t0z, t1z));
  const float tf = fmin_sel(fmin_sel(fmax_sel(t0x, t1x), fmax_sel(t0y, t1y)), fmax_sel(t0z, t1z));
  return tn <= tf && tf >= 0.0f && tn <= tbest * kCullSlack;
}

template <bool kCount>
__global__ __launch_bounds__(128) void k_trace_accel(TraceArgs A, AccelArgs C) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.ray_count) return;
  const float4 o = ldg4(A.orig + r), d = ldg4(A.dir + r);
  const float tmax0 = A.tmax ? __ldg(A.tmax + r) : kHuge;
  int32_t best = -1;
  float bt = tmax0, bu = 0.0f, bv = 0.0f;
  uint32_t visits = 0, tests = 0;
  if (tmax0 > 0.0f) {
    const float ix = 1.0f / fix_dir(d.x), iy = 1.0f / fix_dir(d.y), iz = 1.0f / fix_dir(d.z);
    const float zu = o.w * 0.0f, zv = d.w * 0.0f;
    uint32_t st_ref[kStack];
    float st_t[kStack];
    int sp = 0;
    uint32_t ref = __ldg(C.hdr);
    for (;;) {
      if (ref & 0x80000000u) {
        // leaf
        const uint4 L = __ldg(C.leaves + (~ref));
        if (kCount) ++visits;
        const uint32_t first = L.x, cnt = L.y, gbase = L.z;
        for (uint32_t g = 0; g * 8 < cnt; ++g) {
          const float4 gmn = ldg4(C.groups + 2 * ((size_t)gbase + g));
          const float4 gmx = ldg4(C.groups + 2 * ((size_t)gbase + g) + 1);
          if (kCount) ++visits;
          float tg;
          if (!slab2(gmn, gmx, o, ix, iy, iz, bt, tg)) continue;
          const uint32_t kend = min(cnt, g * 8 + 8);
          for (uint32_t k = g * 8; k < kend; ++k) {
            const uint32_t pos = first + k;
            const float4 v0 = ldg4(A.tris + 3 * (size_t)pos);
            const float4 e1 = ldg4(A.tris + 3 * (size_t)pos + 1);
            const float4 e2 = ldg4(A.tris + 3 * (size_t)pos + 2);
            if (kCount) ++tests;
            float t, u, v;
            if (!mt_test(o, d, zu, zv, v0, e1, e2, t, u, v)) continue;
            if (t < bt || (best >= 0 && t == bt && (int32_t)pos < best)) {
              best = (int32_t)pos; bt = t; bu = u; bv = v;
            }
          }
        }
      } else {
        const float4* tn = C.tnodes + 4 * (size_t)ref;
        const float4 a0 = ldg4(tn), a1 = ldg4(tn + 1), b0 = ldg4(tn + 2), b1 = ldg4(tn + 3);
        if (kCount) visits += 2;
        float ta, tb;
        const bool ha = slab2(a0, a1, o, ix, iy, iz, bt, ta);
        const bool hb = slab2(b0, b1, o, ix, iy, iz, bt, tb);
        const uint32_t ra = __float_as_uint(a0.w), rb = __float_as_uint(b0.w);
        if (ha && hb) {
          const bool a_first = ta <= tb;
          if (sp < kStack) {
            st_ref[sp] = a_first ? rb : ra;
            st_t[sp] = a_first ? tb : ta;
            ++sp;
          } else if (A.err) {
            atomicOr(A.err, (uint32_t)RT_DEVERR_STACK_OVERFLOW);
          }
          ref = a_first ? ra : rb;
          continue;
        }
        if (ha) { ref = ra; continue; }
        if (hb) { ref = rb; continue; }
      }
      // pop the next subtree whose entry is still within reach
      bool found = false;
      while (sp > 0) {
        --sp;
        if (st_t[sp] <= bt * kCullSlack) { ref = st_ref[sp]; found = true; break; }
      }
      if (!found) break;
    }
  }
  if (best >= 0) {
    A.hit_id[r] = A.id_mode == 1 ? (int32_t)__ldg(A.indices + best) : best;
    A.hit_t[r] = bt;
    A.hit_uv[r] = make_float2(bu, bv);
  } else {
    A.hit_id[r] = -1;
    A.hit_t[r] = tmax0;
    A.hit_uv[r] = make_float2(0.0f, 0.0f);
  }
  if (kCount) {
    if (A.visits) A.visits[r] = visits;
    if (A.tests) A.tests[r] = tests;
  }
}

// kernels/CUDA_calcPrimaryRays.cu:20-32
__global__ __launch_bounds__(256) void k_primary(float4 ro, float4 rd, float4 rx, float4 ry, uint32_t w, uint32_t h,
                                                 float4* __restrict__ orig, float4* __restrict__ dir) {
  const size_t total = (size_t)w * h;
  for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < total; n += (size_t)gridDim.x * blockDim.x) {
    const float x = (float)(uint32_t)(n % w), y = (float)(uint32_t)(n / w);
    orig[n] = ro;
    dir[n] = make_float4((rd.x - x * rx.x) - y * ry.x, (rd.y - x * rx.y) - y * ry.y, (rd.z - x * rx.z) - y * ry.z,
                         (rd.w - x * rx.w) - y * ry.w);
  }
}

// PCG-XSH-RR 64/32 (O'Neill), pcg32_srandom_r / pcg32_random_r.
struct Pcg {
  uint64_t state, inc;
  __device__ __forceinline__ uint32_t next() {
    uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31u));
  }
  __device__ __forceinline__ void seed(uint64_t initstate, uint64_t initseq) {
    state = 0u;
    inc = (initseq << 1u) | 1u;
    next();
    state += initstate;
    next();
  }
};

__global__ __launch_bounds__(256) void k_bounce(const float4* __restrict__ tris, const float4* __restrict__ orig,
                                               const float4* __restrict__ dir, const int32_t* __restrict__ hit_pos,
                                               const float* __restrict__ hit_t, uint32_t count, uint64_t seed,
                                               float4* __restrict__ orig_out, float4* __restrict__ dir_out, float* __restrict__ tmax_out) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < count; r += gridDim.x * blockDim.x) {
    const int32_t pos = hit_pos[r];
    if (pos < 0) {
      orig_out[r] = make_float4(0.f, 0.f, 0.f, 0.f);
      dir_out[r] = make_float4(0.f, 0.f, 0.f, 0.f);
      tmax_out[r] = -1.0f;
      continue;
    }
    const float4 o = orig[r], d = dir[r];
    const float t = hit_t[r];
    const float4 e1 = ldg4(tris + 3 * (size_t)pos + 1), e2 = ldg4(tris + 3 * (size_t)pos + 2);
    float nx = e1.y * e2.z - e1.z * e2.y, ny = e1.z * e2.x - e1.x * e2.z, nz = e1.x * e2.y - e1.y * e2.x;
    const float inv = 1.0f / sqrtf((nx * nx + ny * ny) + nz * nz);
    nx = nx * inv; ny = ny * inv; nz = nz * inv;
    if ((nx * d.x + ny * d.y) + nz * d.z > 0.0f) { nx = -nx; ny = -ny; nz = -nz; }
    const float px = o.x + t * d.x, py = o.y + t * d.y, pz = o.z + t * d.z;
    const float eps = 1e-4f;
    Pcg g;
    g.seed(seed, (uint64_t)r);
    float a = 0.0f, b = 0.0f;
    for (int it = 0; it < 64; ++it) {
      const float u1 = (float)(g.next() >> 8) * 5.9604644775390625e-8f;
      const float u2 = (float)(g.next() >> 8) * 5.9604644775390625e-8f;
      const float aa = 2.0f * u1 - 1.0f, bb = 2.0f * u2 - 1.0f;
      if (aa * aa + bb * bb < 1.0f) { a = aa; b = bb; break; }
    }
    const float c = sqrtf(1.0f - (a * a + b * b));
    const float sgn = copysignf(1.0f, nz);
    const float A = -1.0f / (sgn + nz);
    const float B = nx * ny * A;
    const float t1x = 1.0f + sgn * nx * nx * A, t1y = sgn * B, t1z = -sgn * nx;
    const float t2x = B, t2y = sgn + ny * ny * A, t2z = -ny;
    orig_out[r] = make_float4(px + nx * eps, py + ny * eps, pz + nz * eps, 0.0f);
    dir_out[r] = make_float4(t1x * a + t2x * b + nx * c, t1y * a + t2y * b + ny * c, t1z * a + t2z * b + nz * c, 0.0f);
    tmax_out[r] = kHuge;
  }
}

int sms() {
  static int s = 0;
  if (!s) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
    if (s <= 0) s = 148;
  }
  return s;
}

}  // namespace
}  // namespace rt

using namespace rt;

extern "C" rt_status rt_device_check(void) {
  static int state = -1;  // -1 unknown, 0 absent, 1 present
  if (state < 0) {
    int count = 0;
    state = (cudaGetDeviceCount(&count) == cudaSuccess && count > 0) ? 1 : 0;
    if (!state) cudaGetLastError();
  }
  return state ? RT_OK : RT_ERR_NO_DEVICE;
}

extern "C" rt_status rt_trace_closest(const rt_trace_desc* d, rt_stream stream) {
  if (!d || !d->nodes || !d->orig || !d->dir || !d->hit_id || !d->hit_t || !d->hit_uv) return RT_ERR_INVALID_ARGUMENT;
  if (!d->tris && (!d->vertices || !d->faces)) return RT_ERR_INVALID_ARGUMENT;
  if (d->id_mode == 1 && !d->indices) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (d->ray_count == 0) return RT_OK;
  TraceArgs A;
  A.nodes = (const uint4*)d->nodes; A.tris = (const float4*)d->tris; A.verts = (const float4*)d->vertices;
  A.faces = (const uint4*)d->faces; A.indices = d->indices; A.orig = (const float4*)d->orig; A.dir = (const float4*)d->dir;
  A.tmax = d->tmax; A.ray_count = d->ray_count; A.id_mode = d->id_mode; A.hit_id = d->hit_id; A.hit_t = d->hit_t;
  A.hit_uv = (float2*)d->hit_uv; A.visits = d->ray_visits; A.tests = d->ray_tests; A.err = d->error_word;
  const bool count = d->ray_visits || d->ray_tests;
  const uint32_t blocks = (d->ray_count + 127) / 128;
  cudaStream_t st = (cudaStream_t)stream;
  if (d->accel) {
    if (!d->tris) return RT_ERR_INVALID_ARGUMENT;
    // blob layout of rt_lbvh_build: header (256 B), records, leaf table, group boxes
    const size_t n = d->face_count_hint;
    AccelArgs C;
    Carve c((void*)d->accel, ~(size_t)0);
    C.hdr = c.take<uint32_t>(64);
    C.tnodes = c.take<float4>(4 * n);
    C.leaves = c.take<uint4>(n);
    C.groups = c.take<float4>(2 * (n / 8 + n + 1));
    if (count) k_trace_accel<true><<<blocks, 128, 0, st>>>(A, C);
    else k_trace_accel<false><<<blocks, 128, 0, st>>>(A, C);
    note_launch();
    RT_CHECK_LAUNCH();
    return RT_OK;
  }
  if (d->tris) {
    if (count) k_trace<true, true><<<blocks, 128, 0, st>>>(A);
    else k_trace<true, false><<<blocks, 128, 0, st>>>(A);
  } else {
    if (count) k_trace<false, true><<<blocks, 128, 0, st>>>(A);
    else k_trace<false, false><<<blocks, 128, 0, st>>>(A);
  }
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_primary_rays(const rt_camera* cam, uint32_t w, uint32_t h, float* orig, float* dir, rt_stream stream) {
  if (!cam || !orig || !dir || w == 0 || h == 0) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  float b[16];
  rt_status s = rt_camera_basis(cam, w, h, b);
  if (s != RT_OK) return s;
  const size_t total = (size_t)w * h;
  const uint32_t blocks = (uint32_t)hmin<size_t>((total + 255) / 256, (size_t)sms() * 16);
  k_primary<<<blocks, 256, 0, (cudaStream_t)stream>>>(make_float4(b[0], b[1], b[2], b[3]), make_float4(b[4], b[5], b[6], b[7]),
                                                      make_float4(b[8], b[9], b[10], b[11]), make_float4(b[12], b[13], b[14], b[15]), w, h,
                                                      (float4*)orig, (float4*)dir);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_bounce_rays(const float* tris, const float* orig, const float* dir, const int32_t* hit_pos, const float* hit_t,
                                    uint32_t count, uint64_t seed, float* orig_out, float* dir_out, float* tmax_out, rt_stream stream) {
  if (count == 0) return RT_OK;
  if (!tris || !orig || !dir || !hit_pos || !hit_t || !orig_out || !dir_out || !tmax_out) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  const uint32_t blocks = (uint32_t)hmin<size_t>((count + 255) / 256, (size_t)sms() * 16);
  k_bounce<<<blocks, 256, 0, (cudaStream_t)stream>>>((const float4*)tris, (const float4*)orig, (const float4*)dir, hit_pos, hit_t, count,
                                                     seed, (float4*)orig_out, (float4*)dir_out, tmax_out);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}
