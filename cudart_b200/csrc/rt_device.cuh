// rt_device.cuh -- device helpers shared by the single-mesh and batched
// build and traversal kernels (one definition of every pinned computation).
#pragma once
#include "rt_common.cuh"

namespace rt {

constexpr uint32_t kNone = 0xFFFFFFFFu;

// float -> uint with the saturating round-toward-zero rule of cvt.rzi.u32.f32.
__device__ __forceinline__ uint32_t f2u_sat(float x) { return __float2uint_rz(x); }

__device__ __forceinline__ uint32_t spread_code(uint32_t qx, uint32_t qy, uint32_t qz, int layout) {
  uint32_t code = 0;
  if (layout == 30) {
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      code |= ((qz >> k) & 1u) << (3 * k + 2);
      code |= ((qy >> k) & 1u) << (3 * k + 3);
      code |= ((qx >> k) & 1u) << (3 * k + 4);
    }
  } else {
    // kernels/CUDA_buildMeshTreeLBVH.cu:138-169: bit 3k = y_k, 3k+1 = x_k, 3k+2 = z_k
#pragma unroll
    for (int k = 0; k < 11; ++k) {
      code |= ((qy >> k) & 1u) << (3 * k + 0);
      code |= ((qx >> k) & 1u) << (3 * k + 1);
      if (k < 10) code |= ((qz >> k) & 1u) << (3 * k + 2);
    }
  }
  return code;
}

// Leaves of the median subtree of a range of s faces entered from a leaf
// (s > max_leaf): recursive floor/ceil halving, a node of fewer than max_leaf
// faces is a leaf (kernels/CUDA_buildMeshTreeLBVH.cu:314-339). The sizes at
// depth j are floor(s/2^j) and floor(s/2^j)+1, the latter s mod 2^j times.
__device__ __forceinline__ uint32_t median_leaves(uint32_t s, uint32_t maxl) {
  if (s < maxl) return 1u;
  uint32_t j0 = 0;
  while ((s >> j0) >= maxl) ++j0;
  uint32_t q0 = s >> j0;
  uint32_t r = s & ((1u << j0) - 1u);
  return (1u << j0) + ((q0 + 1u == maxl) ? r : 0u);
}
__device__ __forceinline__ uint32_t median_depth(uint32_t s, uint32_t maxl) {
  if (s < maxl) return 0u;
  uint32_t j0 = 0;
  while ((s >> j0) >= maxl) ++j0;
  uint32_t q0 = s >> j0;
  uint32_t r = s & ((1u << j0) - 1u);
  return j0 + ((q0 + 1u == maxl && r) ? 1u : 0u);
}

template <int NT>
__device__ __forceinline__ uint32_t block_excl_scan_nt(uint32_t v, uint32_t* s_warp, uint32_t& total) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < W ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < W) s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t prefix = warp ? s_warp[warp - 1] : 0u;
  total = s_warp[W - 1];
  __syncthreads();
  return prefix + x - v;
}

// First index j >= start[L] of C with C[j] > a, scanning the level lists in
// order (each is ascending). Returns S when none.
__device__ __forceinline__ uint32_t split_scan(const uint32_t* __restrict__ C, const uint32_t* s_start, uint32_t L, uint32_t a) {
  for (uint32_t l = L; l < 32; ++l) {
    uint32_t st = s_start[l], en = s_start[l + 1];
    if (st < en && __ldg(C + en - 1) > a) {
      uint32_t lo = st, hi = en - 1;
      while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(C + mid) > a) hi = mid; else lo = mid + 1;
      }
      return lo;
    }
  }
  return s_start[32];
}

constexpr float kAccelPad = 1.220703125e-4f;  // 2^-13 of the largest coordinate magnitude per axis

// Box padded for the traversal's conservative slab test.
__device__ __forceinline__ void pad_box(float3& mn, float3& mx) {
  const float px = fmax_sel(fabsf(mn.x), fabsf(mx.x)) * kAccelPad;
  const float py = fmax_sel(fabsf(mn.y), fabsf(mx.y)) * kAccelPad;
  const float pz = fmax_sel(fabsf(mn.z), fabsf(mx.z)) * kAccelPad;
  mn.x = mn.x - px; mn.y = mn.y - py; mn.z = mn.z - pz;
  mx.x = mx.x + px; mx.y = mx.y + py; mx.z = mx.z + pz;
}

__device__ __forceinline__ void write_box(uint32_t* node, float3 mn, float3 mx) {
  float* f = (float*)node;
  __stcg(f + 2, mn.x); __stcg(f + 3, mn.y); __stcg(f + 4, mn.z);
  __stcg(f + 5, mx.x); __stcg(f + 6, mx.y); __stcg(f + 7, mx.z);
}

// Two-child traversal records, indexed by pre-order rank (internal node p
// with left child c has rank (c - 1) / 2): both children's padded boxes and
// references (rank for an internal child, ~leaf index for a leaf child).
// One internal node's two-child record.
__device__ __forceinline__ void accel_node(const uint32_t* __restrict__ nodes, const uint32_t* __restrict__ leaf_lambda,
                                           float4* __restrict__ tnodes, const uint32_t p) {
  const uint2 w = *(const uint2*)(nodes + 8 * (size_t)p);
  if (w.x & 1u) return;
  const uint32_t rank = (w.y - 1u) >> 1;
  float4 out[4];
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const uint32_t c = w.y + side;
    const uint32_t* cn = nodes + 8 * (size_t)c;
    const uint32_t cw0 = cn[0], cw1 = cn[1];
    float3 mn = make_float3(__uint_as_float(cn[2]), __uint_as_float(cn[3]), __uint_as_float(cn[4]));
    float3 mx = make_float3(__uint_as_float(cn[5]), __uint_as_float(cn[6]), __uint_as_float(cn[7]));
    pad_box(mn, mx);
    const uint32_t ref = (cw0 & 1u) ? ~leaf_lambda[c] : ((cw1 - 1u) >> 1);
    out[2 * side] = make_float4(mn.x, mn.y, mn.z, __uint_as_float(ref));
    out[2 * side + 1] = make_float4(mx.x, mx.y, mx.z, 0.0f);
  }
  float4* dst = tnodes + 4 * (size_t)rank;
  dst[0] = out[0]; dst[1] = out[1]; dst[2] = out[2]; dst[3] = out[3];
}

// ---------------------------------------------------------------------------
// Cluster tree: a second traversal tree in the blob, independent of the node
// tree, whose leaves hold at most `leaf_max` (1..8, default 3) triangles. It is
// the binary radix tree of the mesh's sorted keys (Morton code, position)
// built bottom-up (rt_clusters.cu), cut at subtrees of at most leaf_max
// positions (a "cluster": a contiguous run of positions) and stored as 4-wide
// records. Internal node p of the radix tree (0 <= p < n - 1) is the split
// between positions p and p + 1; its record, at record index p, holds the
// boxes of up to four children: each child of p that is a cluster, or else
// that child's two children. The root's record is at the index in the header;
// a mesh whose root is itself a cluster (n <= leaf_max) gets a one-slot record
// at index n - 1. Records of mesh m sit at F_m + index (F_m = its first face).
// A record (128 B) is eight float4: min x, min y, min z, max x, max y, max z of
// the four slots (component k = slot k), the four slot references and a spare.
// A reference is a record index, or kClusterLeaf | (count - 1) << 28 | first
// for the positions first .. first + count - 1; an unused slot has kNoChild
// and NaN bounds, which every slab comparison rejects.
// ---------------------------------------------------------------------------
constexpr uint32_t kClusterLeaf = 0x80000000u;
constexpr uint32_t kClusterFirstMask = 0x0FFFFFFFu;  // meshes of fewer than 2^28 positions
constexpr uint32_t kClusterLeafMax = 8;
constexpr uint32_t kClusterLeafDefault = 3;
// Header words (per mesh, inside the blob header of 64 words) describing the cluster tree. Every build clears
// the valid word (in the kernel that writes the node records' header words); the cluster build sets it last.
constexpr int kHdrClusterValid = 16;  // 1 once the build wrote the cluster tree for this mesh, else 0
constexpr int kHdrClusterN = 17;      // positions n
constexpr int kHdrClusterRoot = 18;   // record index of the root
__host__ __device__ __forceinline__ uint32_t cluster_leaf_ref(uint32_t first, uint32_t count) {
  return kClusterLeaf | ((count - 1u) << 28) | first;
}
// The build works in chunks of kClusterChunk positions (one CTA each, never across meshes; mesh m's chunks start
// at chunk cluster_chunk_base(F_m, m)); each chunk leaves at most two nodes for the global pass (`frontier`).
constexpr uint32_t kClusterChunk = 512;
__host__ __device__ __forceinline__ uint32_t cluster_chunk_base(uint32_t F, uint32_t m) { return F / kClusterChunk + m; }
__host__ __device__ __forceinline__ uint32_t cluster_chunks(uint32_t N, uint32_t M) { return N / kClusterChunk + M + 1; }
// Build temporaries (per position of all meshes, indexed by F_m + boundary): the arrival word of each internal
// node, its two child references (kClusterLeaf | position for a position) and the padded boxes of those two
// children, the range of each node the global pass completes (first, last + 1); per chunk the (at most two)
// frontier nodes, their boxes and the nodes their climbs completed.
struct ClusterTemps {
  uint32_t* other;
  uint32_t* child;
  float4* cbox;     // [4 N]: box of child k of boundary b at 4 b + 2 k (min, max)
  uint2* prange;
  uint4* frontier;  // [2 chunks]: (reference, first, last, 1) of a node whose parent lies outside its chunk, else zero
  float4* fbox;     // [4 chunks]: the frontier nodes' boxes (min, max)
  uint32_t* chain;  // [2 chunks x kClusterChain]: the nodes each frontier node's climb completed, then their count
};
constexpr uint32_t kClusterChain = 64;  // a climb completes at most one node per bit of the 64-bit keys
inline void carve_cluster_temps(Carve& c, ClusterTemps& T, size_t N, size_t M) {
  const size_t chunks = N / kClusterChunk + M + 1;
  T.other = c.take<uint32_t>(N);
  T.child = c.take<uint32_t>(2 * N);
  T.cbox = c.take<float4>(4 * N);
  T.prange = c.take<uint2>(N);
  T.frontier = c.take<uint4>(2 * chunks);
  T.fbox = c.take<float4>(4 * chunks);
  T.chain = c.take<uint32_t>(2 * chunks * (kClusterChain + 1));
}

// Traversal blob: header (256 B), internal-node records (64 B, <= N - 1),
// leaf table (16 B, <= N), group boxes (32 B, <= N/8 + N), 4-wide records
// (128 B, <= N - 1, see wide_node) and the cluster tree (128 B records, <= N).
struct AccelLayout {
  uint32_t* hdr;
  float4* tnodes;
  uint4* leaves;
  float4* groups;
  float4* wide;
  float4* crec;
};
inline size_t carve_accel(Carve& c, AccelLayout& A, uint32_t n) {
  A.hdr = c.take<uint32_t>(64);
  A.tnodes = c.take<float4>(4 * (size_t)n);
  A.leaves = c.take<uint4>(n);
  A.groups = c.take<float4>(2 * ((size_t)n / 8 + n + 1));
  A.wide = c.take<float4>(8 * (size_t)n);
  A.crec = c.take<float4>(8 * (size_t)n);
  return c.off + 256;
}

// 4-wide record of binary record r: r's two children, each internal child
// replaced by that child's two children (their padded boxes come from the
// child's own record). Layout (8 x float4): min x / y / z of the 4 children,
// max x / y / z, child references (as in the two-child records; kNoChild for an
// unused slot), and one spare. Every record gets one; a walk that starts at
// the root only reaches those of even depth.
constexpr uint32_t kNoChild = 0x7FFFFFFEu;
__device__ __forceinline__ void wide_node(const float4* __restrict__ tnodes, float4* __restrict__ wide, uint32_t r) {
  const float4* rec = tnodes + 4 * (size_t)r;
  float mnx[4] = {0.f, 0.f, 0.f, 0.f}, mny[4] = {0.f, 0.f, 0.f, 0.f}, mnz[4] = {0.f, 0.f, 0.f, 0.f};
  float mxx[4] = {0.f, 0.f, 0.f, 0.f}, mxy[4] = {0.f, 0.f, 0.f, 0.f}, mxz[4] = {0.f, 0.f, 0.f, 0.f};
  uint32_t ref[4] = {kNoChild, kNoChild, kNoChild, kNoChild};
  int k = 0;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const float4 a0 = rec[2 * side], a1 = rec[2 * side + 1];
    const uint32_t c = __float_as_uint(a0.w);
    if (c & 0x80000000u) {
      mnx[k] = a0.x; mny[k] = a0.y; mnz[k] = a0.z; mxx[k] = a1.x; mxy[k] = a1.y; mxz[k] = a1.z; ref[k] = c;
      ++k;
    } else {
      const float4* cr = tnodes + 4 * (size_t)c;
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2) {
        const float4 b0 = cr[2 * s2], b1 = cr[2 * s2 + 1];
        mnx[k] = b0.x; mny[k] = b0.y; mnz[k] = b0.z; mxx[k] = b1.x; mxy[k] = b1.y; mxz[k] = b1.z; ref[k] = __float_as_uint(b0.w);
        ++k;
      }
    }
  }
  float4* w = wide + 8 * (size_t)r;
  w[0] = make_float4(mnx[0], mnx[1], mnx[2], mnx[3]);
  w[1] = make_float4(mny[0], mny[1], mny[2], mny[3]);
  w[2] = make_float4(mnz[0], mnz[1], mnz[2], mnz[3]);
  w[3] = make_float4(mxx[0], mxx[1], mxx[2], mxx[3]);
  w[4] = make_float4(mxy[0], mxy[1], mxy[2], mxy[3]);
  w[5] = make_float4(mxz[0], mxz[1], mxz[2], mxz[3]);
  w[6] = make_float4(__uint_as_float(ref[0]), __uint_as_float(ref[1]), __uint_as_float(ref[2]), __uint_as_float(ref[3]));
  w[7] = make_float4(0.f, 0.f, 0.f, 0.f);
}
// The two-child record and the 4-wide record of internal node p, both from the nodes (the same values as
// accel_node followed by wide_node, in one pass: a grandchild's padded box and reference are computed from its
// node as accel_node computes them for the child's record).
__device__ __forceinline__ void accel_wide_node(const uint32_t* __restrict__ nodes, const uint32_t* __restrict__ leaf_lambda,
                                                float4* __restrict__ tnodes, float4* __restrict__ wide, const uint32_t p) {
  const uint2 w = *(const uint2*)(nodes + 8 * (size_t)p);
  if (w.x & 1u) return;
  const uint32_t rank = (w.y - 1u) >> 1;
  // padded box and reference of node c, as a parent's record holds them
  auto child = [&](uint32_t c, float3& mn, float3& mx, uint32_t& ref, uint32_t& first_child) {
    const uint32_t* cn = nodes + 8 * (size_t)c;
    const uint32_t cw0 = cn[0], cw1 = cn[1];
    mn = make_float3(__uint_as_float(cn[2]), __uint_as_float(cn[3]), __uint_as_float(cn[4]));
    mx = make_float3(__uint_as_float(cn[5]), __uint_as_float(cn[6]), __uint_as_float(cn[7]));
    pad_box(mn, mx);
    const bool leaf = (cw0 & 1u) != 0;
    ref = leaf ? ~leaf_lambda[c] : ((cw1 - 1u) >> 1);
    first_child = leaf ? kNone : cw1;
  };
  float4 out[4];
  float mnx[4] = {0.f, 0.f, 0.f, 0.f}, mny[4] = {0.f, 0.f, 0.f, 0.f}, mnz[4] = {0.f, 0.f, 0.f, 0.f};
  float mxx[4] = {0.f, 0.f, 0.f, 0.f}, mxy[4] = {0.f, 0.f, 0.f, 0.f}, mxz[4] = {0.f, 0.f, 0.f, 0.f};
  uint32_t wref[4] = {kNoChild, kNoChild, kNoChild, kNoChild};
  int k = 0;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    float3 mn, mx;
    uint32_t ref, fc;
    child(w.y + side, mn, mx, ref, fc);
    out[2 * side] = make_float4(mn.x, mn.y, mn.z, __uint_as_float(ref));
    out[2 * side + 1] = make_float4(mx.x, mx.y, mx.z, 0.0f);
    if (fc == kNone) {
      mnx[k] = mn.x; mny[k] = mn.y; mnz[k] = mn.z; mxx[k] = mx.x; mxy[k] = mx.y; mxz[k] = mx.z; wref[k] = ref;
      ++k;
    } else {
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2) {
        float3 gmn, gmx;
        uint32_t gref, gfc;
        child(fc + s2, gmn, gmx, gref, gfc);
        mnx[k] = gmn.x; mny[k] = gmn.y; mnz[k] = gmn.z; mxx[k] = gmx.x; mxy[k] = gmx.y; mxz[k] = gmx.z; wref[k] = gref;
        ++k;
      }
    }
  }
  float4* dst = tnodes + 4 * (size_t)rank;
  dst[0] = out[0]; dst[1] = out[1]; dst[2] = out[2]; dst[3] = out[3];
  float4* wd = wide + 8 * (size_t)rank;
  wd[0] = make_float4(mnx[0], mnx[1], mnx[2], mnx[3]);
  wd[1] = make_float4(mny[0], mny[1], mny[2], mny[3]);
  wd[2] = make_float4(mnz[0], mnz[1], mnz[2], mnz[3]);
  wd[3] = make_float4(mxx[0], mxx[1], mxx[2], mxx[3]);
  wd[4] = make_float4(mxy[0], mxy[1], mxy[2], mxy[3]);
  wd[5] = make_float4(mxz[0], mxz[1], mxz[2], mxz[3]);
  wd[6] = make_float4(__uint_as_float(wref[0]), __uint_as_float(wref[1]), __uint_as_float(wref[2]), __uint_as_float(wref[3]));
  wd[7] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// All records of a blob whose header holds the leaf count (hdr[1]).
static __global__ __launch_bounds__(256) void k_wide_nodes(const float4* __restrict__ tnodes, const uint32_t* __restrict__ acc_hdr,
                                                    float4* __restrict__ wide) {
  const uint32_t leaves = acc_hdr[1];
  const uint32_t records = leaves ? leaves - 1 : 0;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < records; r += gridDim.x * blockDim.x) wide_node(tnodes, wide, r);
}

constexpr int kStack = 64;
constexpr float kBoxPad = 1.220703125e-4f;      // 2^-13
constexpr float kCullSlack = 1.0001220703125f;  // 1 + 2^-13

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

// Three-input min / max (one instruction each on sm_100).
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// Slab test of a padded box. `oi` is the ray origin scaled by the inverse
// direction (o.x * ix, o.y * iy, o.z * iz): each plane distance is one fused
// multiply-add, box * inv - origin * inv, whose error (the rounding of o * inv
// and of the result) is of the same order as that of (box - origin) * inv and
// is absorbed the same way by the 2^-13 padding and the cull slack.
__device__ __forceinline__ bool slab2(const float4& mn, const float4& mx, const float4& oi, float ix, float iy, float iz, float tbest,
                                      float& tn) {
  const float t0x = __fmaf_rn(mn.x, ix, -oi.x), t1x = __fmaf_rn(mx.x, ix, -oi.x);
  const float t0y = __fmaf_rn(mn.y, iy, -oi.y), t1y = __fmaf_rn(mx.y, iy, -oi.y);
  const float t0z = __fmaf_rn(mn.z, iz, -oi.z), t1z = __fmaf_rn(mx.z, iz, -oi.z);
  tn = max3f(fminf(t0x, t1x), fminf(t0y, t1y), fminf(t0z, t1z));
  const float tf = min3f(fmaxf(t0x, t1x), fmaxf(t0y, t1y), fmaxf(t0z, t1z));
  return tn <= tf && tf >= 0.0f && tn <= tbest * kCullSlack;
}
__device__ __forceinline__ float4 scaled_origin(const float4& o, float ix, float iy, float iz) {
  return make_float4(o.x * ix, o.y * iy, o.z * iz, 0.0f);
}

// One 4-wide record against a ray: entry distance of every child the ray
// enters within reach (+inf otherwise), children sorted nearest first
// (5-comparator network), references alongside.
__device__ __forceinline__ float f4c(const float4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }
__device__ __forceinline__ uint32_t u4c(const uint4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }
__device__ __forceinline__ void cswap_tr(float (&t)[4], uint32_t (&r)[4], int a, int b) {
  if (t[b] < t[a]) {
    const float tt = t[a]; t[a] = t[b]; t[b] = tt;
    const uint32_t rr = r[a]; r[a] = r[b]; r[b] = rr;
  }
}
// The test of a 4-wide record held in registers (w[0..5]: min x / y / z, max x / y / z of the 4 children;
// w[6]: their references): entry distances (INFINITY for a miss) and references, nearest first.
__device__ __forceinline__ void wide_test_regs(const float4 (&w)[8], const float4& oi, float ix, float iy, float iz, float tbest,
                                               uint32_t skip, float (&t)[4], uint32_t (&r)[4]) {
  const float4 w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3], w4 = w[4], w5 = w[5], wrf = w[6];
  const uint4 wr = make_uint4(__float_as_uint(wrf.x), __float_as_uint(wrf.y), __float_as_uint(wrf.z), __float_as_uint(wrf.w));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t rk = u4c(wr, k);
    float tn;
    const bool h = rk != kNoChild && rk != skip &&
                   slab2(make_float4(f4c(w0, k), f4c(w1, k), f4c(w2, k), 0.0f), make_float4(f4c(w3, k), f4c(w4, k), f4c(w5, k), 0.0f), oi,
                         ix, iy, iz, tbest, tn);
    t[k] = h ? tn : INFINITY;
    r[k] = rk;
  }
  cswap_tr(t, r, 0, 1);
  cswap_tr(t, r, 2, 3);
  cswap_tr(t, r, 0, 2);
  cswap_tr(t, r, 1, 3);
  cswap_tr(t, r, 1, 2);
}
__device__ __forceinline__ void wide_test(const float4* __restrict__ wn, const float4& oi, float ix, float iy, float iz, float tbest,
                                          uint32_t skip, float (&t)[4], uint32_t (&r)[4]) {
  float4 w[8];  // the 128-byte record in four 32-byte loads
  ldg8(wn, w[0], w[1]);
  ldg8(wn + 2, w[2], w[3]);
  ldg8(wn + 4, w[4], w[5]);
  ldg8(wn + 6, w[6], w[7]);
  wide_test_regs(w, oi, ix, iy, iz, tbest, skip, t, r);
}

// The four slots of a cluster record against a ray, in slot order: entry distance of each slot the ray enters
// within reach (+inf otherwise) and the slot references.
__device__ __forceinline__ void cluster_slots(const float4* __restrict__ rec, const float4& oi, float ix, float iy, float iz,
                                              float tbest, float (&t)[4], uint32_t (&r)[4]) {
  float4 w0, w1, w2, w3, w4, w5;
  ldg8(rec, w0, w1);
  ldg8(rec + 2, w2, w3);
  ldg8(rec + 4, w4, w5);
  const uint4 wr = ldg4((const uint4*)(rec + 6));
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const float t0x = __fmaf_rn(f4c(w0, s), ix, -oi.x), t1x = __fmaf_rn(f4c(w3, s), ix, -oi.x);
    const float t0y = __fmaf_rn(f4c(w1, s), iy, -oi.y), t1y = __fmaf_rn(f4c(w4, s), iy, -oi.y);
    const float t0z = __fmaf_rn(f4c(w2, s), iz, -oi.z), t1z = __fmaf_rn(f4c(w5, s), iz, -oi.z);
    const float tn = max3f(fminf(t0x, t1x), fminf(t0y, t1y), fminf(t0z, t1z));
    const float tf = min3f(fmaxf(t0x, t1x), fmaxf(t0y, t1y), fmaxf(t0z, t1z));
    t[s] = (tn <= tf && tf >= 0.0f && tn <= tbest * kCullSlack) ? tn : INFINITY;
    r[s] = u4c(wr, s);
  }
}
// The same, nearest first (5-comparator network).
__device__ __forceinline__ void cluster_test(const float4* __restrict__ rec, const float4& oi, float ix, float iy, float iz,
                                             float tbest, float (&t)[4], uint32_t (&r)[4]) {
  cluster_slots(rec, oi, ix, iy, iz, tbest, t, r);
  cswap_tr(t, r, 0, 1);
  cswap_tr(t, r, 2, 3);
  cswap_tr(t, r, 0, 2);
  cswap_tr(t, r, 1, 3);
  cswap_tr(t, r, 1, 2);
}

// ---------------------------------------------------------------------------
// batched meshes
// ---------------------------------------------------------------------------
// Largest m in [0, M) with off[m] <= x (off ascending, off[0] = 0).
__device__ __forceinline__ uint32_t find_seg(const uint32_t* __restrict__ off, uint32_t M, uint32_t x) {
  uint32_t lo = 0, hi = M - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Per-mesh bases inside the batched arrays, all derived from F_m (the mesh's
// first face) and m: node records (capacity 2 n_m - 1), Morton-level arrays
// (capacity 2 n_m + 3), group boxes (mesh m uses fewer than n_m + n_m / 8 + 1).
__host__ __device__ __forceinline__ uint32_t node_base(uint32_t F, uint32_t m) { return 2 * F - m; }
__host__ __device__ __forceinline__ uint32_t bfs_base(uint32_t F, uint32_t m) { return 2 * F + 3 * m; }
__host__ __device__ __forceinline__ uint32_t group_base(uint32_t F, uint32_t m) { return F + F / 8 + m; }

// Batched traversal blob: per-mesh headers (64 words), two-child records at
// 4 F_m, leaf tables at F_m, group boxes at 2 group_base(F_m, m).
// Mesh m (F = faces before it) owns header words 64 m .., two-child records
// 4 F .., leaves F .., group boxes 2 group_base(F, m) .. and 4-wide records 8 F ..
struct BatchAccel {
  uint32_t* hdr;
  float4* tnodes;
  uint4* leaves;
  float4* groups;
  float4* wide;
  float4* crec;  // cluster records, 8 float4 each; mesh m's from record F_m
};
inline size_t carve_batch_accel_layout(Carve& c, BatchAccel& L, uint32_t M, uint32_t N) {
  L.hdr = c.take<uint32_t>(64 * (size_t)M);
  L.tnodes = c.take<float4>(4 * (size_t)N);
  L.leaves = c.take<uint4>(N);
  L.groups = c.take<float4>(2 * ((size_t)N + N / 8 + M + 1));
  L.wide = c.take<float4>(8 * (size_t)N);
  L.crec = c.take<float4>(8 * (size_t)N);
  return c.off + 256;
}

// Cluster tree builds (rt_clusters.cu), from the sorted Morton codes and the pre-gathered triangles of the
// position order: a single mesh (header hdr, records crec) and all meshes of a batched build (headers 64 words
// apart, records of mesh m from F_m). Two launches each (the chunk pass and the global pass).
rt_status build_cluster_tree(const float4* tris, const uint32_t* codes, uint32_t n, uint32_t leaf_max, const ClusterTemps& T,
                             uint32_t* hdr, float4* crec, cudaStream_t st);
rt_status batch_build_cluster_tree(const float4* tris, const uint32_t* codes, const uint32_t* foff, uint32_t M, uint32_t N,
                                   uint32_t leaf_max, const ClusterTemps& T, uint32_t* hdr, float4* crec, cudaStream_t st);

}  // namespace rt
