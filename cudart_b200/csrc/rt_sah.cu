// rt_sah.cu -- SAH and Hybrid BVH builds (CUDAMeshTree::buildMeshTreeSAH /
// buildMeshTreeHybrid, CUDAMeshTree.cpp:93-103; kernels/CUDA_buildMeshTreeSAH.cu).
//
// The reference processes one stacked node per 32-thread block with thread 0
// doing the binning and the partition serially, and numbers nodes in the order
// its concurrent blocks happen to reach atomicAdd. This build is level
// synchronous: every node of a level is processed at once, one CTA per node of
// more than kBigNode faces and one warp per smaller node, each doing the
// centroid bounds, the 32-bin histogram (shared-memory atomics on order-keyed
// floats, exact because min / max do not depend on order), the bin sweep
// (lane m holds bin m: prefix / suffix by shuffles) and the stable partition
// (ballots, block scans) in one kernel. Decisions use the reference's float
// expressions in its order, so every node is decided exactly as the serial
// reference decides it. The node ids of the serial reference (depth first,
// left first: the k-th split of a subtree rooted when the counter stood at B
// gets B + 2k, B + 2k + 1) are assigned afterwards from the tree's shape:
// subtree split counts bottom-up, pre-order ranks top-down.
#include <utility>
#include <vector>

#include "../../include/rt_sah.h"
#include "rt_device.cuh"

namespace rt {
namespace {

constexpr int kBins = 32;                      // SM_BIN_COUNT, kernels/CUDA_buildMeshTreeSAH.cu:48
constexpr float kTriCost = 0.125f;             // TRI_RAY_COST, :52
constexpr float kBoxCost = 1.0f;               // BOX_RAY_COST, :53
constexpr uint32_t kSahMinLeaf = 16;           // MIN_LEAF_SIZE, :55
constexpr uint32_t kSahMaxLeaf = 224;          // MAX_LEAF_SIZE, :56
constexpr uint32_t kBigNode = 4096;            // nodes above this many faces get a whole CTA
constexpr int kCta = 256;

// Node of the build table (level order). info: bit 0 right child, bit 1 leaf,
// bits 2-3 split axis.
struct SNode {
  float4 mn, mx;
  uint32_t first, count, parent, info;
  uint32_t child, sub, internal, id;
};
static_assert(sizeof(SNode) == 64, "SNode is 64 bytes");

struct Item {  // a face in position order: its box (aabox) and id
  float4 mn, mx;
};

// order-preserving keys of floats (sign-magnitude read as unsigned): key(a) <
// key(b) iff a < b, and -0 < +0
__device__ __forceinline__ uint32_t okey(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ofloat(uint32_t k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k); }
__device__ __forceinline__ float omin(float a, float b) { return okey(b) < okey(a) ? b : a; }
__device__ __forceinline__ float omax(float a, float b) { return okey(b) > okey(a) ? b : a; }

// aabox::getArea (CUDABox.h:35-45): v = max - min, 2 (x y + x z + y z)
__device__ __forceinline__ float box_area(float3 mn, float3 mx) {
  const float vx = mx.x - mn.x, vy = mx.y - mn.y, vz = mx.z - mn.z;
  return 2.f * (vx * vy + vx * vz + vy * vz);
}

struct Split {  // how a node is cut: axis, bin mapping, chosen boundary
  int axis;
  float scale, bmin;
};

__device__ __forceinline__ float center_on(const Item& it, int axis) {
  const float a = axis == 0 ? it.mn.x : (axis == 1 ? it.mn.y : it.mn.z);
  const float b = axis == 0 ? it.mx.x : (axis == 1 ? it.mx.y : it.mx.z);
  return 0.5f * (a + b);
}
// bin of a centroid: (int) of (c - bmin) * scale as a kernel converts it
// (toward zero, saturating, NaN -> 0), clamped to [0, 31] (:375-385)
__device__ __forceinline__ int bin_of(float c, const Split& s) {
  int m = __float2int_rz((c - s.bmin) * s.scale);
  if (m < 0) m = 0;
  else if (m >= kBins - 1) m = kBins - 1;
  return m;
}

// Longest axis of the centroid bounds and the bin mapping (:310-341).
__device__ __forceinline__ Split make_split(float3 cmn, float3 cmx) {
  const float ex = cmx.x - cmn.x, ey = cmx.y - cmn.y, ez = cmx.z - cmn.z;
  Split s;
  if (ex > ey) s.axis = ex > ez ? 0 : 2;
  else s.axis = ey > ez ? 1 : 2;
  const float e = s.axis == 0 ? ex : (s.axis == 1 ? ey : ez);
  s.scale = (float)(kBins - 1) / e;
  s.bmin = s.axis == 0 ? cmn.x : (s.axis == 1 ? cmn.y : cmn.z);
  return s;
}

// 32 bins as order keys (count, min xyz, max xyz); empty: +HUGE / -HUGE.
struct Bins {
  uint32_t cnt[kBins];
  uint32_t mn[3][kBins];
  uint32_t mx[3][kBins];
};
__device__ __forceinline__ void bins_reset(Bins& B, int m) {
  B.cnt[m] = 0;
  for (int k = 0; k < 3; ++k) { B.mn[k][m] = okey(kHuge); B.mx[k][m] = okey(-kHuge); }
}
__device__ __forceinline__ void bins_add(Bins& B, int m, const Item& it) {
  atomicAdd(&B.cnt[m], 1u);
  atomicMin(&B.mn[0][m], okey(it.mn.x)); atomicMin(&B.mn[1][m], okey(it.mn.y)); atomicMin(&B.mn[2][m], okey(it.mn.z));
  atomicMax(&B.mx[0][m], okey(it.mx.x)); atomicMax(&B.mx[1][m], okey(it.mx.y)); atomicMax(&B.mx[2][m], okey(it.mx.z));
}

struct Decision {
  int m_min;       // chosen boundary (bins <= m_min go left), -1 = leaf
  uint32_t nl;     // faces on the left
  float3 lmn, lmx, rmn, rmx;
};

// The bin sweep of :423-474 with lane m holding bin m (one full warp): left
// prefix over bins <= m, right suffix over bins > m, the cost of boundary m,
// and the reference's choice (descending scan, strict <: the largest m among
// equal minima, only costs below +HUGE). Then the leaf test of :479-480.
__device__ Decision decide(const Bins& B, float3 pmn, float3 pmx, uint32_t count) {
  const int m = (int)(threadIdx.x & 31u);
  uint32_t c = B.cnt[m];
  float3 bmn = make_float3(ofloat(B.mn[0][m]), ofloat(B.mn[1][m]), ofloat(B.mn[2][m]));
  float3 bmx = make_float3(ofloat(B.mx[0][m]), ofloat(B.mx[1][m]), ofloat(B.mx[2][m]));
  // inclusive prefix (bins 0..m)
  uint32_t lc = c;
  float3 lmn = bmn, lmx = bmx;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yc = __shfl_up_sync(0xffffffffu, lc, o);
    const float a0 = __shfl_up_sync(0xffffffffu, lmn.x, o), a1 = __shfl_up_sync(0xffffffffu, lmn.y, o),
                a2 = __shfl_up_sync(0xffffffffu, lmn.z, o);
    const float b0 = __shfl_up_sync(0xffffffffu, lmx.x, o), b1 = __shfl_up_sync(0xffffffffu, lmx.y, o),
                b2 = __shfl_up_sync(0xffffffffu, lmx.z, o);
    if (m >= o) {
      lc += yc;
      lmn = make_float3(omin(lmn.x, a0), omin(lmn.y, a1), omin(lmn.z, a2));
      lmx = make_float3(omax(lmx.x, b0), omax(lmx.y, b1), omax(lmx.z, b2));
    }
  }
  // inclusive suffix (bins m..31), then shifted to bins > m
  uint32_t sc = c;
  float3 smn = bmn, smx = bmx;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yc = __shfl_down_sync(0xffffffffu, sc, o);
    const float a0 = __shfl_down_sync(0xffffffffu, smn.x, o), a1 = __shfl_down_sync(0xffffffffu, smn.y, o),
                a2 = __shfl_down_sync(0xffffffffu, smn.z, o);
    const float b0 = __shfl_down_sync(0xffffffffu, smx.x, o), b1 = __shfl_down_sync(0xffffffffu, smx.y, o),
                b2 = __shfl_down_sync(0xffffffffu, smx.z, o);
    if (m + o < 32) {
      sc += yc;
      smn = make_float3(omin(smn.x, a0), omin(smn.y, a1), omin(smn.z, a2));
      smx = make_float3(omax(smx.x, b0), omax(smx.y, b1), omax(smx.z, b2));
    }
  }
  uint32_t rc = __shfl_down_sync(0xffffffffu, sc, 1);
  float3 rmn = make_float3(__shfl_down_sync(0xffffffffu, smn.x, 1), __shfl_down_sync(0xffffffffu, smn.y, 1),
                           __shfl_down_sync(0xffffffffu, smn.z, 1));
  float3 rmx = make_float3(__shfl_down_sync(0xffffffffu, smx.x, 1), __shfl_down_sync(0xffffffffu, smx.y, 1),
                           __shfl_down_sync(0xffffffffu, smx.z, 1));
  const float pa = box_area(pmn, pmx);
  const float larea = 0.0f + box_area(lmn, lmx);  // bvbin::insertLeft adds to a zero area
  const float rarea = 0.0f + box_area(rmn, rmx);
  const float t = kBoxCost * 2.f + kTriCost * ((larea / pa) * (float)lc + (rarea / pa) * (float)rc);
  const bool valid = m < kBins - 1 && t < kHuge;
  float tv = valid ? t : INFINITY;
#pragma unroll
  for (int o = 16; o; o >>= 1) tv = fminf(tv, __shfl_xor_sync(0xffffffffu, tv, o));
  const unsigned at_min = __ballot_sync(0xffffffffu, valid && t == tv);
  Decision d;
  d.m_min = at_min ? 31 - __clz((int)at_min) : -1;
  const float t_min = at_min ? tv : kHuge;
  const int src = d.m_min < 0 ? 0 : d.m_min;
  d.nl = __shfl_sync(0xffffffffu, lc, src);
  d.lmn = make_float3(__shfl_sync(0xffffffffu, lmn.x, src), __shfl_sync(0xffffffffu, lmn.y, src), __shfl_sync(0xffffffffu, lmn.z, src));
  d.lmx = make_float3(__shfl_sync(0xffffffffu, lmx.x, src), __shfl_sync(0xffffffffu, lmx.y, src), __shfl_sync(0xffffffffu, lmx.z, src));
  d.rmn = make_float3(__shfl_sync(0xffffffffu, rmn.x, src), __shfl_sync(0xffffffffu, rmn.y, src), __shfl_sync(0xffffffffu, rmn.z, src));
  d.rmx = make_float3(__shfl_sync(0xffffffffu, rmx.x, src), __shfl_sync(0xffffffffu, rmx.y, src), __shfl_sync(0xffffffffu, rmx.z, src));
  if ((count < kSahMaxLeaf && t_min > (float)(count + 1) * kTriCost) || d.m_min < 0) d.m_min = -1;
  return d;
}

struct LevelArgs {
  SNode* table;
  uint32_t* table_count;  // [0] entries, [1] big entries of the next level, [2] no-split leaves
  uint2* big_next;        // (table index, faces) of the next level's big nodes
  const uint32_t* big_cur;  // table indices of this level's big nodes handled one CTA each
  uint32_t level_begin, level_end;
  const uint32_t* idx_in;
  const Item* box_in;
  uint32_t* idx_out;
  Item* box_out;
  uint32_t* final_idx;
  uint32_t* err;
  uint32_t table_cap;
};

__device__ __forceinline__ Item load_item(const Item* p) {
  Item it;
  it.mn = __ldg(&p->mn);
  it.mx = __ldg(&p->mx);
  return it;
}

// Children of a split node: table entries c, c + 1 (lane 0 writes).
__device__ __forceinline__ void write_split(const LevelArgs& A, uint32_t e, const SNode& nd, const Split& sp, const Decision& d,
                                            uint32_t& child_out) {
  uint32_t c = atomicAdd(A.table_count, 2u);
  if (c + 2 > A.table_cap) {
    atomicOr(A.err, (uint32_t)RT_DEVERR_NODE_CAPACITY);
    child_out = kNone;
    return;
  }
  SNode L, R;
  L.mn = make_float4(d.lmn.x, d.lmn.y, d.lmn.z, kHuge);
  L.mx = make_float4(d.lmx.x, d.lmx.y, d.lmx.z, -kHuge);
  L.first = nd.first; L.count = d.nl; L.parent = e; L.info = 0; L.child = kNone; L.sub = nd.sub; L.internal = 0; L.id = kNone;
  R.mn = make_float4(d.rmn.x, d.rmn.y, d.rmn.z, kHuge);
  R.mx = make_float4(d.rmx.x, d.rmx.y, d.rmx.z, -kHuge);
  R.first = nd.first + d.nl; R.count = nd.count - d.nl; R.parent = e; R.info = 1; R.child = kNone; R.sub = nd.sub; R.internal = 0;
  R.id = kNone;
  A.table[c] = L;
  A.table[c + 1] = R;
  if (L.count > kBigNode) A.big_next[atomicAdd(A.table_count + 1, 1u)] = make_uint2(c, L.count);
  if (R.count > kBigNode) A.big_next[atomicAdd(A.table_count + 1, 1u)] = make_uint2(c + 1, R.count);
  A.table[e].child = c;
  A.table[e].info = (nd.info & 1u) | ((uint32_t)sp.axis << 2);  // keep the right-child bit
  child_out = c;
}

// One warp per node of at most kBigNode faces (8 warps per CTA).
__global__ __launch_bounds__(kCta) void k_sah_small(LevelArgs A) {
  __shared__ Bins s_bins[kCta / 32];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t e = A.level_begin + blockIdx.x * (kCta / 32) + warp;
  if (e >= A.level_end) return;
  const SNode nd = A.table[e];
  if (nd.count > kBigNode) return;
  if (nd.count <= kSahMinLeaf) {
    if (lane < nd.count) A.final_idx[nd.first + lane] = A.idx_in[nd.first + lane];
    if (lane == 0) A.table[e].info = (nd.info & 1u) | 2u;  // keep the right-child bit
    return;
  }
  // centroid bounds
  float3 cmn = make_float3(kHuge, kHuge, kHuge), cmx = make_float3(-kHuge, -kHuge, -kHuge);
  for (uint32_t i = lane; i < nd.count; i += 32) {
    const Item it = load_item(A.box_in + nd.first + i);
    const float3 c = make_float3(0.5f * (it.mn.x + it.mx.x), 0.5f * (it.mn.y + it.mx.y), 0.5f * (it.mn.z + it.mx.z));
    cmn = make_float3(omin(cmn.x, c.x), omin(cmn.y, c.y), omin(cmn.z, c.z));
    cmx = make_float3(omax(cmx.x, c.x), omax(cmx.y, c.y), omax(cmx.z, c.z));
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    cmn = make_float3(omin(cmn.x, __shfl_xor_sync(0xffffffffu, cmn.x, o)), omin(cmn.y, __shfl_xor_sync(0xffffffffu, cmn.y, o)),
                      omin(cmn.z, __shfl_xor_sync(0xffffffffu, cmn.z, o)));
    cmx = make_float3(omax(cmx.x, __shfl_xor_sync(0xffffffffu, cmx.x, o)), omax(cmx.y, __shfl_xor_sync(0xffffffffu, cmx.y, o)),
                      omax(cmx.z, __shfl_xor_sync(0xffffffffu, cmx.z, o)));
  }
  const Split sp = make_split(cmn, cmx);
  Bins& B = s_bins[warp];
  bins_reset(B, (int)lane);
  __syncwarp();
  for (uint32_t i = lane; i < nd.count; i += 32) {
    const Item it = load_item(A.box_in + nd.first + i);
    bins_add(B, bin_of(center_on(it, sp.axis), sp), it);
  }
  __syncwarp();
  const Decision d = decide(B, make_float3(nd.mn.x, nd.mn.y, nd.mn.z), make_float3(nd.mx.x, nd.mx.y, nd.mx.z), nd.count);
  if (d.m_min < 0) {
    for (uint32_t i = lane; i < nd.count; i += 32) A.final_idx[nd.first + i] = A.idx_in[nd.first + i];
    if (lane == 0) {
      A.table[e].info = (nd.info & 1u) | 2u;  // keep the right-child bit
      if (nd.count >= kSahMaxLeaf) atomicAdd(A.table_count + 2, 1u);
    }
    return;
  }
  uint32_t c = 0;
  if (lane == 0) write_split(A, e, nd, sp, d, c);
  c = __shfl_sync(0xffffffffu, c, 0);
  if (c == kNone) return;
  // stable partition, 32 faces at a time
  uint32_t lo = nd.first, ro = nd.first + d.nl;
  for (uint32_t base = 0; base < nd.count; base += 32) {
    const uint32_t i = base + lane;
    const bool valid = i < nd.count;
    Item it;
    uint32_t id = 0;
    bool left = false;
    if (valid) {
      it = load_item(A.box_in + nd.first + i);
      id = A.idx_in[nd.first + i];
      left = bin_of(center_on(it, sp.axis), sp) <= d.m_min;
    }
    const unsigned lb = __ballot_sync(0xffffffffu, valid && left), rb = __ballot_sync(0xffffffffu, valid && !left);
    const unsigned below = (1u << lane) - 1u;
    if (valid) {
      const uint32_t dst = left ? lo + __popc(lb & below) : ro + __popc(rb & below);
      A.idx_out[dst] = id;
      A.box_out[dst] = it;
    }
    lo += __popc(lb);
    ro += __popc(rb);
  }
}

// One CTA per node of more than kBigNode faces.
__global__ __launch_bounds__(kCta) void k_sah_big(LevelArgs A, uint32_t count_big) {
  __shared__ Bins B;
  __shared__ float s_red[6][kCta / 32];
  __shared__ uint32_t s_scan[kCta / 32];
  __shared__ Decision s_d;
  __shared__ uint32_t s_child;
  if (blockIdx.x >= count_big) return;
  const uint32_t e = A.big_cur[blockIdx.x];
  const SNode nd = A.table[e];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  float3 cmn = make_float3(kHuge, kHuge, kHuge), cmx = make_float3(-kHuge, -kHuge, -kHuge);
  for (uint32_t i = threadIdx.x; i < nd.count; i += kCta) {
    const Item it = load_item(A.box_in + nd.first + i);
    const float3 c = make_float3(0.5f * (it.mn.x + it.mx.x), 0.5f * (it.mn.y + it.mx.y), 0.5f * (it.mn.z + it.mx.z));
    cmn = make_float3(omin(cmn.x, c.x), omin(cmn.y, c.y), omin(cmn.z, c.z));
    cmx = make_float3(omax(cmx.x, c.x), omax(cmx.y, c.y), omax(cmx.z, c.z));
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    cmn = make_float3(omin(cmn.x, __shfl_xor_sync(0xffffffffu, cmn.x, o)), omin(cmn.y, __shfl_xor_sync(0xffffffffu, cmn.y, o)),
                      omin(cmn.z, __shfl_xor_sync(0xffffffffu, cmn.z, o)));
    cmx = make_float3(omax(cmx.x, __shfl_xor_sync(0xffffffffu, cmx.x, o)), omax(cmx.y, __shfl_xor_sync(0xffffffffu, cmx.y, o)),
                      omax(cmx.z, __shfl_xor_sync(0xffffffffu, cmx.z, o)));
  }
  if (lane == 0) {
    s_red[0][warp] = cmn.x; s_red[1][warp] = cmn.y; s_red[2][warp] = cmn.z;
    s_red[3][warp] = cmx.x; s_red[4][warp] = cmx.y; s_red[5][warp] = cmx.z;
  }
  if (threadIdx.x < kBins) bins_reset(B, (int)threadIdx.x);
  __syncthreads();
  cmn = make_float3(s_red[0][0], s_red[1][0], s_red[2][0]);
  cmx = make_float3(s_red[3][0], s_red[4][0], s_red[5][0]);
  for (int w = 1; w < kCta / 32; ++w) {
    cmn = make_float3(omin(cmn.x, s_red[0][w]), omin(cmn.y, s_red[1][w]), omin(cmn.z, s_red[2][w]));
    cmx = make_float3(omax(cmx.x, s_red[3][w]), omax(cmx.y, s_red[4][w]), omax(cmx.z, s_red[5][w]));
  }
  const Split sp = make_split(cmn, cmx);
  for (uint32_t i = threadIdx.x; i < nd.count; i += kCta) {
    const Item it = load_item(A.box_in + nd.first + i);
    bins_add(B, bin_of(center_on(it, sp.axis), sp), it);
  }
  __syncthreads();
  if (warp == 0) {
    const Decision d = decide(B, make_float3(nd.mn.x, nd.mn.y, nd.mn.z), make_float3(nd.mx.x, nd.mx.y, nd.mx.z), nd.count);
    uint32_t c = kNone;
    if (lane == 0) {
      if (d.m_min >= 0) {
        write_split(A, e, nd, sp, d, c);
      } else {
        A.table[e].info = (nd.info & 1u) | 2u;  // keep the right-child bit
        if (nd.count >= kSahMaxLeaf) atomicAdd(A.table_count + 2, 1u);
      }
      s_d = d;
      s_child = c;
    }
  }
  __syncthreads();
  const Decision d = s_d;
  if (d.m_min < 0) {
    for (uint32_t i = threadIdx.x; i < nd.count; i += kCta) A.final_idx[nd.first + i] = A.idx_in[nd.first + i];
    return;
  }
  if (s_child == kNone) return;
  // stable partition: thread t owns the contiguous slice [t S, (t + 1) S) of
  // the node; one block scan of the per-slice left counts places every slice
  const uint32_t S = (nd.count + kCta - 1) / kCta;
  const uint32_t a = min(nd.count, threadIdx.x * S), b = min(nd.count, a + S);
  uint32_t my_left = 0;
  for (uint32_t i = a; i < b; ++i) my_left += bin_of(center_on(load_item(A.box_in + nd.first + i), sp.axis), sp) <= d.m_min ? 1u : 0u;
  uint32_t total_left;
  const uint32_t lpre = block_excl_scan_nt<kCta>(my_left, s_scan, total_left);
  uint32_t lo = nd.first + lpre, ro = nd.first + d.nl + (a - lpre);
  for (uint32_t i = a; i < b; ++i) {
    const Item it = load_item(A.box_in + nd.first + i);
    const uint32_t id = A.idx_in[nd.first + i];
    const uint32_t dst = bin_of(center_on(it, sp.axis), sp) <= d.m_min ? lo++ : ro++;
    A.idx_out[dst] = id;
    A.box_out[dst] = it;
  }
}

// ---------------------------------------------------------------- huge nodes
// Nodes of more than kHugeNode faces are cut into tiles of kTile faces that
// separate CTAs process: bounds and bins meet in global order-key atomics, one
// warp per node decides, a scan over the tiles' left counts places every
// tile, and each tile scatters its faces stably (per-thread slices + a block
// scan), so the result equals the single-owner kernels'.
constexpr uint32_t kHugeNode = 32768;
constexpr uint32_t kTile = 8192;

struct HugeArgs {
  const uint32_t* node;   // [H] table index of huge node h
  const uint32_t* tnode;  // [tiles] huge slot of tile t
  const uint32_t* tstart; // [tiles] first face (position) of tile t
  const uint32_t* tfirst; // [H] first tile of node h
  uint32_t* keys;         // [H][8] centroid bounds as order keys (min xyz, max xyz)
  Bins* bins;             // [H]
  Decision* dec;          // [H]
  Split* split;           // [H]
  uint32_t* child;        // [H] first child table index, kNone when a leaf
  uint32_t* tleft;        // [tiles] left faces per tile, then its exclusive scan
  uint32_t H, tiles;
};

__global__ __launch_bounds__(256) void k_huge_reset(HugeArgs G) {
  const uint32_t h = blockIdx.x;
  if (h >= G.H) return;
  if (threadIdx.x < 3) { G.keys[8 * h + threadIdx.x] = 0xFFFFFFFFu; G.keys[8 * h + 3 + threadIdx.x] = 0u; }
  if (threadIdx.x < kBins) bins_reset(G.bins[h], (int)threadIdx.x);
}

__global__ __launch_bounds__(kCta) void k_huge_bounds(LevelArgs A, HugeArgs G) {
  const uint32_t t = blockIdx.x;
  const uint32_t h = G.tnode[t];
  const SNode nd = A.table[G.node[h]];
  const uint32_t ts = G.tstart[t], te = min(nd.first + nd.count, ts + kTile);
  uint32_t k[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
  for (uint32_t p = ts + threadIdx.x; p < te; p += kCta) {
    const Item it = load_item(A.box_in + p);
    const uint32_t cx = okey(0.5f * (it.mn.x + it.mx.x)), cy = okey(0.5f * (it.mn.y + it.mx.y)), cz = okey(0.5f * (it.mn.z + it.mx.z));
    k[0] = min(k[0], cx); k[1] = min(k[1], cy); k[2] = min(k[2], cz);
    k[3] = max(k[3], cx); k[4] = max(k[4], cy); k[5] = max(k[5], cz);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      k[c] = min(k[c], __shfl_xor_sync(0xffffffffu, k[c], o));
      k[3 + c] = max(k[3 + c], __shfl_xor_sync(0xffffffffu, k[3 + c], o));
    }
  }
  if ((threadIdx.x & 31u) == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) { atomicMin(G.keys + 8 * h + c, k[c]); atomicMax(G.keys + 8 * h + 3 + c, k[3 + c]); }
  }
}

__device__ __forceinline__ Split huge_split(const HugeArgs& G, uint32_t h) {
  const uint32_t* k = G.keys + 8 * h;
  return make_split(make_float3(ofloat(k[0]), ofloat(k[1]), ofloat(k[2])), make_float3(ofloat(k[3]), ofloat(k[4]), ofloat(k[5])));
}

__global__ __launch_bounds__(kCta) void k_huge_bins(LevelArgs A, HugeArgs G) {
  __shared__ Bins B;
  const uint32_t t = blockIdx.x;
  const uint32_t h = G.tnode[t];
  const SNode nd = A.table[G.node[h]];
  const uint32_t ts = G.tstart[t], te = min(nd.first + nd.count, ts + kTile);
  const Split sp = huge_split(G, h);
  if (threadIdx.x < kBins) bins_reset(B, (int)threadIdx.x);
  __syncthreads();
  for (uint32_t p = ts + threadIdx.x; p < te; p += kCta) {
    const Item it = load_item(A.box_in + p);
    bins_add(B, bin_of(center_on(it, sp.axis), sp), it);
  }
  __syncthreads();
  if (threadIdx.x < kBins) {
    const int m = (int)threadIdx.x;
    if (B.cnt[m]) {
      Bins& g = G.bins[h];
      atomicAdd(&g.cnt[m], B.cnt[m]);
      for (int c = 0; c < 3; ++c) { atomicMin(&g.mn[c][m], B.mn[c][m]); atomicMax(&g.mx[c][m], B.mx[c][m]); }
    }
  }
}

// one warp per huge node
__global__ __launch_bounds__(32) void k_huge_decide(LevelArgs A, HugeArgs G) {
  const uint32_t h = blockIdx.x;
  const uint32_t e = G.node[h];
  const SNode nd = A.table[e];
  const Split sp = huge_split(G, h);
  const Decision d = decide(G.bins[h], make_float3(nd.mn.x, nd.mn.y, nd.mn.z), make_float3(nd.mx.x, nd.mx.y, nd.mx.z), nd.count);
  if (threadIdx.x == 0) {
    uint32_t c = kNone;
    if (d.m_min >= 0) {
      write_split(A, e, nd, sp, d, c);
    } else {
      A.table[e].info = (nd.info & 1u) | 2u;
      atomicAdd(A.table_count + 2, 1u);
    }
    G.dec[h] = d;
    G.split[h] = sp;
    G.child[h] = c;
  }
}

__global__ __launch_bounds__(kCta) void k_huge_count(LevelArgs A, HugeArgs G) {
  __shared__ uint32_t s_w[kCta / 32];
  const uint32_t t = blockIdx.x;
  const uint32_t h = G.tnode[t];
  const SNode nd = A.table[G.node[h]];
  const uint32_t ts = G.tstart[t], te = min(nd.first + nd.count, ts + kTile);
  const Decision& d = G.dec[h];
  const Split sp = G.split[h];
  uint32_t n = 0;
  if (d.m_min >= 0)
    for (uint32_t p = ts + threadIdx.x; p < te; p += kCta) n += bin_of(center_on(load_item(A.box_in + p), sp.axis), sp) <= d.m_min ? 1u : 0u;
  uint32_t total;
  block_excl_scan_nt<kCta>(n, s_w, total);
  if (threadIdx.x == 0) G.tleft[t] = total;
}

__global__ __launch_bounds__(kCta) void k_huge_scatter(LevelArgs A, HugeArgs G) {
  __shared__ uint32_t s_w[kCta / 32];
  const uint32_t t = blockIdx.x;
  const uint32_t h = G.tnode[t];
  const SNode nd = A.table[G.node[h]];
  const uint32_t ts = G.tstart[t], te = min(nd.first + nd.count, ts + kTile);
  const Decision d = G.dec[h];
  if (d.m_min < 0) {  // a leaf: its faces are final
    for (uint32_t p = ts + threadIdx.x; p < te; p += kCta) A.final_idx[p] = A.idx_in[p];
    return;
  }
  if (G.child[h] == kNone) return;
  const Split sp = G.split[h];
  const uint32_t left_before = G.tleft[t] - G.tleft[G.tfirst[h]];  // left faces in the node's earlier tiles
  const uint32_t S = (te - ts + kCta - 1) / kCta;
  const uint32_t a = min(te, ts + threadIdx.x * S), b = min(te, a + S);
  uint32_t my_left = 0;
  for (uint32_t p = a; p < b; ++p) my_left += bin_of(center_on(load_item(A.box_in + p), sp.axis), sp) <= d.m_min ? 1u : 0u;
  uint32_t total;
  const uint32_t lpre = block_excl_scan_nt<kCta>(my_left, s_w, total);
  uint32_t lo = nd.first + left_before + lpre;
  uint32_t ro = nd.first + d.nl + ((ts - nd.first) - left_before) + ((a - ts) - lpre);
  for (uint32_t p = a; p < b; ++p) {
    const Item it = load_item(A.box_in + p);
    const uint32_t id = A.idx_in[p];
    const uint32_t dst = bin_of(center_on(it, sp.axis), sp) <= d.m_min ? lo++ : ro++;
    A.idx_out[dst] = id;
    A.box_out[dst] = it;
  }
}

// ---------------------------------------------------------------- setup
// SAH: positions start as the faces in order, the root's box is the mesh box.
__global__ __launch_bounds__(256) void k_sah_init(const float4* __restrict__ boxes, uint32_t n, const float* __restrict__ hit,
                                                  uint32_t* idx, Item* items, SNode* table, uint32_t* counts) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    idx[p] = p;
    items[p].mn = boxes[2 * (size_t)p];
    items[p].mx = boxes[2 * (size_t)p + 1];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    SNode r;
    r.mn = make_float4(hit[0], hit[1], hit[2], hit[3]);
    r.mx = make_float4(hit[4], hit[5], hit[6], hit[7]);
    r.first = 0; r.count = n; r.parent = kNone; r.info = 0; r.child = kNone; r.sub = 0; r.internal = 0; r.id = 0;
    table[0] = r;
    counts[0] = 1;
    counts[1] = 0;
    counts[2] = 0;
    if (n > kBigNode) { counts[1] = 1; }
  }
}

// The mesh box (CUDAModel: reset, then merge of every vertex) as order keys:
// keys[0..3] min xyzw (start 0xFFFFFFFF), keys[4..7] max xyzw (start 0).
__global__ __launch_bounds__(256) void k_vertex_bounds(const float4* __restrict__ v, uint32_t n, uint32_t* keys) {
  uint32_t mn[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, mx[4] = {0u, 0u, 0u, 0u};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 p = __ldg(v + i);
    const uint32_t k[4] = {okey(p.x), okey(p.y), okey(p.z), okey(p.w)};
#pragma unroll
    for (int c = 0; c < 4; ++c) { mn[c] = min(mn[c], k[c]); mx[c] = max(mx[c], k[c]); }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      mn[c] = min(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
      mx[c] = max(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
    }
  }
  if ((threadIdx.x & 31u) == 0) {
#pragma unroll
    for (int c = 0; c < 4; ++c) { atomicMin(keys + c, mn[c]); atomicMax(keys + 4 + c, mx[c]); }
  }
}
__global__ void k_keys_to_box(const uint32_t* keys, float* hit) {
  const int c = threadIdx.x;
  if (c < 8) hit[c] = ofloat(keys[c]);
}

// Hybrid: positions in the LBVH's order; one subtree per LBVH leaf, in
// descending node id (the order in which the reference's stack pops them).
__global__ __launch_bounds__(256) void k_hyb_items(const float4* __restrict__ boxes, const uint32_t* __restrict__ lbvh_idx, uint32_t n,
                                                   uint32_t* idx, Item* items) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t f = lbvh_idx[p];
    idx[p] = f;
    items[p].mn = boxes[2 * (size_t)f];
    items[p].mx = boxes[2 * (size_t)f + 1];
  }
}
__global__ __launch_bounds__(256) void k_hyb_leaf_flags(const uint32_t* __restrict__ nodes, uint32_t m, uint32_t* flags_rev) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
    flags_rev[m - 1 - k] = nodes[8 * (size_t)k] & 1u;
}
__global__ __launch_bounds__(256) void k_hyb_roots(const uint32_t* __restrict__ nodes, uint32_t m, const uint32_t* __restrict__ order_rev,
                                                   SNode* table, uint2* big, uint32_t* counts) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
    const uint32_t* w = nodes + 8 * (size_t)k;
    if (!(w[0] & 1u)) continue;
    const uint32_t j = order_rev[m - 1 - k];  // leaves with a larger id come first
    SNode r;
    r.mn = make_float4(__uint_as_float(w[2]), __uint_as_float(w[3]), __uint_as_float(w[4]), 0.0f);
    r.mx = make_float4(__uint_as_float(w[5]), __uint_as_float(w[6]), __uint_as_float(w[7]), 0.0f);
    r.first = w[1]; r.count = w[0] >> 1; r.parent = kNone; r.info = 0; r.child = kNone; r.sub = j; r.internal = 0; r.id = k;
    table[j] = r;
    if (r.count > kBigNode) big[atomicAdd(counts + 1, 1u)] = make_uint2(j, r.count);
  }
}

// ---------------------------------------------------------------- numbering
__global__ __launch_bounds__(256) void k_sah_internal(SNode* table, uint32_t b, uint32_t e) {
  for (uint32_t i = b + blockIdx.x * blockDim.x + threadIdx.x; i < e; i += gridDim.x * blockDim.x) {
    SNode& x = table[i];
    x.internal = ((x.info & 2u) || x.child == kNone) ? 0u : 1u + table[x.child].internal + table[x.child + 1].internal;
  }
}
// subtree bases: base[j] = first + 2 * (splits of subtrees 0..j-1) (inclusive scan input 2 * internal)
__global__ __launch_bounds__(256) void k_sah_base_in(const SNode* table, uint32_t roots, uint32_t* v) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < roots; j += gridDim.x * blockDim.x) v[j] = 2u * table[j].internal;
}
// top-down: rank = pre-order index of a split node among its subtree's splits
__global__ __launch_bounds__(256) void k_sah_rank(SNode* table, uint32_t b, uint32_t e, uint32_t* rank, const uint32_t* base,
                                                  uint32_t first_base) {
  for (uint32_t i = b + blockIdx.x * blockDim.x + threadIdx.x; i < e; i += gridDim.x * blockDim.x) {
    SNode& x = table[i];
    if (x.parent == kNone) {
      rank[i] = 0;
      continue;
    }
    const SNode& p = table[x.parent];
    const uint32_t rp = rank[x.parent];
    rank[i] = (x.info & 1u) ? rp + 1u + table[p.child].internal : rp + 1u;
    x.id = first_base + base[x.sub] + 2u * rp + (x.info & 1u);
  }
}
__global__ __launch_bounds__(256) void k_sah_write(const SNode* table, uint32_t count, const uint32_t* rank, const uint32_t* base,
                                                   uint32_t first_base, uint32_t* nodes, uint32_t max_nodes, uint32_t* marks,
                                                   uint32_t* err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const SNode x = table[i];
    if (x.id >= max_nodes) {
      atomicOr(err, (uint32_t)RT_DEVERR_NODE_CAPACITY);
      continue;
    }
    uint32_t* w = nodes + 8 * (size_t)x.id;
    if (x.info & 2u) {
      w[0] = 1u | (x.count << 1);
      w[1] = x.first;
      marks[x.first] = 1u;
    } else {
      w[0] = ((x.info >> 2) & 3u) << 1;
      w[1] = first_base + base[x.sub] + 2u * rank[i];
    }
    w[2] = __float_as_uint(x.mn.x); w[3] = __float_as_uint(x.mn.y); w[4] = __float_as_uint(x.mn.z);
    w[5] = __float_as_uint(x.mx.x); w[6] = __float_as_uint(x.mx.y); w[7] = __float_as_uint(x.mx.z);
  }
}

// ---------------------------------------------------------------- outputs
// One warp per leaf: leaf table entry, faces in position order, triangle
// stream and padded 8-face group boxes (the layout of the LBVH build's blob).
__global__ __launch_bounds__(256) void k_sah_leaves(const uint32_t* __restrict__ nodes, uint32_t node_count, const uint32_t* __restrict__ lam,
                                                    const uint32_t* __restrict__ idx, const uint4* __restrict__ faces_in,
                                                    const float4* __restrict__ verts, uint4* __restrict__ faces_out, float4* __restrict__ tris,
                                                    uint4* __restrict__ acc_leaves, float4* __restrict__ acc_groups,
                                                    uint32_t* __restrict__ leaf_lambda, uint32_t n, uint32_t* err) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < node_count; k += (gridDim.x * blockDim.x) >> 5) {
    const uint2 w = *(const uint2*)(nodes + 8 * (size_t)k);
    if (!(w.x & 1u)) continue;
    const uint32_t first = w.y, cnt = w.x >> 1;
    if (first >= n || cnt > n - first) {  // a malformed record: report, do not touch memory
      if (lane == 0) atomicOr(err, (uint32_t)RT_DEVERR_NODE_CAPACITY);
      continue;
    }
    const uint32_t g = lam[first];
    const uint32_t gbase = (first >> 3) + g;
    if (lane == 0) {
      if (acc_leaves) acc_leaves[g] = make_uint4(first, cnt, gbase, k);
      if (leaf_lambda) leaf_lambda[k] = g;
    }
    for (uint32_t base = 0; base < cnt; base += 32) {
      const uint32_t i = first + base + lane;
      float3 tmn = make_float3(kHuge, kHuge, kHuge), tmx = make_float3(-kHuge, -kHuge, -kHuge);
      if (base + lane < cnt) {
        const uint4 f = __ldg(faces_in + idx[i]);
        const float4 v0 = __ldg(verts + f.x), v1 = __ldg(verts + f.y), v2 = __ldg(verts + f.z);
        faces_out[i] = f;
        if (tris) {
          tris[3 * (size_t)i + 0] = make_float4(v0.x, v0.y, v0.z, 0.0f);
          tris[3 * (size_t)i + 1] = make_float4(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z, 0.0f);
          tris[3 * (size_t)i + 2] = make_float4(v2.x - v0.x, v2.y - v0.y, v2.z - v0.z, 0.0f);
        }
        tmn = make_float3(fmin_sel(fmin_sel(v0.x, v1.x), v2.x), fmin_sel(fmin_sel(v0.y, v1.y), v2.y), fmin_sel(fmin_sel(v0.z, v1.z), v2.z));
        tmx = make_float3(fmax_sel(fmax_sel(v0.x, v1.x), v2.x), fmax_sel(fmax_sel(v0.y, v1.y), v2.y), fmax_sel(fmax_sel(v0.z, v1.z), v2.z));
      }
      if (acc_groups) {
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
          tmn.x = fmin_sel(tmn.x, __shfl_xor_sync(0xffffffffu, tmn.x, o));
          tmn.y = fmin_sel(tmn.y, __shfl_xor_sync(0xffffffffu, tmn.y, o));
          tmn.z = fmin_sel(tmn.z, __shfl_xor_sync(0xffffffffu, tmn.z, o));
          tmx.x = fmax_sel(tmx.x, __shfl_xor_sync(0xffffffffu, tmx.x, o));
          tmx.y = fmax_sel(tmx.y, __shfl_xor_sync(0xffffffffu, tmx.y, o));
          tmx.z = fmax_sel(tmx.z, __shfl_xor_sync(0xffffffffu, tmx.z, o));
        }
        if ((lane & 7u) == 0 && base + lane < cnt) {
          pad_box(tmn, tmx);
          const size_t gi = (size_t)gbase + ((base + lane) >> 3);
          acc_groups[2 * gi] = make_float4(tmn.x, tmn.y, tmn.z, 0.0f);
          acc_groups[2 * gi + 1] = make_float4(tmx.x, tmx.y, tmx.z, 0.0f);
        }
      }
    }
  }
}
__global__ __launch_bounds__(256) void k_sah_accel(const uint32_t* __restrict__ nodes, uint32_t node_count, uint32_t leaf_count,
                                                   const uint32_t* __restrict__ leaf_lambda, float4* __restrict__ tnodes, uint32_t* acc_hdr) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    acc_hdr[0] = (nodes[0] & 1u) ? ~leaf_lambda[0] : 0u;
    acc_hdr[1] = leaf_count;
    acc_hdr[2] = node_count;
  }
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < node_count; p += gridDim.x * blockDim.x)
    accel_node(nodes, leaf_lambda, tnodes, p);
}
__global__ void k_sah_info(rt_build_info* info, uint32_t node_count, const uint32_t* leaf_total, uint32_t levels, const uint32_t* err,
                           const uint32_t* counts) {
  info->node_count = node_count;
  info->leaf_count = *leaf_total;
  info->real_depth = levels;
  info->split_count = 0;
  info->overrun_visits = counts[2];  // leaves made because no bin boundary splits a node of >= 224 faces
  info->nondet_reads = 0;
  info->past_end_reads = 0;
  info->error = *err;
}

int sm_count() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

struct SahLayout {
  uint32_t *idx_a, *idx_b, *big_list, *counts, *rank, *base, *marks, *sums, *scalars, *keys, *err, *leaf_lambda;
  uint2 *big_a, *big_b;
  uint32_t *h_node, *h_tnode, *h_tstart, *h_tfirst, *h_keys, *h_child, *h_tleft, *h_sums;
  Bins* h_bins;
  Decision* h_dec;
  Split* h_split;
  uint32_t h_cap, t_cap;
  Item *box_a, *box_b;
  SNode* table;
  rt_build_info* lb_info;
  uint32_t* lb_codes;
  void* lb_scratch;
  size_t lb_scratch_bytes;
  uint32_t table_cap;
};

size_t carve_sah(Carve& c, SahLayout& L, uint32_t n, uint32_t lbvh_depth, uint32_t max_nodes) {
  L.table_cap = 2 * n + 2;
  if (lbvh_depth) L.table_cap += n;  // level 0: one entry per LBVH leaf
  L.idx_a = c.take<uint32_t>(n);
  L.idx_b = c.take<uint32_t>(n);
  L.box_a = c.take<Item>(n);
  L.box_b = c.take<Item>(n);
  L.big_a = c.take<uint2>(n / kBigNode + 2);
  L.big_b = c.take<uint2>(n / kBigNode + 2);
  L.big_list = c.take<uint32_t>(n / kBigNode + 2);
  L.h_cap = n / kHugeNode + 2;
  L.t_cap = n / kTile + L.h_cap + 2;
  L.h_node = c.take<uint32_t>(L.h_cap);
  L.h_tfirst = c.take<uint32_t>(L.h_cap);
  L.h_keys = c.take<uint32_t>(8 * (size_t)L.h_cap);
  L.h_child = c.take<uint32_t>(L.h_cap);
  L.h_bins = c.take<Bins>(L.h_cap);
  L.h_dec = c.take<Decision>(L.h_cap);
  L.h_split = c.take<Split>(L.h_cap);
  L.h_tnode = c.take<uint32_t>(L.t_cap);
  L.h_tstart = c.take<uint32_t>(L.t_cap);
  L.h_tleft = c.take<uint32_t>(L.t_cap + 1);
  L.h_sums = c.take<uint32_t>(L.t_cap / 1024 + 2);
  L.counts = c.take<uint32_t>(8);
  L.table = c.take<SNode>(L.table_cap);
  L.rank = c.take<uint32_t>(L.table_cap);
  L.base = c.take<uint32_t>(n + 2);
  L.marks = c.take<uint32_t>((size_t)(n > max_nodes ? n : max_nodes) + 1);
  L.sums = c.take<uint32_t>(((size_t)(n > max_nodes ? n : max_nodes) + 1023) / 1024 + 2);
  L.scalars = c.take<uint32_t>(8);
  L.keys = c.take<uint32_t>(8);
  L.err = c.take<uint32_t>(1);
  L.leaf_lambda = c.take<uint32_t>(max_nodes);
  L.lb_info = c.take<rt_build_info>(1);
  L.lb_codes = c.take<uint32_t>(lbvh_depth ? n : 0);
  L.lb_scratch_bytes = 0;
  L.lb_scratch = nullptr;
  if (lbvh_depth) {
    rt_build_params p = {lbvh_depth, 0, 0, 0, 32};
    uint32_t mx = 0;
    rt_lbvh_scratch_bytes(n, &p, &L.lb_scratch_bytes, &mx);
    L.lb_scratch = c.take<char>(L.lb_scratch_bytes);
  }
  return c.off + 256;
}

uint32_t sah_max_nodes(uint32_t n, uint32_t lbvh_depth) {
  uint64_t m = 2ull * n + 1;  // every split adds two nodes to a tree of at most n leaves
  if (lbvh_depth) {
    rt_build_params p = {lbvh_depth, 0, 0, 0, 32};
    size_t sb = 0;
    uint32_t lm = 0;
    rt_lbvh_scratch_bytes(n, &p, &sb, &lm);
    m = (uint64_t)lm + 2ull * n + 1;
  }
  return (uint32_t)(m > 0xFFFFFFF0ull ? 0xFFFFFFF0ull : m);
}

}  // namespace
}  // namespace rt

using namespace rt;

extern "C" rt_status rt_sah_sizes(uint32_t face_count, uint32_t lbvh_depth, size_t* scratch_bytes, uint32_t* max_nodes) {
  if (!scratch_bytes || face_count == 0 || face_count > 0x3FFFFFFFu || lbvh_depth > 32) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t mx = sah_max_nodes(face_count, lbvh_depth);
  Carve c(nullptr, 0);
  SahLayout L;
  *scratch_bytes = carve_sah(c, L, face_count, lbvh_depth, mx);
  if (max_nodes) *max_nodes = mx;
  return RT_OK;
}

extern "C" rt_status rt_sah_build(const rt_sah_desc* d, rt_stream stream) {
  if (!d || d->face_count == 0 || !d->vertices || !d->faces_in || !d->faces_out || !d->boxes || !d->indices || !d->nodes ||
      !d->info || d->max_nodes == 0 || d->lbvh_depth > 32 || d->face_count > 0x3FFFFFFFu)
    return RT_ERR_INVALID_ARGUMENT;
  if ((const void*)d->faces_out == (const void*)d->faces_in) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  const uint32_t n = d->face_count;
  const uint32_t mx = sah_max_nodes(n, d->lbvh_depth);
  size_t need = 0;
  rt_sah_sizes(n, d->lbvh_depth, &need, nullptr);
  if (!d->scratch || d->scratch_bytes < need) return RT_ERR_SCRATCH_TOO_SMALL;
  if (d->max_nodes < mx) return RT_ERR_CAPACITY;
  if (d->accel) {
    size_t ab = 0;
    rt_lbvh_accel_bytes(n, &ab);
    if (d->accel_bytes < ab) return RT_ERR_SCRATCH_TOO_SMALL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  Carve c(d->scratch, d->scratch_bytes);
  SahLayout L;
  carve_sah(c, L, n, d->lbvh_depth, mx);
  const int sms = sm_count();
  const uint32_t grid = (uint32_t)hmin<uint64_t>((n + 255) / 256, (uint64_t)sms * 8);
  float* hit = (float*)L.scalars;  // 8 floats, then reused
  if (cudaMemsetAsync(L.err, 0, 4, st) != cudaSuccess) return RT_ERR_CUDA;
  if (cudaMemsetAsync(L.counts, 0, 32, st) != cudaSuccess) return RT_ERR_CUDA;
  uint32_t first_base = 1, roots = 1;
  if (d->lbvh_depth == 0) {
    rt_status s = rt_mesh_boxes(d->vertices, d->faces_in, n, d->boxes, d->indices, stream);
    if (s != RT_OK) return s;
    // the root's box: the caller's hit box or the vertices' min / max
    if (d->hitbox) {
      if (cudaMemcpyAsync(hit, d->hitbox, 32, cudaMemcpyHostToDevice, st) != cudaSuccess) return RT_ERR_CUDA;
    } else {
      const uint32_t init[8] = {~0u, ~0u, ~0u, ~0u, 0u, 0u, 0u, 0u};
      if (d->vertex_count == 0) return RT_ERR_INVALID_ARGUMENT;
      if (cudaMemcpyAsync(L.keys, init, 32, cudaMemcpyHostToDevice, st) != cudaSuccess) return RT_ERR_CUDA;
      k_vertex_bounds<<<(uint32_t)hmin<uint64_t>((d->vertex_count + 255) / 256, (uint64_t)sms * 4), 256, 0, st>>>(
          (const float4*)d->vertices, d->vertex_count, L.keys);
      k_keys_to_box<<<1, 32, 0, st>>>(L.keys, hit);
      note_launch(2);
    }
    k_sah_init<<<grid, 256, 0, st>>>((const float4*)d->boxes, n, hit, L.idx_a, L.box_a, L.table, L.counts);
    note_launch();
    if (n > kBigNode) {
      const uint2 root = make_uint2(0u, n);
      if (cudaMemcpyAsync(L.big_a, &root, 8, cudaMemcpyHostToDevice, st) != cudaSuccess) return RT_ERR_CUDA;
    }
  } else {
    rt_build_desc b = {};
    b.vertices = d->vertices; b.vertex_count = d->vertex_count; b.face_count = n; b.faces_in = d->faces_in;
    b.faces_out = nullptr; b.hitbox = d->hitbox; b.params = rt_build_params{d->lbvh_depth, 0, 0, 0, 32};
    b.boxes = d->boxes; b.indices = d->indices; b.codes = L.lb_codes; b.nodes = d->nodes; b.max_nodes = d->max_nodes;
    b.tris = nullptr; b.info = L.lb_info; b.scratch = L.lb_scratch; b.scratch_bytes = L.lb_scratch_bytes;
    rt_status s = rt_lbvh_build(&b, stream);
    if (s != RT_OK) return s;
    rt_build_info hi;
    if (cudaMemcpyAsync(&hi, L.lb_info, sizeof(hi), cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return RT_ERR_CUDA;
    if (hi.error) return RT_ERR_CAPACITY;
    const uint32_t m = hi.node_count;
    first_base = m;
    roots = hi.leaf_count;
    k_hyb_items<<<grid, 256, 0, st>>>((const float4*)d->boxes, d->indices, n, L.idx_a, L.box_a);
    k_hyb_leaf_flags<<<(m + 255) / 256, 256, 0, st>>>(d->nodes, m, L.marks);
    note_launch(2);
    excl_scan(L.marks, m, L.sums, nullptr, st);
    const uint32_t init[3] = {roots, 0, 0};
    if (cudaMemcpyAsync(L.counts, init, 12, cudaMemcpyHostToDevice, st) != cudaSuccess) return RT_ERR_CUDA;
    k_hyb_roots<<<(m + 255) / 256, 256, 0, st>>>(d->nodes, m, L.marks, L.table, L.big_a, L.counts);
    note_launch();
  }
  RT_CHECK_LAUNCH();

  // levels
  std::vector<uint32_t> level_start;
  uint32_t begin = 0, end = roots;
  uint32_t host_counts[3];
  if (cudaMemcpyAsync(host_counts, L.counts, 12, cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return RT_ERR_CUDA;
  uint32_t nbig = host_counts[1];
  uint32_t* idx_in = L.idx_a;
  uint32_t* idx_out = L.idx_b;
  Item* box_in = L.box_a;
  Item* box_out = L.box_b;
  uint2* big_cur = L.big_a;
  uint2* big_next = L.big_b;
  std::vector<uint2> bigs;
  std::vector<uint32_t> regular, h_node, h_tfirst, t_node, t_start;
  while (begin < end) {
    level_start.push_back(begin);
    // this level's big nodes: a CTA each, or tiles of several CTAs when huge
    bigs.resize(nbig);
    regular.clear(); h_node.clear(); h_tfirst.clear(); t_node.clear(); t_start.clear();
    if (nbig) {
      if (cudaMemcpyAsync(bigs.data(), big_cur, (size_t)nbig * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        return RT_ERR_CUDA;
    }
    std::vector<SNode> firsts;  // first position of each huge node, read below
    for (const uint2& bg : bigs) {
      if (bg.y > kHugeNode && h_node.size() < L.h_cap) h_node.push_back(bg.x);
      else regular.push_back(bg.x);
    }
    const uint32_t H = (uint32_t)h_node.size();
    if (H) {
      firsts.resize(H);
      for (uint32_t h = 0; h < H; ++h)
        if (cudaMemcpyAsync(&firsts[h], L.table + h_node[h], sizeof(SNode), cudaMemcpyDeviceToHost, st) != cudaSuccess) return RT_ERR_CUDA;
      if (cudaStreamSynchronize(st) != cudaSuccess) return RT_ERR_CUDA;
      for (uint32_t h = 0; h < H; ++h) {
        h_tfirst.push_back((uint32_t)t_node.size());
        for (uint32_t o = 0; o < firsts[h].count; o += kTile) {
          t_node.push_back(h);
          t_start.push_back(firsts[h].first + o);
        }
      }
    }
    const uint32_t tiles = (uint32_t)t_node.size();
    if (tiles > L.t_cap) return RT_ERR_CAPACITY;
    const uint32_t zero = 0;
    if (cudaMemcpyAsync(L.counts + 1, &zero, 4, cudaMemcpyHostToDevice, st) != cudaSuccess) return RT_ERR_CUDA;
    if (!regular.empty() &&
        cudaMemcpyAsync(L.big_list, regular.data(), regular.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
      return RT_ERR_CUDA;
    LevelArgs A;
    A.table = L.table; A.table_count = L.counts; A.big_next = big_next; A.big_cur = L.big_list; A.level_begin = begin; A.level_end = end;
    A.idx_in = idx_in; A.box_in = box_in; A.idx_out = idx_out; A.box_out = box_out; A.final_idx = d->indices; A.err = L.err;
    A.table_cap = L.table_cap;
    if (H) {
      if (cudaMemcpyAsync(L.h_node, h_node.data(), H * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(L.h_tfirst, h_tfirst.data(), H * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(L.h_tnode, t_node.data(), tiles * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(L.h_tstart, t_start.data(), tiles * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return RT_ERR_CUDA;
      HugeArgs G;
      G.node = L.h_node; G.tnode = L.h_tnode; G.tstart = L.h_tstart; G.tfirst = L.h_tfirst; G.keys = L.h_keys; G.bins = L.h_bins;
      G.dec = L.h_dec; G.split = L.h_split; G.child = L.h_child; G.tleft = L.h_tleft; G.H = H; G.tiles = tiles;
      k_huge_reset<<<H, 64, 0, st>>>(G);
      k_huge_bounds<<<tiles, kCta, 0, st>>>(A, G);
      k_huge_bins<<<tiles, kCta, 0, st>>>(A, G);
      k_huge_decide<<<H, 32, 0, st>>>(A, G);
      k_huge_count<<<tiles, kCta, 0, st>>>(A, G);
      note_launch(5);
      excl_scan(L.h_tleft, tiles, L.h_sums, nullptr, st);
      k_huge_scatter<<<tiles, kCta, 0, st>>>(A, G);
      note_launch();
    }
    if (!regular.empty()) {
      k_sah_big<<<(uint32_t)regular.size(), kCta, 0, st>>>(A, (uint32_t)regular.size());
      note_launch();
    }
    k_sah_small<<<(end - begin + 7) / 8, kCta, 0, st>>>(A);
    note_launch();
    RT_CHECK_LAUNCH();
    if (cudaMemcpyAsync(host_counts, L.counts, 12, cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return RT_ERR_CUDA;
    begin = end;
    end = host_counts[0] < L.table_cap ? host_counts[0] : L.table_cap;
    nbig = host_counts[1];
    std::swap(idx_in, idx_out);
    std::swap(box_in, box_out);
    std::swap(big_cur, big_next);
  }
  const uint32_t total = end;
  const uint32_t levels = (uint32_t)level_start.size();
  level_start.push_back(total);

  // numbering: split counts bottom-up, subtree bases, ranks top-down
  for (int l = (int)levels - 1; l >= 0; --l) {
    const uint32_t b = level_start[l], e = level_start[l + 1];
    k_sah_internal<<<(uint32_t)hmin<uint64_t>((e - b + 255) / 256, (uint64_t)sms * 8), 256, 0, st>>>(L.table, b, e);
  }
  note_launch(levels);
  k_sah_base_in<<<(roots + 255) / 256, 256, 0, st>>>(L.table, roots, L.base);
  note_launch();
  excl_scan(L.base, roots, L.sums, L.scalars + 4, st);
  for (uint32_t l = 0; l < levels; ++l) {
    const uint32_t b = level_start[l], e = level_start[l + 1];
    k_sah_rank<<<(uint32_t)hmin<uint64_t>((e - b + 255) / 256, (uint64_t)sms * 8), 256, 0, st>>>(L.table, b, e, L.rank, L.base, first_base);
  }
  note_launch(levels);
  // node count = first_base + 2 * (all splits) = first_base + scan total
  uint32_t splits2 = 0;
  if (cudaMemcpyAsync(&splits2, L.scalars + 4, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return RT_ERR_CUDA;
  const uint32_t node_count = first_base + splits2;
  if (cudaMemsetAsync(L.marks, 0, (size_t)n * 4 + 4, st) != cudaSuccess) return RT_ERR_CUDA;
  k_sah_write<<<(uint32_t)hmin<uint64_t>((total + 255) / 256, (uint64_t)sms * 8), 256, 0, st>>>(L.table, total, L.rank, L.base, first_base,
                                                                                              d->nodes, d->max_nodes, L.marks, L.err);
  note_launch();
  // leaf index of every position that starts a leaf: exclusive scan of the marks
  excl_scan(L.marks, n, L.sums, L.scalars + 5, st);
  AccelLayout AL = {};
  if (d->accel) {
    Carve ca(d->accel, d->accel_bytes);
    carve_accel(ca, AL, n);
  }
  k_sah_leaves<<<(uint32_t)hmin<uint64_t>(((uint64_t)node_count * 32 + 255) / 256, (uint64_t)sms * 16), 256, 0, st>>>(
      d->nodes, node_count, L.marks, d->indices, (const uint4*)d->faces_in, (const float4*)d->vertices, (uint4*)d->faces_out,
      (float4*)d->tris, AL.leaves, AL.groups, L.leaf_lambda, n, L.err);
  note_launch();
  uint32_t leaf_total = 0;
  if (cudaMemcpyAsync(&leaf_total, L.scalars + 5, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return RT_ERR_CUDA;
  if (d->accel) {
    k_sah_accel<<<(uint32_t)hmin<uint64_t>((node_count + 255) / 256, (uint64_t)sms * 8), 256, 0, st>>>(d->nodes, node_count, leaf_total,
                                                                                                        L.leaf_lambda, AL.tnodes, AL.hdr);
    note_launch();
    k_wide_nodes<<<(uint32_t)hmin<uint64_t>((node_count + 255) / 256, (uint64_t)sms * 8), 256, 0, st>>>(AL.tnodes, AL.hdr, AL.wide);
    note_launch();
  }
  k_sah_info<<<1, 1, 0, st>>>(d->info, node_count, L.scalars + 5, levels, L.err, L.counts);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}
