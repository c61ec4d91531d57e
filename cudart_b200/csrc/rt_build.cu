// rt_build.cu -- LBVH build for sm_100a.
//
// Replaces CUDA_buildMeshTreeLBVH (kernels/CUDA_buildMeshTreeLBVH.cu:457-681)
// and its helpers. The reference runs ~10 launches with a host sync after
// each, copies the split list to the host, builds the topology with a
// sequential host recursion (:309-455), copies the nodes back, then runs
// real_depth full passes for the boxes. Here everything stays on the device,
// with no host round trip:
//
//   k_boxes_morton   per face: box (4-wide min/max of the 3 vertices), index,
//                    Morton code (reference 11/11/10 layout or 10/10/10)
//   radix sort       (code, index) pairs, stable (rt_sort.cu)
//   k_levels         split level of each adjacent code pair (clz of the xor)
//   radix pass       stable partition of split positions by level, which is
//                    the per-level ascending split list the recursion walks
//   k_topo_morton    one CTA: the Morton levels of the tree, level by level,
//                    with the reference's split-pointer semantics (see below);
//                    leaf counts, pre-order ranks and node ids
//   k_leaves         one warp per final leaf: expands median subtrees, writes
//                    node records, reorders faces, pre-gathers triangles
//                    {v0, e1, e2}, reduces the leaf box and records the
//                    parents of median nodes
//   k_propagate      one thread per node: each leaf climbs to the root with
//                    per-node arrival counters (the second arrival merges the
//                    two child boxes; nobody waits)
//
// Node numbering follows the reference's recursion: the k-th internal node in
// pre-order gets children 2k+1 and 2k+2. A node's pre-order rank among
// internal nodes is computed from subtree leaf counts (rank(left) = rank + 1,
// rank(right) = rank + leaves(left)).
//
// Split-pointer semantics (host recursion :360-411): each level L keeps a
// pointer into the concatenated, level-ordered split list C. A Morton visit of
// a range [a, b) at level L (b - a >= min_leaf, L < tree_depth) is a leaf when
// the pointer sits exactly at the start of level L+1's list; otherwise the
// pointer advances past every entry <= a -- it may run into deeper levels'
// lists -- and the entry found cuts the range if it is < b. Because visits at a
// level come in increasing a, the pointer after a visit is "the first index at
// or after start(L) holding a value > a"; it sticks at start(L+1) exactly when
// the first visit with a >= last(P_L) finds C[start(L+1)] > a. Both facts make
// every visit of a level independent once that one visit is known.
#include "rt_device.cuh"

namespace rt {
namespace {

constexpr int kTopoThreads = 1024;
constexpr int kTopoWarps = kTopoThreads / 32;

// ----------------------------------------------------------------------------
// hit box (when the caller gives none): min/max over all vertices
// ----------------------------------------------------------------------------
__global__ void k_set_hitbox(float4* hit, float4 mn, float4 mx) {
  hit[0] = mn;
  hit[1] = mx;
}

// Hit box over all vertices: each block reduces its grid-stride share to a partial box; the block that finishes
// last (a counter the host zeroes) combines the partials, strided over its threads and then as a shared-memory
// tree, and writes hit[0..1]. Nothing waits for it inside the launch.
__global__ __launch_bounds__(256) void k_hitbox(const float4* __restrict__ v, uint32_t count, float4* __restrict__ partial,
                                               uint32_t* __restrict__ done, float4* __restrict__ hit) {
  // four loads in flight per thread, one accumulator each
  float4 mn[4], mx[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    mn[k] = make_float4(kHuge, kHuge, kHuge, kHuge);
    mx[k] = make_float4(-kHuge, -kHuge, -kHuge, -kHuge);
  }
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  for (; (uint64_t)i + 3ull * stride < count; i += 4 * stride) {
    float4 p[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) p[k] = ldg4(v + i + k * stride);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      mn[k] = f4min(mn[k], p[k]);
      mx[k] = f4max(mx[k], p[k]);
    }
  }
  for (; i < count; i += stride) {
    const float4 p = ldg4(v + i);
    mn[0] = f4min(mn[0], p);
    mx[0] = f4max(mx[0], p);
  }
  __shared__ float4 s_mn[256], s_mx[256];
  __shared__ uint32_t s_last;
  s_mn[threadIdx.x] = f4min(f4min(mn[0], mn[1]), f4min(mn[2], mn[3]));
  s_mx[threadIdx.x] = f4max(f4max(mx[0], mx[1]), f4max(mx[2], mx[3]));
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s_mn[threadIdx.x] = f4min(s_mn[threadIdx.x], s_mn[threadIdx.x + o]);
      s_mx[threadIdx.x] = f4max(s_mx[threadIdx.x], s_mx[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s_mn[0];
    partial[2 * blockIdx.x + 1] = s_mx[0];
    __threadfence();
    s_last = atomicAdd(done, 1u) == gridDim.x - 1 ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  float4 a = make_float4(kHuge, kHuge, kHuge, kHuge), b = make_float4(-kHuge, -kHuge, -kHuge, -kHuge);
  for (uint32_t j = threadIdx.x; j < gridDim.x; j += blockDim.x) {
    a = f4min(a, __ldcg(partial + 2 * j));
    b = f4max(b, __ldcg(partial + 2 * j + 1));
  }
  s_mn[threadIdx.x] = a;
  s_mx[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s_mn[threadIdx.x] = f4min(s_mn[threadIdx.x], s_mn[threadIdx.x + o]);
      s_mx[threadIdx.x] = f4max(s_mx[threadIdx.x], s_mx[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    hit[0] = s_mn[0];
    hit[1] = s_mx[0];
  }
}

// ----------------------------------------------------------------------------
// boxes + Morton + iota
// ----------------------------------------------------------------------------
// kernels/CUDA_calcMeshBoxes.cu:30-58 (boxes, iota) fused with
// kernels/CUDA_buildMeshTreeLBVH.cu:115-173 (Morton code of the box centre).
// code_counts (optional, 4 x 256 zeroed words): the digit counts of the codes for the four 8-bit passes of their
// sort, so that the sort need not read the codes once more to count them.
__global__ __launch_bounds__(256) void k_boxes_morton(const float4* __restrict__ verts, const uint4* __restrict__ faces, uint32_t n,
                                                     const float4* __restrict__ hit, int layout, float4* __restrict__ boxes,
                                                     uint32_t* __restrict__ codes, uint32_t* __restrict__ idx,
                                                     uint32_t* __restrict__ code_counts) {
  __shared__ uint32_t s_cc[4 * 256];
  if (code_counts) {
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) s_cc[i] = 0;
    __syncthreads();
  }
  const float4 hmin = codes ? hit[0] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 hmax = codes ? hit[1] : make_float4(1.f, 1.f, 1.f, 1.f);
  const float lx = hmax.x - hmin.x, ly = hmax.y - hmin.y, lz = hmax.z - hmin.z;
  const float sx = (layout == 30 ? 1023.0f : 2047.0f) / lx;
  const float sy = (layout == 30 ? 1023.0f : 2047.0f) / ly;
  const float sz = 1023.0f / lz;
  auto face = [&](uint32_t k, const float4& v0, const float4& v1, const float4& v2) {
    const float4 mn = f4min(f4min(v0, v1), v2);
    const float4 mx = f4max(f4max(v0, v1), v2);
    boxes[2 * (size_t)k] = mn;
    boxes[2 * (size_t)k + 1] = mx;
    if (idx) idx[k] = k;
    if (codes) {
      const float cx = 0.5f * (mn.x + mx.x), cy = 0.5f * (mn.y + mx.y), cz = 0.5f * (mn.z + mx.z);
      const uint32_t qx = f2u_sat((cx - hmin.x) * sx);
      const uint32_t qy = f2u_sat((cy - hmin.y) * sy);
      const uint32_t qz = f2u_sat((cz - hmin.z) * sz);
      const uint32_t code = spread_code(qx, qy, qz, layout);
      codes[k] = code;
      if (code_counts) {
#pragma unroll
        for (int p = 0; p < 4; ++p) atomicAdd(&s_cc[p * 256 + ((code >> (8 * p)) & 255u)], 1u);
      }
    }
  };
  // two faces per iteration: their face and vertex loads are in flight together
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += 2 * stride) {
    const uint32_t k2 = k + stride;
    const bool two = k2 < n;
    const uint4 f = ldg4(faces + k);
    const uint4 f2 = two ? ldg4(faces + k2) : f;
    const float4 v0 = ldg4(verts + f.x), v1 = ldg4(verts + f.y), v2 = ldg4(verts + f.z);
    const float4 w0 = ldg4(verts + f2.x), w1 = ldg4(verts + f2.y), w2 = ldg4(verts + f2.z);
    face(k, v0, v1, v2);
    if (two) face(k2, w0, w1, w2);
  }
  if (code_counts) {
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x)
      if (s_cc[i]) atomicAdd(code_counts + i, s_cc[i]);
  }
}

// ----------------------------------------------------------------------------
// split levels: key = clz(code[i] ^ code[i+1]) (32 when equal), value = i + 1
// (kernels/CUDA_buildMeshTreeLBVH.cu:175-233)
// ----------------------------------------------------------------------------
// lev_counts (256 zeroed words): how many pairs have each level, the digit counts of the level sort's one pass.
__global__ __launch_bounds__(256) void k_levels(const uint32_t* __restrict__ codes, uint32_t n, uint32_t* __restrict__ lev,
                                               uint32_t* __restrict__ pos, uint32_t* __restrict__ lev_counts) {
  __shared__ uint32_t s_lc[33];
  if (threadIdx.x < 33) s_lc[threadIdx.x] = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n; i += gridDim.x * blockDim.x) {
    uint32_t d = __ldg(codes + i) ^ __ldg(codes + i + 1);
    const uint32_t l = d ? (uint32_t)__clz(d) : 32u;
    lev[i] = l;
    pos[i] = i + 1;
    atomicAdd(&s_lc[l], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 33 && s_lc[threadIdx.x]) atomicAdd(lev_counts + threadIdx.x, s_lc[threadIdx.x]);
}

// ----------------------------------------------------------------------------
// Morton top tree (one CTA)
// ----------------------------------------------------------------------------
struct TopoArgs {
  const uint32_t* C;         // split positions, level ordered
  const uint32_t* lev_count; // [33] per-level counts (level 32 = no split)
  uint32_t n, D, min_leaf, max_leaf, complete;
  uint32_t cap_m;
  // BFS arrays
  uint32_t *ra, *rb, *parent, *info, *child, *leaves, *mleaves, *rank, *lambda, *ord, *id;
  // Morton leaves in position order
  uint32_t* ml_lambda;
  uint4* ml_rec;     // (node id, first, count, depth | median << 31)
  uint32_t* ml_rank; // pre-order rank (median roots)
  uint32_t* parent_id; // [max_nodes] parent node id of Morton nodes
  uint32_t* nodes;     // bvnode words
  uint32_t max_nodes;
  uint32_t* hdr;       // [16] header: 0 leaf_count, 1 morton_leaves, 2 node_count, 3 real_depth, 4 split_count,
                       //             5 overrun, 6 nondet, 7 past_end, 8 error
  const uint32_t* level_hist;   // optional [33] pair counts of this mesh's levels (batched build); else lev_count
  uint32_t level_base;          // with level_hist: where this mesh's level lists start in C
  uint32_t pos_base;            // first position of this mesh (0 for a single mesh)
};

__device__ __forceinline__ void topo_morton(const TopoArgs& A) {
  __shared__ uint32_t s_start[34];
  __shared__ uint32_t s_level_lo[34];
  __shared__ uint32_t s_warp[kTopoWarps];
  __shared__ uint32_t s_vstar, s_stuck, s_levels;
  __shared__ uint32_t s_overrun, s_nondet, s_past, s_err, s_depth;
  const uint32_t tid = threadIdx.x;
  if (tid == 0) {
    if (A.level_hist) {
      uint32_t acc = A.level_base;
      for (int l = 0; l < 33; ++l) { s_start[l] = acc; acc += (l < 32) ? A.level_hist[l] : 0u; }
    } else {
      uint32_t acc = 0;
      for (int l = 0; l < 33; ++l) { s_start[l] = acc; acc += (l < 32) ? A.lev_count[l] : 0u; }
    }
    s_start[33] = s_start[32];
    s_overrun = s_nondet = s_past = s_err = s_depth = 0;
    A.ra[0] = A.pos_base; A.rb[0] = A.pos_base + A.n; A.parent[0] = kNone;
  }
  __syncthreads();
  const uint32_t S = s_start[32];
  const uint32_t D = A.D;
  uint32_t lo = 0, hi = 1, L = 0;
  for (; lo < hi; ++L) {
    if (tid == 0) { s_level_lo[L] = lo; s_vstar = kNone; s_stuck = 0; }
    __syncthreads();
    const bool nonempty = L < 32 && s_start[L] < s_start[L + 1];
    const uint32_t lastL = nonempty ? __ldg(A.C + s_start[L + 1] - 1) : 0u;
    if (nonempty && L < D) {
      for (uint32_t i = lo + tid; i < hi; i += kTopoThreads) {
        uint32_t a = A.ra[i], b = A.rb[i];
        if (b - a >= A.min_leaf && a >= lastL) atomicMin(&s_vstar, i);
      }
    }
    __syncthreads();
    if (tid == 0 && s_vstar != kNone) {
      uint32_t j = split_scan(A.C, s_start, L, A.ra[s_vstar]);
      s_stuck = (j == s_start[L + 1]) ? 1u : 0u;
    }
    __syncthreads();
    uint32_t running = hi;
    for (uint32_t base = lo; base < hi; base += kTopoThreads) {
      const uint32_t i = base + tid;
      bool internal = false;
      uint32_t a = 0, b = 0, s = 0, inf = 0;
      if (i < hi) {
        a = A.ra[i]; b = A.rb[i];
        const bool visit = (b - a >= A.min_leaf) && L < D && nonempty;
        if (visit && !(s_vstar != kNone && i > s_vstar && s_stuck)) {
          uint32_t j = split_scan(A.C, s_start, L, a);
          s = (j < S) ? __ldg(A.C + j) : kNone;
          internal = s < b;
          if (j >= s_start[L + 1]) atomicAdd(&s_overrun, 1u);
          if (j < S && j >= s_start[min(D + 1, 32u)]) atomicAdd(&s_nondet, 1u);
          if (j == S) atomicAdd(&s_past, 1u);
        }
        const bool median = !internal && A.complete && (b - a > A.max_leaf);
        inf = L | (internal ? 0x100u : 0u) | (median ? 0x200u : 0u);
      }
      uint32_t total;
      uint32_t ex = block_excl_scan_nt<kTopoThreads>(internal ? 2u : 0u, s_warp, total);
      if (i < hi) {
        uint32_t c = kNone;
        if (internal) {
          c = running + ex;
          if (c + 1 < A.cap_m) {
            A.ra[c] = a; A.rb[c] = s; A.ra[c + 1] = s; A.rb[c + 1] = b;
            A.parent[c] = i; A.parent[c + 1] = i;
          } else {
            // cannot happen (the Morton levels hold at most min(2^(D+1), 2n) - 1
            // nodes); kept as a guarded leaf so that no index leaves its array
            atomicOr(&s_err, (uint32_t)RT_DEVERR_MORTON_CAPACITY);
            c = kNone;
            inf &= ~0x100u;
          }
        }
        A.child[i] = c;
        A.info[i] = inf;
      }
      running += total;
    }
    __syncthreads();
    lo = hi;
    hi = min(running, A.cap_m);
  }
  if (tid == 0) { s_level_lo[L] = lo; s_levels = L; }
  __syncthreads();
  const uint32_t levels = s_levels;
  const uint32_t maxl = A.max_leaf;

  // bottom-up: leaves (final tree) and Morton leaves per subtree
  for (int l = (int)levels - 1; l >= 0; --l) {
    for (uint32_t i = s_level_lo[l] + tid; i < s_level_lo[l + 1]; i += kTopoThreads) {
      uint32_t inf = A.info[i];
      if (inf & 0x100u) {
        uint32_t c = A.child[i];
        A.leaves[i] = A.leaves[c] + A.leaves[c + 1];
        A.mleaves[i] = A.mleaves[c] + A.mleaves[c + 1];
      } else {
        uint32_t size = A.rb[i] - A.ra[i];
        A.leaves[i] = (inf & 0x200u) ? median_leaves(size, maxl) : 1u;
        A.mleaves[i] = 1u;
      }
    }
    __syncthreads();
  }
  // top-down: rank, lambda (leaves to the left), Morton-leaf ordinal, node id
  if (tid == 0) { A.rank[0] = 0; A.lambda[0] = 0; A.ord[0] = 0; A.id[0] = 0; }
  __syncthreads();
  for (uint32_t l = 0; l < levels; ++l) {
    for (uint32_t i = s_level_lo[l] + tid; i < s_level_lo[l + 1]; i += kTopoThreads) {
      if (A.info[i] & 0x100u) {
        uint32_t c = A.child[i];
        uint32_t r = A.rank[i], lam = A.lambda[i], o = A.ord[i];
        uint32_t ll = A.leaves[c];
        A.rank[c] = r + 1; A.lambda[c] = lam; A.ord[c] = o; A.id[c] = 2 * r + 1;
        A.rank[c + 1] = r + ll; A.lambda[c + 1] = lam + ll; A.ord[c + 1] = o + A.mleaves[c]; A.id[c + 1] = 2 * r + 2;
      }
    }
    __syncthreads();
  }
  // emit Morton node records and the Morton-leaf table
  const uint32_t total_m = s_level_lo[levels];
  for (uint32_t i = tid; i < total_m; i += kTopoThreads) {
    const uint32_t inf = A.info[i];
    const uint32_t lvl = inf & 0xFFu;
    const uint32_t nid = A.id[i];
    if (nid >= A.max_nodes) { atomicOr(&s_err, (uint32_t)RT_DEVERR_NODE_CAPACITY); continue; }
    A.parent_id[nid] = (i == 0) ? kNone : A.id[A.parent[i]];
    if (inf & 0x100u) {
      uint2 w = make_uint2((lvl % 3u) << 1, 2 * A.rank[i] + 1);
      *(uint2*)(A.nodes + 8 * (size_t)nid) = w;
    } else {
      const uint32_t k = A.ord[i];
      const uint32_t first = A.ra[i], cnt = A.rb[i] - A.ra[i];
      const bool median = (inf & 0x200u) != 0;
      A.ml_lambda[k] = A.lambda[i];
      A.ml_rec[k] = make_uint4(nid, first, cnt, lvl | (median ? 0x80000000u : 0u));
      A.ml_rank[k] = A.rank[i];
      uint32_t depth = lvl + (median ? median_depth(cnt, maxl) : 0u) + 1u;
      atomicMax(&s_depth, depth);
    }
  }
  __syncthreads();
  if (tid == 0) {
    const uint32_t leaves = A.leaves[0];
    A.hdr[0] = leaves;
    A.hdr[1] = A.mleaves[0];
    A.hdr[2] = 2 * leaves - 1;
    A.hdr[3] = s_depth;
    A.hdr[4] = S - s_start[0];
    A.hdr[5] = s_overrun;
    A.hdr[6] = s_nondet;
    A.hdr[7] = s_past;
    A.hdr[8] = s_err | ((2 * leaves - 1 > A.max_nodes) ? (uint32_t)RT_DEVERR_NODE_CAPACITY : 0u);
  }
}

__global__ __launch_bounds__(kTopoThreads) void k_topo_morton(TopoArgs A) { topo_morton(A); }

// ----------------------------------------------------------------------------
// leaves: one warp per final leaf
// ----------------------------------------------------------------------------
struct LeafArgs {
  const float4* verts;
  const uint4* faces_in;
  uint4* faces_out;      // may be null (tree_complete == 0)
  float4* tris;          // may be null
  const uint32_t* indices;
  const uint32_t* ml_lambda;
  const uint4* ml_rec;
  const uint32_t* ml_rank;
  uint32_t* parent_id;
  uint32_t* arrive;
  uint32_t* nodes;
  uint32_t max_nodes;
  uint32_t max_leaf;
  const uint32_t* hdr;
  uint32_t* err;
  // traversal blob (optional): leaf table in leaf order, 8-triangle group boxes
  uint4* acc_leaves;
  float4* acc_groups;
  uint32_t* leaf_lambda;  // node id -> leaf order index
  uint32_t pos_base;      // first position of this mesh (node records store positions relative to it)
  uint32_t vert_base;     // first vertex of this mesh (faces index vertices relative to it)
  uint32_t* local_indices; // optional: indices[i] - pos_base written here (batched build)
  uint32_t parent_cap;     // entries of parent_id (median nodes' parents are written here)
};

constexpr int kMaxMedianDepth = 40;
// One final leaf (leaf-order index g of its mesh), processed by one warp.
// `hint` (lane 0's) is the Morton leaf of the warp's previous leaf of the same
// mesh, or ~0u: a warp walking consecutive leaves then finds each one's Morton
// leaf in a step or two instead of a binary search.
__device__ __forceinline__ void leaf_body(const LeafArgs& A, const uint32_t g, uint32_t& hint) {
  const uint32_t lane = lane_id();
  const uint32_t mleaf_count = A.hdr[1];
  {
    uint32_t leaf_id = 0, first = 0, cnt = 0;
    int plen = 0;  // median levels walked
    if (lane == 0) {
      // Morton leaf owning global leaf slot g: last k with ml_lambda[k] <= g
      // (ml_lambda is non-decreasing)
      uint32_t lo = 0;
      if (hint < mleaf_count && A.ml_lambda[hint] <= g) {
        lo = hint;
        while (lo + 1 < mleaf_count && A.ml_lambda[lo + 1] <= g) ++lo;
      } else {
        uint32_t hi = mleaf_count - 1;
        while (lo < hi) {
          uint32_t mid = (lo + hi + 1) >> 1;
          if (A.ml_lambda[mid] <= g) lo = mid; else hi = mid - 1;
        }
      }
      hint = lo;
      const uint4 rec = A.ml_rec[lo];
      leaf_id = rec.x; first = rec.y; cnt = rec.z;  // first: absolute position
      if (rec.w & 0x80000000u) {
        uint32_t q = g - A.ml_lambda[lo];
        uint32_t rank = A.ml_rank[lo];
        uint32_t depth = rec.w & 0xFFFFu;
        uint32_t nid = rec.x, size = rec.z, a = rec.y;
        while (size >= A.max_leaf && plen < kMaxMedianDepth) {
          const uint32_t left = size >> 1, right = size - left;
          const uint32_t ll = median_leaves(left, A.max_leaf);
          // the subtree's first leaf writes the internal record and its children's parent ids
          if (q == 0 && nid < A.max_nodes) {
            *(uint2*)(A.nodes + 8 * (size_t)nid) = make_uint2((depth % 3u) << 1, 2 * rank + 1);
            if (2 * rank + 2 < A.parent_cap) {
              A.parent_id[2 * rank + 1] = nid;
              A.parent_id[2 * rank + 2] = nid;
            }
          }
          ++plen;
          if (q < ll) { nid = 2 * rank + 1; rank = rank + 1; size = left; }
          else { q -= ll; nid = 2 * rank + 2; rank = rank + ll; a += left; size = right; }
          ++depth;
        }
        leaf_id = nid; first = a; cnt = size;
      }
    }
    leaf_id = __shfl_sync(0xffffffffu, leaf_id, 0);
    first = __shfl_sync(0xffffffffu, first, 0);
    cnt = __shfl_sync(0xffffffffu, cnt, 0);

    float3 mn = make_float3(kHuge, kHuge, kHuge), mx = make_float3(-kHuge, -kHuge, -kHuge);
    const uint32_t lfirst = first - A.pos_base;  // position inside the mesh
    const uint32_t gbase = (lfirst >> 3) + g;      // leaf g's groups: disjoint across leaves, no scan needed
    if (A.acc_leaves && lane == 0) {
      A.acc_leaves[g] = make_uint4(lfirst, cnt, gbase, leaf_id);
      A.leaf_lambda[leaf_id] = g;
    }
    for (uint32_t base = 0; base < cnt; base += 32) {
      const uint32_t i = first + base + lane;
      float3 tmn = make_float3(kHuge, kHuge, kHuge), tmx = make_float3(-kHuge, -kHuge, -kHuge);
      if (base + lane < cnt) {
        const uint32_t orig = A.indices[i];
        const uint4 f = ldg4(A.faces_in + orig);
        const float4 v0 = ldg4(A.verts + A.vert_base + f.x), v1 = ldg4(A.verts + A.vert_base + f.y), v2 = ldg4(A.verts + A.vert_base + f.z);
        if (A.local_indices) A.local_indices[i] = orig - A.pos_base;
        if (A.faces_out) A.faces_out[i] = f;
        if (A.tris) {
          float4 e1 = make_float4(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z, 0.0f);
          float4 e2 = make_float4(v2.x - v0.x, v2.y - v0.y, v2.z - v0.z, 0.0f);
          A.tris[3 * (size_t)i + 0] = make_float4(v0.x, v0.y, v0.z, 0.0f);
          A.tris[3 * (size_t)i + 1] = e1;
          A.tris[3 * (size_t)i + 2] = e2;
        }
        tmn = make_float3(fmin_sel(fmin_sel(v0.x, v1.x), v2.x), fmin_sel(fmin_sel(v0.y, v1.y), v2.y), fmin_sel(fmin_sel(v0.z, v1.z), v2.z));
        tmx = make_float3(fmax_sel(fmax_sel(v0.x, v1.x), v2.x), fmax_sel(fmax_sel(v0.y, v1.y), v2.y), fmax_sel(fmax_sel(v0.z, v1.z), v2.z));
      }
      mn = make_float3(fmin_sel(mn.x, tmn.x), fmin_sel(mn.y, tmn.y), fmin_sel(mn.z, tmn.z));
      mx = make_float3(fmax_sel(mx.x, tmx.x), fmax_sel(mx.y, tmx.y), fmax_sel(mx.z, tmx.z));
      if (A.acc_groups) {
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
          A.acc_groups[2 * gi] = make_float4(tmn.x, tmn.y, tmn.z, 0.0f);
          A.acc_groups[2 * gi + 1] = make_float4(tmx.x, tmx.y, tmx.z, 0.0f);
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn.x = fmin_sel(mn.x, __shfl_xor_sync(0xffffffffu, mn.x, o));
      mn.y = fmin_sel(mn.y, __shfl_xor_sync(0xffffffffu, mn.y, o));
      mn.z = fmin_sel(mn.z, __shfl_xor_sync(0xffffffffu, mn.z, o));
      mx.x = fmax_sel(mx.x, __shfl_xor_sync(0xffffffffu, mx.x, o));
      mx.y = fmax_sel(mx.y, __shfl_xor_sync(0xffffffffu, mx.y, o));
      mx.z = fmax_sel(mx.z, __shfl_xor_sync(0xffffffffu, mx.z, o));
    }
    if (lane == 0) {
      if (leaf_id >= A.max_nodes) { atomicOr(A.err, (uint32_t)RT_DEVERR_NODE_CAPACITY); return; }
      uint32_t* nd = A.nodes + 8 * (size_t)leaf_id;
      *(uint2*)nd = make_uint2(1u | (cnt << 1), lfirst);
      write_box(nd, mn, mx);
    }
  }
}

// Node boxes bottom-up, one thread per leaf: the leaf (its box written by the
// leaf kernel) climbs through parent_id; at each internal node the first of
// its two children to arrive stops, the second merges both children's boxes
// and climbs on. cap bounds every node id (the node array's capacity).
__device__ __forceinline__ void climb(uint32_t* __restrict__ nodes, const uint32_t* __restrict__ parent_id, uint32_t* __restrict__ arrive,
                                      uint32_t cap, uint32_t leaf) {
  uint32_t cur = leaf;
  for (;;) {
    const uint32_t p = parent_id[cur];
    if (p == kNone || p >= cap) break;
    __threadfence();
    if (atomicAdd(arrive + p, 1u) == 0u) break;
    __threadfence();
    const uint32_t c0 = __ldcg(nodes + 8 * (size_t)p + 1);
    if (c0 + 1 >= cap) break;
    const float* l = (const float*)(nodes + 8 * (size_t)c0);
    const float* r = (const float*)(nodes + 8 * (size_t)(c0 + 1));
    float lb[6], rb[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) { lb[q] = __ldcg(l + 2 + q); rb[q] = __ldcg(r + 2 + q); }
    float3 bmn, bmx;
    // kernels/CUDA_buildMeshTreeLBVH.cu:269-300: merged only when both children have a positive z extent
    if (lb[5] - lb[2] > 0.0f && rb[5] - rb[2] > 0.0f) {
      bmn = make_float3(fmin_sel(lb[0], rb[0]), fmin_sel(lb[1], rb[1]), fmin_sel(lb[2], rb[2]));
      bmx = make_float3(fmax_sel(lb[3], rb[3]), fmax_sel(lb[4], rb[4]), fmax_sel(lb[5], rb[5]));
    } else {
      bmn = make_float3(kHuge, kHuge, kHuge);
      bmx = make_float3(-kHuge, -kHuge, -kHuge);
    }
    write_box(nodes + 8 * (size_t)p, bmn, bmx);
    cur = p;
  }
}

// Bottom-up boxes of a single mesh: one thread per node, the leaves climb.
__global__ __launch_bounds__(256) void k_propagate(uint32_t* __restrict__ nodes, const uint32_t* __restrict__ parent_id,
                                                   uint32_t* __restrict__ arrive, const uint32_t* __restrict__ hdr, uint32_t cap) {
  if (hdr[8] & (RT_DEVERR_NODE_CAPACITY | RT_DEVERR_MORTON_CAPACITY)) return;
  const uint32_t node_count = min(hdr[2], cap);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < node_count; p += gridDim.x * blockDim.x)
    if (nodes[8 * (size_t)p] & 1u) climb(nodes, parent_id, arrive, cap, p);
}

__global__ __launch_bounds__(256) void k_leaves(LeafArgs A) {
  const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t leaf_count = A.hdr[0];
  if (A.hdr[8] & (RT_DEVERR_NODE_CAPACITY | RT_DEVERR_MORTON_CAPACITY)) return;
  // a contiguous run of leaves per warp (the grid is one resident wave)
  const uint32_t per = (leaf_count + nwarps - 1) / nwarps;
  const uint32_t g0 = min(leaf_count, warp_global * per), g1 = min(leaf_count, g0 + per);
  uint32_t hint = ~0u;
  for (uint32_t g = g0; g < g1; ++g) leaf_body(A, g, hint);
}

// Two-child traversal records, indexed by pre-order rank (internal node p
// with left child c has rank (c - 1) / 2): both children's padded boxes and
// references (rank for an internal child, ~leaf index for a leaf child).
__global__ __launch_bounds__(256) void k_accel_nodes(const uint32_t* __restrict__ nodes, const uint32_t* __restrict__ hdr,
                                                    const uint32_t* __restrict__ leaf_lambda, float4* __restrict__ tnodes,
                                                    float4* __restrict__ wide, uint32_t* __restrict__ acc_hdr) {
  const uint32_t node_count = hdr[2];
  if (blockIdx.x == 0 && threadIdx.x == 0) acc_hdr[kHdrClusterValid] = 0;  // set again by the cluster build, if any
  if (hdr[8] & (RT_DEVERR_NODE_CAPACITY | RT_DEVERR_MORTON_CAPACITY)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const bool root_leaf = (nodes[0] & 1u) != 0;
    acc_hdr[0] = root_leaf ? ~0u : 0u;  // root reference
    acc_hdr[1] = hdr[0];                // leaf count
    acc_hdr[2] = node_count;
  }
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < node_count; p += gridDim.x * blockDim.x)
    accel_wide_node(nodes, leaf_lambda, tnodes, wide, p);
}

__global__ void k_write_info(const uint32_t* __restrict__ hdr, const uint32_t* __restrict__ err, rt_build_info* info) {
  if (threadIdx.x != 0) return;
  info->leaf_count = hdr[0];
  info->node_count = hdr[2];
  info->real_depth = hdr[3];
  info->split_count = hdr[4];
  info->overrun_visits = hdr[5];
  info->nondet_reads = hdr[6];
  info->past_end_reads = hdr[7];
  info->error = hdr[8] | *err;
}

struct BuildLayout {
  uint32_t n, cap_m, max_nodes, tiles;
  float4* hit;
  float4* partial;
  uint32_t* codes;
  uint32_t* lev;
  uint32_t* C;
  uint32_t* lev_count;
  void* sort_scratch;
  size_t sort_bytes;
  uint32_t *ra, *rb, *parent, *info, *child, *leaves, *mleaves, *rank, *lambda, *ord, *id;
  uint32_t* ml_lambda;
  uint4* ml_rec;
  uint32_t* ml_rank;
  uint32_t* parent_id;
  uint32_t* arrive;
  uint32_t* hdr;
  uint32_t* err;
  uint32_t* leaf_lambda;
  uint4* faces_tmp;
  uint32_t* counts;  // [5 x 256]: the code sort's digit counts (4 passes), then the level sort's (1 pass)
  ClusterTemps ct;   // cluster tree build (RT_ACCEL_CLUSTERS only)
};

constexpr uint32_t kHitParts = 1184;  // 8 blocks per SM on 148 SMs
constexpr uint32_t kHitSplit = 8;     // CTAs per mesh of the batched hit box

__host__ __device__ uint32_t morton_cap_dev(uint32_t n, uint32_t D) {
  uint64_t a = (D >= 31) ? (1ull << 32) : ((1ull << (D + 1)) - 1);
  uint64_t b = 2ull * n + 1;
  uint64_t c = a < b ? a : b;
  return (uint32_t)(c + 2);
}

uint32_t morton_cap(uint32_t n, uint32_t D) {
  uint64_t a = (D >= 31) ? (1ull << 32) : ((1ull << (D + 1)) - 1);
  uint64_t b = 2ull * n + 1;
  uint64_t c = a < b ? a : b;
  return (uint32_t)(c + 2);
}

size_t carve_build(Carve& c, BuildLayout& L, uint32_t n, uint32_t D, bool need_codes, bool need_faces_tmp, bool clusters) {
  L.n = n;
  L.cap_m = morton_cap(n, D);
  L.max_nodes = 2 * n - 1;
  L.hit = c.take<float4>(2);
  L.partial = c.take<float4>(2 * kHitParts);
  L.codes = need_codes ? c.take<uint32_t>(n) : nullptr;
  L.lev = c.take<uint32_t>(n);
  L.C = c.take<uint32_t>(n);
  L.lev_count = c.take<uint32_t>(256);
  L.sort_bytes = radix_scratch_bytes(n);
  L.sort_scratch = c.take<char>(L.sort_bytes);
  uint32_t** bfs[] = {&L.ra, &L.rb, &L.parent, &L.info, &L.child, &L.leaves, &L.mleaves, &L.rank, &L.lambda, &L.ord, &L.id};
  for (auto p : bfs) *p = c.take<uint32_t>(L.cap_m);
  L.ml_lambda = c.take<uint32_t>(L.cap_m);
  L.ml_rec = c.take<uint4>(L.cap_m);
  L.ml_rank = c.take<uint32_t>(L.cap_m);
  L.parent_id = c.take<uint32_t>(L.max_nodes);
  L.arrive = c.take<uint32_t>(L.max_nodes);
  L.hdr = c.take<uint32_t>(16);
  L.err = c.take<uint32_t>(4);
  L.leaf_lambda = c.take<uint32_t>(L.max_nodes);
  L.faces_tmp = need_faces_tmp ? c.take<uint4>(n) : nullptr;
  L.counts = c.take<uint32_t>(5 * 256 + 1);  // digit counts of the code and level sorts, then the hit box's block counter
  L.ct = ClusterTemps{};
  if (clusters) carve_cluster_temps(c, L.ct, n, 1);
  return c.off + 256;
}

// SM count of the current device (cached per device).
int sm_count() {
  static std::atomic<int> cache[PerDeviceOnce::kMaxDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= PerDeviceOnce::kMaxDevices) return 148;
  int s = cache[dev].load(std::memory_order_relaxed);
  if (s <= 0) {
    if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || s <= 0) s = 148;
    cache[dev].store(s, std::memory_order_relaxed);
  }
  return s;
}

// Blocks of `kernel` (with `threads` per block and no dynamic shared memory)
// that one SM holds at once: a grid of sm_count() times this is one resident
// wave. Queried once per kernel (the first call).
template <typename K>
int resident_blocks_of(K kernel, int threads) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, 0) != cudaSuccess || nb <= 0) {
    cudaGetLastError();
    nb = 1;
  }
  return nb;
}

}  // namespace

SideStream* side_stream() {
  // one per host thread and device (a stream takes part in one capture at a time, and a thread's calls are
  // ordered, so the fork and join events of two calls never interleave); kept until the process exits
  constexpr int kMaxDevices = 64;
  thread_local SideStream per_device[kMaxDevices];
  thread_local int state[kMaxDevices] = {};  // 0 not yet, 1 ready, -1 refused
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return nullptr;
  }
  if (state[dev] == 0) {
    SideStream& x = per_device[dev];
    const bool ok = cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking) == cudaSuccess &&
                    cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming) == cudaSuccess &&
                    cudaEventCreateWithFlags(&x.join, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) cudaGetLastError();
    state[dev] = ok ? 1 : -1;
  }
  return state[dev] == 1 ? &per_device[dev] : nullptr;
}

}  // namespace rt

using namespace rt;

static rt_build_params normalized(const rt_build_params* p) {
  rt_build_params q = p ? *p : rt_build_params{12, 1, 0, 0, 32};
  if (q.tree_depth == 0) q.tree_depth = 12;
  if (q.tree_depth > 32) q.tree_depth = 32;
  if (q.min_leaf == 0) q.min_leaf = kMinLeafDefault;
  if (q.max_leaf == 0) q.max_leaf = kMaxLeafDefault;
  if (q.morton_bits == 0) q.morton_bits = 32;
  if (q.cluster_leaf == 0) q.cluster_leaf = kClusterLeafDefault;
  return q;
}

extern "C" rt_status rt_lbvh_scratch_bytes(uint32_t face_count, const rt_build_params* params, size_t* scratch_bytes, uint32_t* max_nodes) {
  if (!scratch_bytes || face_count == 0) return RT_ERR_INVALID_ARGUMENT;
  rt_build_params q = normalized(params);
  Carve c(nullptr, 0);
  BuildLayout L;
  *scratch_bytes = carve_build(c, L, face_count, q.tree_depth, true, true, (q.accel_trees & RT_ACCEL_CLUSTERS) != 0);
  if (max_nodes) *max_nodes = 2 * face_count - 1;
  return RT_OK;
}

extern "C" rt_status rt_lbvh_accel_bytes(uint32_t face_count, size_t* bytes) {
  if (!bytes || face_count == 0) return RT_ERR_INVALID_ARGUMENT;
  Carve c(nullptr, 0);
  AccelLayout A;
  *bytes = carve_accel(c, A, face_count);
  return RT_OK;
}

extern "C" rt_status rt_lbvh_build(const rt_build_desc* d, rt_stream stream_) {
  const rt::NvtxRange nvtx_range("rt_lbvh_build");
  if (!d || d->face_count == 0 || !d->vertices || !d->faces_in || !d->boxes || !d->indices || !d->nodes || d->max_nodes == 0)
    return RT_ERR_INVALID_ARGUMENT;
  if (d->face_count > 0x7FFFFFFFu) return RT_ERR_INVALID_ARGUMENT;
  const rt_build_params q = normalized(&d->params);
  if (q.morton_bits != 32 && q.morton_bits != 30) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t n = d->face_count;
  // every size check comes before the first launch, so that a refused call leaves the caller's buffers untouched
  if (d->max_nodes < 2 * n - 1) return RT_ERR_CAPACITY;
  const bool complete = q.tree_complete != 0;
  const bool in_place = complete && d->faces_out && (d->faces_out == d->faces_in);
  Carve c(d->scratch, d->scratch_bytes);
  BuildLayout L;
  const bool clusters = (q.accel_trees & RT_ACCEL_CLUSTERS) != 0;
  if (clusters && (n > kClusterFirstMask || q.cluster_leaf > kClusterLeafMax)) return RT_ERR_UNSUPPORTED;
  carve_build(c, L, n, q.tree_depth, d->codes == nullptr, in_place, clusters);
  if (!d->scratch || !c.ok()) return RT_ERR_SCRATCH_TOO_SMALL;
  AccelLayout AL{};
  const bool accel = complete && d->accel && d->tris;
  if (accel) {
    Carve ca(d->accel, d->accel_bytes);
    carve_accel(ca, AL, n);
    if (!ca.ok()) return RT_ERR_SCRATCH_TOO_SMALL;
  }
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  cudaStream_t st = (cudaStream_t)stream_;
  uint32_t* codes = d->codes ? d->codes : L.codes;
  const int sms = sm_count();

  // 1. hit box (the sorts' digit counts and the hit box's block counter start at zero)
  if (cudaMemsetAsync(L.counts, 0, (5 * 256 + 1) * 4, st) != cudaSuccess) return RT_ERR_CUDA;
  if (d->hitbox) {
    float4 mn = make_float4(d->hitbox[0], d->hitbox[1], d->hitbox[2], d->hitbox[3]);
    float4 mx = make_float4(d->hitbox[4], d->hitbox[5], d->hitbox[6], d->hitbox[7]);
    k_set_hitbox<<<1, 1, 0, st>>>(L.hit, mn, mx);
    note_launch();
  } else {
    k_hitbox<<<kHitParts, 256, 0, st>>>((const float4*)d->vertices, d->vertex_count, L.partial, L.counts + 5 * 256, L.hit);
    note_launch();
  }
  RT_CHECK_LAUNCH();
  // 2. boxes, indices, codes (and the digit counts of both sorts, counted by the kernels that make the keys)
  {
    uint32_t blocks = (uint32_t)hmin<uint64_t>((n + 255) / 256, (uint64_t)sms * 16);
    k_boxes_morton<<<blocks, 256, 0, st>>>((const float4*)d->vertices, (const uint4*)d->faces_in, n, L.hit, (int)q.morton_bits,
                                           (float4*)d->boxes, codes, d->indices, L.counts);
    note_launch();
    RT_CHECK_LAUNCH();
  }
  // 3. sort (code, index); the build's error word starts here, so that the sorts' bounded waits report into it
  if (cudaMemsetAsync(L.err, 0, 16, st) != cudaSuccess) return RT_ERR_CUDA;
  rt_status s = radix_sort_pairs(codes, d->indices, n, 0, 32, 0, L.sort_scratch, L.sort_bytes, st, nullptr, L.err, L.counts);
  if (s != RT_OK) return s;
  // 4. per-level split lists
  if (cudaMemsetAsync(L.lev_count, 0, 256 * 4, st) != cudaSuccess) return RT_ERR_CUDA;
  if (n > 1) {
    uint32_t blocks = (uint32_t)hmin<uint64_t>((n + 255) / 256, (uint64_t)sms * 16);
    k_levels<<<blocks, 256, 0, st>>>(codes, n, L.lev, L.C, L.counts + 4 * 256);
    note_launch();
    RT_CHECK_LAUNCH();
    s = radix_sort_pairs(L.lev, L.C, n - 1, 0, 8, 0, L.sort_scratch, L.sort_bytes, st, L.lev_count, L.err, L.counts + 4 * 256);
    if (s != RT_OK) return s;
  }
  // 5. Morton top tree
  {
    TopoArgs A;
    A.C = L.C; A.lev_count = L.lev_count; A.n = n; A.D = q.tree_depth; A.min_leaf = q.min_leaf; A.max_leaf = q.max_leaf;
    A.complete = complete ? 1u : 0u; A.cap_m = L.cap_m;
    A.ra = L.ra; A.rb = L.rb; A.parent = L.parent; A.info = L.info; A.child = L.child; A.leaves = L.leaves; A.mleaves = L.mleaves;
    A.rank = L.rank; A.lambda = L.lambda; A.ord = L.ord; A.id = L.id;
    A.ml_lambda = L.ml_lambda; A.ml_rec = L.ml_rec; A.ml_rank = L.ml_rank; A.parent_id = L.parent_id;
    A.nodes = d->nodes; A.max_nodes = d->max_nodes; A.hdr = L.hdr;
    A.level_hist = nullptr; A.level_base = 0; A.pos_base = 0;
    k_topo_morton<<<1, kTopoThreads, 0, st>>>(A);
    note_launch();
    RT_CHECK_LAUNCH();
  }
  // 6. leaves: median subtrees, reorder, triangles, boxes bottom-up
  {
    uint32_t count = d->max_nodes < L.max_nodes ? d->max_nodes : L.max_nodes;
    if (cudaMemsetAsync(L.arrive, 0, (size_t)count * 4, st) != cudaSuccess) return RT_ERR_CUDA;
    LeafArgs A;
    A.verts = (const float4*)d->vertices;
    A.faces_in = (const uint4*)d->faces_in;
    A.faces_out = complete && d->faces_out ? (in_place ? L.faces_tmp : (uint4*)d->faces_out) : nullptr;
    A.tris = complete ? (float4*)d->tris : nullptr;
    A.indices = d->indices; A.ml_lambda = L.ml_lambda; A.ml_rec = L.ml_rec; A.ml_rank = L.ml_rank; A.parent_id = L.parent_id;
    A.arrive = L.arrive; A.nodes = d->nodes; A.max_nodes = d->max_nodes; A.max_leaf = q.max_leaf; A.hdr = L.hdr; A.err = L.err;
    A.acc_leaves = accel ? AL.leaves : nullptr;
    A.acc_groups = accel ? AL.groups : nullptr;
    A.leaf_lambda = L.leaf_lambda;
    A.pos_base = 0;
    A.vert_base = 0;
    A.local_indices = nullptr;
    A.parent_cap = count;
    static const int leaf_blocks = resident_blocks_of(k_leaves, 256);
    k_leaves<<<sms * leaf_blocks, 256, 0, st>>>(A);
    k_propagate<<<sms * 8, 256, 0, st>>>(d->nodes, L.parent_id, L.arrive, L.hdr, count);
    note_launch(2);
    RT_CHECK_LAUNCH();
    if (accel) {
      k_accel_nodes<<<sms * 4, 256, 0, st>>>(d->nodes, L.hdr, L.leaf_lambda, AL.tnodes, AL.wide, AL.hdr);
      note_launch();
      RT_CHECK_LAUNCH();
      if (clusters) {
        s = build_cluster_tree((const float4*)d->tris, codes, n, q.cluster_leaf, L.ct, AL.hdr, AL.crec, st);
        if (s != RT_OK) return s;
      }
    }
  }
  if (in_place && cudaMemcpyAsync(d->faces_out, L.faces_tmp, (size_t)n * 16, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return RT_ERR_CUDA;
  if (d->info) {
    k_write_info<<<1, 32, 0, st>>>(L.hdr, L.err, d->info);
    note_launch();
    RT_CHECK_LAUNCH();
  }
  return RT_OK;
}

extern "C" rt_status rt_mesh_boxes(const float* vertices, const uint32_t* faces, uint32_t n, float* boxes, uint32_t* indices, rt_stream st) {
  if (n == 0) return RT_OK;
  if (!vertices || !faces || !boxes) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  uint32_t blocks = (uint32_t)hmin<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 16);
  k_boxes_morton<<<blocks, 256, 0, (cudaStream_t)st>>>((const float4*)vertices, (const uint4*)faces, n, nullptr, 32, (float4*)boxes,
                                                      nullptr, indices, nullptr);
    note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

namespace rt { namespace {
__global__ __launch_bounds__(256) void k_reorder(const uint4* __restrict__ in, const uint32_t* __restrict__ idx, uint32_t n, uint4* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = ldg4(in + __ldg(idx + i));
}
}}  // namespace rt

extern "C" rt_status rt_reorder_faces(const uint32_t* faces_in, const uint32_t* indices, uint32_t n, uint32_t* faces_out, rt_stream st) {
  if (n == 0) return RT_OK;
  if (!faces_in || !indices || !faces_out) return RT_ERR_INVALID_ARGUMENT;
  const char* a = (const char*)faces_in;
  const char* b = (const char*)faces_out;
  if (a < b + (size_t)n * 16 && b < a + (size_t)n * 16) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  uint32_t blocks = (uint32_t)hmin<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 16);
  k_reorder<<<blocks, 256, 0, (cudaStream_t)st>>>((const uint4*)faces_in, indices, n, (uint4*)faces_out);
    note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

// ============================================================================
// Batched build: M meshes, every stage in one set of launches.
// ============================================================================
namespace rt {
namespace {


struct BatchArgs {
  uint32_t M, N;
  const uint32_t* foff;
  const uint32_t* voff;
  const float4* verts;
  const uint4* faces_in;
  uint4* faces_out;
  float4* boxes;
  uint32_t* indices_out;
  uint32_t* codes;
  uint32_t* nodes;
  float4* tris;
  rt_build_params q;
  // scratch
  float4* hits;           // [2M]
  float4* hitpart;        // [2 M kHitSplit]: the hit box shares of k_batch_hitbox
  uint32_t* hitdone;      // [M]: finished shares per mesh
  uint32_t* idx;          // [N] global face index in sorted order
  uint32_t* codes_raw;    // [N] codes before sorting
  uint32_t* mkey;         // [N] mesh id per position
  uint32_t* lev;          // [N] (mesh, level) keys
  uint32_t* C;            // [N] split positions
  uint32_t* hist;         // [M * 64 + 1]
  uint32_t *ra, *rb, *parent, *info, *child, *leaves, *mleaves, *rank, *lambda, *ord, *id;  // [2N + 3M]
  uint32_t* ml_lambda;
  uint4* ml_rec;
  uint32_t* ml_rank;
  uint32_t* parent_id;    // [2N - M]
  uint32_t* arrive;       // [2N - M]
  uint32_t* leaf_lambda;  // [2N - M]
  uint32_t* hdr;          // [16 M]
  uint32_t* leaf_base;    // [M + 1]
  uint32_t* err;          // [4]
  uint32_t* counts;       // [9 x 256 + 64]: digit counts of the code sort (4 passes), the mesh sort (2), the level
                          // sort (3), then the count of finished topology CTAs

  // traversal blob
  uint32_t* acc_hdr;      // [64 M]
  float4* tnodes;         // [4 N]
  uint4* acc_leaves;      // [N]
  float4* groups;         // [2 (N + N/8 + M + 1)]
  float4* wide;           // [8 N]
  float4* crec;           // cluster records (from F_m per mesh)
  ClusterTemps ct;        // cluster tree build temporaries (RT_ACCEL_CLUSTERS only)
  rt_build_info* info_out;
};

// Per-mesh hitbox: one 512-thread block per mesh, four loads in flight per
// thread (the largest meshes bound the launch).
__global__ __launch_bounds__(512) void k_batch_hitbox(BatchArgs B) {
  // kHitSplit CTAs per mesh, each over its share of the mesh's vertices; the last of them combines the shares
  const uint32_t m = blockIdx.x / kHitSplit, part = blockIdx.x % kHitSplit;
  const uint32_t w0 = B.voff[m], w1 = B.voff[m + 1], share = (w1 - w0 + kHitSplit - 1) / kHitSplit;
  const uint32_t v0 = min(w1, w0 + part * share), v1 = min(w1, v0 + share);
  if (part == 0 && threadIdx.x == 0) {
    B.acc_hdr[64 * (size_t)m + kHdrClusterValid] = 0;  // set again by the cluster build, if any
    // the mesh sort's digit counts: mesh m holds foff[m + 1] - foff[m] keys of value m
    const uint32_t faces = B.foff[m + 1] - B.foff[m];
    atomicAdd(B.counts + 4 * 256 + (m & 255u), faces);
    atomicAdd(B.counts + 5 * 256 + ((m >> 8) & 255u), faces);
  }
  float4 mn[4], mx[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    mn[k] = make_float4(kHuge, kHuge, kHuge, kHuge);
    mx[k] = make_float4(-kHuge, -kHuge, -kHuge, -kHuge);
  }
  uint32_t i = v0 + threadIdx.x;
  for (; i + 3 * 512 < v1; i += 4 * 512) {
    float4 p[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) p[k] = ldg4(B.verts + i + k * 512);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      mn[k] = f4min(mn[k], p[k]);
      mx[k] = f4max(mx[k], p[k]);
    }
  }
  for (; i < v1; i += 512) {
    const float4 p = ldg4(B.verts + i);
    mn[0] = f4min(mn[0], p);
    mx[0] = f4max(mx[0], p);
  }
  __shared__ float4 s_mn[512], s_mx[512];
  s_mn[threadIdx.x] = f4min(f4min(mn[0], mn[1]), f4min(mn[2], mn[3]));
  s_mx[threadIdx.x] = f4max(f4max(mx[0], mx[1]), f4max(mx[2], mx[3]));
  __syncthreads();
  for (int o = 256; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s_mn[threadIdx.x] = f4min(s_mn[threadIdx.x], s_mn[threadIdx.x + o]);
      s_mx[threadIdx.x] = f4max(s_mx[threadIdx.x], s_mx[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    B.hitpart[2 * (size_t)blockIdx.x] = s_mn[0];
    B.hitpart[2 * (size_t)blockIdx.x + 1] = s_mx[0];
    __threadfence();
    // the mesh's last share to finish combines its kHitSplit shares in share order (an empty share holds +-huge
    // and changes nothing); nothing waits for it inside the launch
    if (atomicAdd(B.hitdone + m, 1u) == kHitSplit - 1) {
      __threadfence();
      float4 a = __ldcg(B.hitpart + 2 * (size_t)m * kHitSplit), b = __ldcg(B.hitpart + 2 * (size_t)m * kHitSplit + 1);
      for (uint32_t p = 1; p < kHitSplit; ++p) {
        a = f4min(a, __ldcg(B.hitpart + 2 * ((size_t)m * kHitSplit + p)));
        b = f4max(b, __ldcg(B.hitpart + 2 * ((size_t)m * kHitSplit + p) + 1));
      }
      B.hits[2 * m] = a;
      B.hits[2 * m + 1] = b;
    }
  }
}

__global__ __launch_bounds__(256) void k_batch_boxes_morton(BatchArgs B) {
  __shared__ uint32_t s_cc[4 * 256];  // the code sort's digit counts of this block's faces
  for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) s_cc[i] = 0;
  __syncthreads();
  const int layout = (int)B.q.morton_bits;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < B.N; k += gridDim.x * blockDim.x) {
    const uint32_t m = find_seg(B.foff, B.M, k);
    const float4 hmin = B.hits[2 * m], hmax = B.hits[2 * m + 1];
    const float sx = (layout == 30 ? 1023.0f : 2047.0f) / (hmax.x - hmin.x);
    const float sy = (layout == 30 ? 1023.0f : 2047.0f) / (hmax.y - hmin.y);
    const float sz = 1023.0f / (hmax.z - hmin.z);
    const uint32_t vb = __ldg(B.voff + m);
    const uint4 f = ldg4(B.faces_in + k);
    const float4 v0 = ldg4(B.verts + vb + f.x), v1 = ldg4(B.verts + vb + f.y), v2 = ldg4(B.verts + vb + f.z);
    const float4 mn = f4min(f4min(v0, v1), v2);
    const float4 mx = f4max(f4max(v0, v1), v2);
    B.boxes[2 * (size_t)k] = mn;
    B.boxes[2 * (size_t)k + 1] = mx;
    B.idx[k] = k;
    const float cx = 0.5f * (mn.x + mx.x), cy = 0.5f * (mn.y + mx.y), cz = 0.5f * (mn.z + mx.z);
    const uint32_t code = spread_code(f2u_sat((cx - hmin.x) * sx), f2u_sat((cy - hmin.y) * sy), f2u_sat((cz - hmin.z) * sz), layout);
    B.codes[k] = code;
    B.codes_raw[k] = code;
#pragma unroll
    for (int p = 0; p < 4; ++p) atomicAdd(&s_cc[p * 256 + ((code >> (8 * p)) & 255u)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x)
    if (s_cc[i]) atomicAdd(B.counts + i, s_cc[i]);
}

// After the (mesh, code) order is complete: the code of each position, and per pair (i, i + 1) the split level
// key (mesh * 64 + level; 32 = no split, also across meshes), its (mesh, level) count and the level sort's digit
// counts (up to three 8-bit passes).
__global__ __launch_bounds__(256) void k_batch_levels(BatchArgs B) {
  __shared__ uint32_t s_lc[3 * 256];
  for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) s_lc[i] = 0;
  __syncthreads();
  // whole warps step together, so that equal keys of a warp are counted with one atomic (the keys of a mesh
  // crowd onto a few levels: one atomic per position would queue on those few counters)
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < B.N; base += gridDim.x * blockDim.x) {
    const uint32_t i = base + lane;
    uint32_t key = ~0u;
    if (i < B.N) {
      const uint32_t c0 = B.codes_raw[B.idx[i]];
      B.codes[i] = c0;
      if (i + 1 < B.N) {
        const uint32_t m = B.mkey[i];
        uint32_t lev = 32;
        if (B.mkey[i + 1] == m) {
          const uint32_t d = c0 ^ B.codes_raw[B.idx[i + 1]];
          if (d) lev = (uint32_t)__clz(d);
        }
        key = m * 64 + lev;
        B.lev[i] = key;
        B.C[i] = i + 1;
      }
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, key);
    if (key != ~0u && lane == (uint32_t)(__ffs(peers) - 1)) {
      const uint32_t cnt = (uint32_t)__popc(peers);
      atomicAdd(B.hist + key, cnt);
#pragma unroll
      for (int p = 0; p < 3; ++p) atomicAdd(&s_lc[p * 256 + ((key >> (8 * p)) & 255u)], cnt);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x)
    if (s_lc[i]) atomicAdd(B.counts + 6 * 256 + i, s_lc[i]);
}

__global__ __launch_bounds__(kTopoThreads) void k_batch_topo(BatchArgs B) {
  const uint32_t m = blockIdx.x;
  const uint32_t F = B.foff[m], n = B.foff[m + 1] - F;
  const uint32_t bb = bfs_base(F, m), nb = node_base(F, m);
  TopoArgs A;
  A.C = B.C; A.lev_count = nullptr; A.n = n; A.D = B.q.tree_depth; A.min_leaf = B.q.min_leaf; A.max_leaf = B.q.max_leaf;
  A.complete = 1u; A.cap_m = morton_cap_dev(n, B.q.tree_depth);
  A.ra = B.ra + bb; A.rb = B.rb + bb; A.parent = B.parent + bb; A.info = B.info + bb; A.child = B.child + bb;
  A.leaves = B.leaves + bb; A.mleaves = B.mleaves + bb; A.rank = B.rank + bb; A.lambda = B.lambda + bb; A.ord = B.ord + bb;
  A.id = B.id + bb; A.ml_lambda = B.ml_lambda + bb; A.ml_rec = B.ml_rec + bb; A.ml_rank = B.ml_rank + bb;
  A.parent_id = B.parent_id + nb; A.nodes = B.nodes + 8 * (size_t)nb; A.max_nodes = 2 * n - 1; A.hdr = B.hdr + 16 * m;
  // the pairs of the meshes before m are their F positions (every position but the last of all has one pair),
  // so this mesh's level lists start at F in the level order
  A.level_hist = B.hist + 64 * m; A.level_base = F; A.pos_base = F;
  topo_morton(A);
  // the CTA that finishes last (every other mesh's header is written) makes the leaf-order bases per mesh (an
  // exclusive scan of the leaf counts) and their total; nothing waits for it inside this kernel
  __shared__ uint32_t s_last;
  __shared__ uint32_t s_warp2[kTopoWarps];
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(B.counts + 9 * 256, 1u) == B.M - 1 ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  uint32_t running = 0;
  for (uint32_t c = 0; c < B.M; c += kTopoThreads) {
    const uint32_t i = c + threadIdx.x;
    const uint32_t bad = i < B.M ? (__ldcg(B.hdr + 16 * i + 8) & (RT_DEVERR_NODE_CAPACITY | RT_DEVERR_MORTON_CAPACITY)) : 0u;
    const uint32_t v = (i < B.M && !bad) ? __ldcg(B.hdr + 16 * i) : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan_nt<kTopoThreads>(v, s_warp2, tot);
    if (i < B.M) B.leaf_base[i] = running + ex;
    running += tot;
  }
  if (threadIdx.x == 0) B.leaf_base[B.M] = running;
}

__global__ __launch_bounds__(256) void k_batch_leaves(BatchArgs B) {
  const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t total = B.leaf_base[B.M];
  // a contiguous run of leaves per warp (the grid is one resident wave): the
  // mesh and the Morton-leaf search carry over from one leaf to the next
  const uint32_t per = (total + nwarps - 1) / nwarps;
  const uint32_t g0 = min(total, warp_global * per), g1 = min(total, g0 + per);
  if (g0 >= g1) return;
  uint32_t m = find_seg(B.leaf_base, B.M, g0), hint = ~0u;
  LeafArgs A;
  auto mesh_args = [&]() {
    const uint32_t F = B.foff[m], n = B.foff[m + 1] - F;
    const uint32_t bb = bfs_base(F, m), nb = node_base(F, m);
    A.verts = B.verts; A.faces_in = B.faces_in; A.faces_out = B.faces_out; A.tris = B.tris; A.indices = B.idx;
    A.ml_lambda = B.ml_lambda + bb; A.ml_rec = B.ml_rec + bb; A.ml_rank = B.ml_rank + bb;
    A.parent_id = B.parent_id + nb; A.arrive = B.arrive + nb; A.nodes = B.nodes + 8 * (size_t)nb; A.max_nodes = 2 * n - 1;
    A.max_leaf = B.q.max_leaf; A.hdr = B.hdr + 16 * m; A.err = B.err;
    A.acc_leaves = B.acc_leaves + F; A.acc_groups = B.groups + 2 * (size_t)group_base(F, m); A.leaf_lambda = B.leaf_lambda + nb;
    A.pos_base = F; A.vert_base = B.voff[m]; A.local_indices = B.indices_out; A.parent_cap = 2 * n - 1;
  };
  mesh_args();
  for (uint32_t g = g0; g < g1; ++g) {
    if (B.leaf_base[m + 1] <= g) {  // the next non-empty mesh
      while (B.leaf_base[m + 1] <= g) ++m;
      mesh_args();
      hint = ~0u;
    }
    leaf_body(A, g - B.leaf_base[m], hint);
  }
}

// Bottom-up boxes of every mesh: one thread per node slot, the leaves climb.
__global__ __launch_bounds__(256) void k_batch_propagate(BatchArgs B) {
  const uint32_t slots = 2 * B.N - B.M;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < slots; p += gridDim.x * blockDim.x) {
    // mesh whose node range holds slot p: largest m with 2 F_m - m <= p
    uint32_t lo = 0, hi = B.M - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (node_base(__ldg(B.foff + mid), mid) <= p) lo = mid; else hi = mid - 1;
    }
    const uint32_t m = lo, F = B.foff[m], n = B.foff[m + 1] - F, nb = node_base(F, m);
    const uint32_t* h = B.hdr + 16 * m;
    if (n == 0 || (h[8] & (RT_DEVERR_NODE_CAPACITY | RT_DEVERR_MORTON_CAPACITY))) continue;
    const uint32_t lp = p - nb, cap = 2 * n - 1;
    if (lp >= h[2] || lp >= cap) continue;
    uint32_t* nodes = B.nodes + 8 * (size_t)nb;
    if (nodes[8 * (size_t)lp] & 1u) climb(nodes, B.parent_id + nb, B.arrive + nb, cap, lp);
  }
}

// Traversal records of every mesh (two-child and 4-wide, per internal node) and each mesh's build info.
__global__ __launch_bounds__(256) void k_batch_records(BatchArgs B) {
  const uint32_t slots = 2 * B.N - B.M;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < slots; p += gridDim.x * blockDim.x) {
    // mesh whose node range holds slot p: largest m with 2 F_m - m <= p
    uint32_t lo = 0, hi = B.M - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (node_base(__ldg(B.foff + mid), mid) <= p) lo = mid; else hi = mid - 1;
    }
    const uint32_t m = lo, F = B.foff[m], nb = node_base(F, m);
    const uint32_t* h = B.hdr + 16 * m;
    if (h[8] & (RT_DEVERR_NODE_CAPACITY | RT_DEVERR_MORTON_CAPACITY)) continue;
    const uint32_t lp = p - nb;
    if (lp >= h[2]) continue;
    if (lp == 0) {
      uint32_t* ah = B.acc_hdr + 64 * m;
      ah[0] = (B.nodes[8 * (size_t)nb] & 1u) ? ~0u : 0u;
      ah[1] = h[0];
      ah[2] = h[2];
    }
    accel_wide_node(B.nodes + 8 * (size_t)nb, B.leaf_lambda + nb, B.tnodes + 4 * (size_t)F, B.wide + 8 * (size_t)F, lp);
  }
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < B.M; m += gridDim.x * blockDim.x) {
    const uint32_t* h = B.hdr + 16 * m;
    rt_build_info* o = B.info_out + m;
    o->leaf_count = h[0]; o->node_count = h[2]; o->real_depth = h[3]; o->split_count = h[4];
    o->overrun_visits = h[5]; o->nondet_reads = h[6]; o->past_end_reads = h[7]; o->error = h[8] | *B.err;
  }
}

size_t carve_batch(Carve& c, BatchArgs& B, uint32_t M, uint32_t N, bool clusters) {
  B.hits = c.take<float4>(2 * (size_t)M);
  B.hitpart = c.take<float4>(2 * (size_t)M * kHitSplit);
  B.hitdone = c.take<uint32_t>(M);
  B.idx = c.take<uint32_t>(N);
  B.codes_raw = c.take<uint32_t>(N);
  B.mkey = c.take<uint32_t>(N);
  B.lev = c.take<uint32_t>(N);
  B.C = c.take<uint32_t>(N);
  B.hist = c.take<uint32_t>((size_t)M * 64 + 1);
  const size_t bfs = 2 * (size_t)N + 3 * (size_t)M + 4;
  uint32_t** arrs[] = {&B.ra, &B.rb, &B.parent, &B.info, &B.child, &B.leaves, &B.mleaves, &B.rank, &B.lambda, &B.ord, &B.id};
  for (auto a : arrs) *a = c.take<uint32_t>(bfs);
  B.ml_lambda = c.take<uint32_t>(bfs);
  B.ml_rec = c.take<uint4>(bfs);
  B.ml_rank = c.take<uint32_t>(bfs);
  const size_t nodes = 2 * (size_t)N;
  B.parent_id = c.take<uint32_t>(nodes);
  B.arrive = c.take<uint32_t>(nodes);
  B.leaf_lambda = c.take<uint32_t>(nodes);
  B.hdr = c.take<uint32_t>(16 * (size_t)M);
  B.leaf_base = c.take<uint32_t>((size_t)M + 1);
  B.err = c.take<uint32_t>(4);
  B.counts = c.take<uint32_t>(9 * 256 + 64);
  B.ct = ClusterTemps{};
  if (clusters) carve_cluster_temps(c, B.ct, N, M);
  const size_t sort_bytes = radix_scratch_bytes(N);
  c.take<char>(sort_bytes);
  return c.off + 256;
}

size_t carve_batch_accel(Carve& c, BatchArgs& B, uint32_t M, uint32_t N) {
  BatchAccel L;
  const size_t bytes = carve_batch_accel_layout(c, L, M, N);
  B.acc_hdr = L.hdr; B.tnodes = L.tnodes; B.acc_leaves = L.leaves; B.groups = L.groups; B.wide = L.wide; B.crec = L.crec;
  return bytes;
}

}  // namespace
}  // namespace rt

extern "C" rt_status rt_batch_sizes(uint32_t M, uint32_t N, const rt_build_params* params, size_t* scratch_bytes, size_t* accel_bytes) {
  if (M == 0 || N < M || !scratch_bytes) return RT_ERR_INVALID_ARGUMENT;
  const rt_build_params q = normalized(params);
  Carve c(nullptr, 0);
  BatchArgs B;
  *scratch_bytes = carve_batch(c, B, M, N, (q.accel_trees & RT_ACCEL_CLUSTERS) != 0);
  if (accel_bytes) {
    Carve a(nullptr, 0);
    *accel_bytes = carve_batch_accel(a, B, M, N);
  }
  return RT_OK;
}

extern "C" rt_status rt_batch_build(const rt_batch_build_desc* d, rt_stream stream_) {
  const rt::NvtxRange nvtx_range("rt_batch_build");
  if (!d || d->mesh_count == 0 || d->face_count < d->mesh_count || !d->face_offsets || !d->vertex_offsets || !d->vertices ||
      !d->faces_in || !d->faces_out || !d->boxes || !d->indices || !d->codes || !d->nodes || !d->tris || !d->accel || !d->info)
    return RT_ERR_INVALID_ARGUMENT;
  if (d->faces_out == d->faces_in) return RT_ERR_INVALID_ARGUMENT;
  if (d->mesh_count > 65536u || d->face_count > 0x3FFFFFFFu) return RT_ERR_INVALID_ARGUMENT;
  rt_build_params q = normalized(&d->params);
  if (!q.tree_complete || (q.morton_bits != 32 && q.morton_bits != 30)) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t M = d->mesh_count, N = d->face_count;
  const bool clusters = (q.accel_trees & RT_ACCEL_CLUSTERS) != 0;
  if (clusters && (N > kClusterFirstMask || q.cluster_leaf > kClusterLeafMax)) return RT_ERR_UNSUPPORTED;
  Carve c(d->scratch, d->scratch_bytes);
  BatchArgs B;
  carve_batch(c, B, M, N, clusters);
  if (!d->scratch || !c.ok()) return RT_ERR_SCRATCH_TOO_SMALL;
  // the sort scratch is the last region
  const size_t sort_bytes = radix_scratch_bytes(N);
  void* sort_scratch = (char*)d->scratch + (c.off - sort_bytes - 0);
  {
    Carve a(d->accel, d->accel_bytes);
    carve_batch_accel(a, B, M, N);
    if (!a.ok()) return RT_ERR_SCRATCH_TOO_SMALL;
  }
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  B.M = M; B.N = N; B.foff = d->face_offsets; B.voff = d->vertex_offsets; B.verts = (const float4*)d->vertices;
  B.faces_in = (const uint4*)d->faces_in; B.faces_out = (uint4*)d->faces_out; B.boxes = (float4*)d->boxes;
  B.indices_out = d->indices; B.codes = d->codes; B.nodes = d->nodes; B.tris = (float4*)d->tris; B.q = q; B.info_out = d->info;
  cudaStream_t st = (cudaStream_t)stream_;
  const int sms = sm_count();
  const uint32_t fblocks = (uint32_t)hmin<uint64_t>((N + 255) / 256, (uint64_t)sms * 16);
  // the error word and every sort's digit counts (counted by the kernels that make the keys) start at zero
  if (cudaMemsetAsync(B.err, 0, 16, st) != cudaSuccess) return RT_ERR_CUDA;
  if (cudaMemsetAsync(B.counts, 0, (9 * 256 + 64) * 4, st) != cudaSuccess) return RT_ERR_CUDA;
  if (cudaMemsetAsync(B.hist, 0, ((size_t)M * 64 + 1) * 4, st) != cudaSuccess) return RT_ERR_CUDA;
  if (cudaMemsetAsync(B.hitdone, 0, (size_t)M * 4, st) != cudaSuccess) return RT_ERR_CUDA;
  k_batch_hitbox<<<M * kHitSplit, 512, 0, st>>>(B);
  k_batch_boxes_morton<<<fblocks, 256, 0, st>>>(B);
  note_launch(2);
  RT_CHECK_LAUNCH();
  // Morton order of all faces; its last pass also writes each position's mesh (the key of the next sort)
  rt_status s = radix_sort_pairs(B.codes, B.idx, N, 0, 32, 0, sort_scratch, sort_bytes, st, nullptr, B.err, B.counts, B.foff, M,
                                 B.mkey);
  if (s != RT_OK) return s;
  // key widths in whole 8-bit digits: mesh ids < M, level keys < 64 (M - 1) + 33
  auto digit_bits = [](uint64_t maxval) -> uint32_t {
    uint32_t b = 1;
    while (b < 64 && (1ull << b) <= maxval) ++b;
    return b > 24 ? 32u : (b + 7) / 8 * 8;
  };
  s = radix_sort_pairs(B.mkey, B.idx, N, 0, digit_bits(M - 1), 0, sort_scratch, sort_bytes, st, nullptr, B.err, B.counts + 4 * 256);
  if (s != RT_OK) return s;
  k_batch_levels<<<fblocks, 256, 0, st>>>(B);
  note_launch();
  RT_CHECK_LAUNCH();
  if (N > 1) {
    s = radix_sort_pairs(B.lev, B.C, N - 1, 0, digit_bits(64ull * (M - 1) + 32), 0, sort_scratch, sort_bytes, st, nullptr, B.err,
                         B.counts + 6 * 256);
    if (s != RT_OK) return s;
  }
  k_batch_topo<<<M, kTopoThreads, 0, st>>>(B);
  note_launch();
  RT_CHECK_LAUNCH();
  if (cudaMemsetAsync(B.arrive, 0, (2 * (size_t)N) * 4, st) != cudaSuccess) return RT_ERR_CUDA;
  static const int leaf_blocks = resident_blocks_of(k_batch_leaves, 256);
  k_batch_leaves<<<sms * leaf_blocks, 256, 0, st>>>(B);
  note_launch();
  RT_CHECK_LAUNCH();
  // the node boxes and records (from the nodes) and the cluster trees (from the codes and triangles) are
  // independent: with cluster trees, the node half runs on a side stream beside them
  SideStream* side = clusters ? side_stream() : nullptr;
  cudaStream_t ns = st;
  if (side) {
    if (cudaEventRecord(side->fork, st) != cudaSuccess || cudaStreamWaitEvent(side->s, side->fork, 0) != cudaSuccess)
      return RT_ERR_CUDA;
    ns = side->s;
  }
  k_batch_propagate<<<sms * 8, 256, 0, ns>>>(B);
  k_batch_records<<<sms * 4, 256, 0, ns>>>(B);
  note_launch(2);
  RT_CHECK_LAUNCH();
  if (clusters) {
    s = batch_build_cluster_tree(B.tris, B.codes, B.foff, M, N, q.cluster_leaf, B.ct, B.acc_hdr, B.crec, st);
    if (side && (cudaEventRecord(side->join, side->s) != cudaSuccess || cudaStreamWaitEvent(st, side->join, 0) != cudaSuccess))
      return RT_ERR_CUDA;
    if (s != RT_OK) return s;
  }
  return RT_OK;
}
