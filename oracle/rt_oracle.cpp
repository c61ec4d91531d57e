// rt_oracle.cpp -- CPU restatement of the reference LBVH build and closest-hit
// traversal (gatouillatpy/cudart).
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product (cudart_b200/, include/)
// links, loads or calls this file; only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py load it, as the checker and as
// the timed host-core baseline.
//
// Parity pin: the restatement below is checked against the reference's own
// source code compiled from its files by oracle/build_ref.sh (host topology
// recursion, split finder, Morton kernel body, per-ray traversal kernel body,
// bounding-box pass), see tests/test_oracle_vs_reference.py, and against the
// committed golden fixtures in tests/golden/.
//
// Arithmetic is pinned: compiled with -ffp-contract=off (no FMA contraction),
// IEEE division and square root, float evaluation order exactly as written in
// the reference sources (left-to-right sums, 4-wide dot products with the w
// products included).
//
// Every exported function is extern "C" with plain pointers so it can be
// loaded with ctypes.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_API extern "C" __attribute__((visibility("default")))

typedef uint32_t u32;
typedef uint64_t u64;

// CUDART_NORM_HUGE_F (math_constants.h), used by aabox::reset and the depth clear.
static const float kHuge = 3.402823466e+38f;
static const u32 kMinLeafDefault = 16;   // kernels/CUDA_buildMeshTreeLBVH.cu:39
static const u32 kMaxLeafDefault = 224;  // kernels/CUDA_buildMeshTreeLBVH.cu:40

struct F4 { float x, y, z, w; };
struct U4 { u32 x, y, z, w; };
struct Box { F4 mn, mx; };                        // aabox, CUDABox.h:17-148 (32 B)
struct Node { u32 w0, w1; float bmin[3], bmax[3]; };  // bvnode, CUDANode.h:20-50 (32 B)

static_assert(sizeof(Box) == 32, "aabox is 32 bytes");
static_assert(sizeof(Node) == 32, "bvnode is 32 bytes");

// Host fminf/fmaxf of the reference (types/_cuda_float.h:11-19).
static inline float fmin_sel(float a, float b) { return a < b ? a : b; }
static inline float fmax_sel(float a, float b) { return a > b ? a : b; }

static inline F4 f4min(F4 a, F4 b) { return {fmin_sel(a.x, b.x), fmin_sel(a.y, b.y), fmin_sel(a.z, b.z), fmin_sel(a.w, b.w)}; }
static inline F4 f4max(F4 a, F4 b) { return {fmax_sel(a.x, b.x), fmax_sel(a.y, b.y), fmax_sel(a.z, b.z), fmax_sel(a.w, b.w)}; }
static inline F4 f4sub(F4 a, F4 b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
static inline F4 f4add(F4 a, F4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
static inline F4 f4scale(F4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
// dot over 4 components, summed left to right (types/_cuda_float4.h:171-174)
static inline float dot4(F4 a, F4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
// cross with w = 0 (types/_cuda_float4.h:198-208)
static inline F4 cross4(F4 a, F4 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0f};
}
// normalize = v * rsqrtf(dot(v,v)); host rsqrtf is 1/sqrtf (types/_cuda_float.h:21-24)
static inline F4 normalize4(F4 v) { float inv = 1.0f / sqrtf(dot4(v, v)); return f4scale(v, inv); }

// float -> uint conversion with the GPU's saturating round-toward-zero rule
// (NaN and negatives give 0, values >= 2^32 give 0xFFFFFFFF); the reference
// casts with (uint) inside a kernel (kernels/CUDA_buildMeshTreeLBVH.cu:132-134).
static inline u32 f2u_rz_sat(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xFFFFFFFFu;
  return (u32)x;
}

// ---------------------------------------------------------------------------
// Stage 1: per-triangle boxes and iota (kernels/CUDA_calcMeshBoxes.cu:30-58)
// ---------------------------------------------------------------------------
OR_API void or_mesh_boxes(const float* vertices, const u32* faces, u32 n, float* boxes_out, u32* indices_out) {
  const F4* v = (const F4*)vertices;
  const U4* f = (const U4*)faces;
  Box* b = (Box*)boxes_out;
#pragma omp parallel for schedule(static)
  for (long k = 0; k < (long)n; ++k) {
    U4 face = f[k];
    Box bx;
    bx.mn = v[face.x]; bx.mx = v[face.x];          // aabox::reset(v0)
    bx.mn = f4min(bx.mn, v[face.y]); bx.mx = f4max(bx.mx, v[face.y]);  // merge(v1)
    bx.mn = f4min(bx.mn, v[face.z]); bx.mx = f4max(bx.mx, v[face.z]);  // merge(v2)
    b[k] = bx;
    if (indices_out) indices_out[k] = (u32)k;      // kernel_initIndices
  }
}

// Mesh hitbox as CUDAModel builds it: reset() then merge() of every vertex
// (CUDAModel.cpp:35, CUDAModel.h:178-183).
OR_API void or_hitbox(const float* vertices, u32 vertex_count, float* hit_out) {
  const F4* v = (const F4*)vertices;
  F4 mn = {kHuge, kHuge, kHuge, kHuge}, mx = {-kHuge, -kHuge, -kHuge, -kHuge};
  for (u32 i = 0; i < vertex_count; ++i) { mn = f4min(mn, v[i]); mx = f4max(mx, v[i]); }
  memcpy(hit_out, &mn, 16); memcpy(hit_out + 4, &mx, 16);
}

// ---------------------------------------------------------------------------
// Stage 2: Morton codes (kernels/CUDA_buildMeshTreeLBVH.cu:115-173).
// layout 32: the reference's 11/11/10 interleave (bit 3k = y_k, 3k+1 = x_k,
// 3k+2 = z_k). layout 30: 10 bits per axis, left aligned by 2 so that level L
// (bit 31-L) keeps axis L % 3 (x, y, z from the top).
// ---------------------------------------------------------------------------
static inline u32 morton_code(const Box& b, F4 hmin, F4 hmax, int layout) {
  F4 len = f4sub(hmax, hmin);
  float sx, sy, sz;
  if (layout == 30) { sx = 1023.0f / len.x; sy = 1023.0f / len.y; sz = 1023.0f / len.z; }
  else { sx = 2047.0f / len.x; sy = 2047.0f / len.y; sz = 1023.0f / len.z; }
  F4 c = f4scale(f4add(b.mn, b.mx), 0.5f);
  u32 qx = f2u_rz_sat((c.x - hmin.x) * sx);
  u32 qy = f2u_rz_sat((c.y - hmin.y) * sy);
  u32 qz = f2u_rz_sat((c.z - hmin.z) * sz);
  u32 code = 0;
  if (layout == 30) {
    for (int k = 0; k < 10; ++k) {
      code |= ((qz >> k) & 1u) << (3 * k + 2);
      code |= ((qy >> k) & 1u) << (3 * k + 3);
      code |= ((qx >> k) & 1u) << (3 * k + 4);
    }
  } else {
    for (int k = 0; k < 11; ++k) {
      code |= ((qy >> k) & 1u) << (3 * k + 0);
      code |= ((qx >> k) & 1u) << (3 * k + 1);
      if (k < 10) code |= ((qz >> k) & 1u) << (3 * k + 2);
    }
  }
  return code;
}

OR_API void or_morton(const float* boxes, u32 n, const float* hitbox, int layout, u32* codes_out) {
  const Box* b = (const Box*)boxes;
  F4 hmin, hmax; memcpy(&hmin, hitbox, 16); memcpy(&hmax, hitbox + 4, 16);
#pragma omp parallel for schedule(static)
  for (long k = 0; k < (long)n; ++k) codes_out[k] = morton_code(b[k], hmin, hmax, layout);
}

// ---------------------------------------------------------------------------
// Stage 3: stable key+index sort. The reference guarantees ascending keys
// (samples/09_how_to_use_a_sorter.cpp:94-241); this build's contract breaks
// ties by the incoming order (stable), i.e. by triangle index when the values
// start as 0..n-1. Keys are compared on their low 8*ceil(bit_depth/8) bits,
// the digits the reference's radix path sorts (kernels/CUDA_radixSortGeneral.cu:397-482).
// LSD radix, 8-bit digits.
// ---------------------------------------------------------------------------
OR_API void or_sort_pairs(u32* keys, u32* vals, u32 n, u32 bit_depth, int init_vals) {
  if (init_vals && vals) for (u32 i = 0; i < n; ++i) vals[i] = i;
  if (n < 2) return;
  u32 bytes = bit_depth == 0 ? 1 : 1 + (bit_depth - 1) / 8;
  if (bytes > 4) bytes = 4;
  std::vector<u32> k2(n), v2(vals ? n : 0);
  u32* ks = keys; u32* vs = vals; u32* kd = k2.data(); u32* vd = vals ? v2.data() : nullptr;
  for (u32 pass = 0; pass < bytes; ++pass) {
    u32 shift = 8 * pass, cnt[257] = {0};
    for (u32 i = 0; i < n; ++i) cnt[((ks[i] >> shift) & 255u) + 1]++;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (u32 i = 0; i < n; ++i) {
      u32 pos = cnt[(ks[i] >> shift) & 255u]++;
      kd[pos] = ks[i];
      if (vs) vd[pos] = vs[i];
    }
    std::swap(ks, kd); std::swap(vs, vd);
  }
  if (ks != keys) { memcpy(keys, ks, n * 4); if (vals) memcpy(vals, vs, n * 4); }
}

// ---------------------------------------------------------------------------
// Stage 4: split list (kernels/CUDA_buildMeshTreeLBVH.cu:175-233) ordered as the
// reference orders it before the host recursion (:565-594): by level, and by
// position inside each level. The reference sorts levels 1..tree_depth by
// position; deeper levels keep the order of the atomic appends, which is not
// deterministic. Here every level is sorted by position, and reads that land
// in those deeper lists are counted (nondet_reads).
// ---------------------------------------------------------------------------
struct SplitLists {
  std::vector<u32> C;     // concatenated positions, level 0 first
  u32 start[34];          // start[L] .. start[L+1]: level L; start[32] = S
};

static void find_splits(const u32* codes, u32 n, SplitLists& sl) {
  u32 count[32] = {0};
  for (u32 i = 0; i + 1 < n; ++i) {
    u32 d = codes[i] ^ codes[i + 1];
    if (d) count[__builtin_clz(d)]++;
  }
  sl.start[0] = 0;
  for (int L = 0; L < 32; ++L) sl.start[L + 1] = sl.start[L] + count[L];
  sl.start[33] = sl.start[32];
  sl.C.assign(sl.start[32], 0);
  u32 fill[32];
  for (int L = 0; L < 32; ++L) fill[L] = sl.start[L];
  for (u32 i = 0; i + 1 < n; ++i) {
    u32 d = codes[i] ^ codes[i + 1];
    if (d) sl.C[fill[__builtin_clz(d)]++] = i + 1;
  }
}

// ---------------------------------------------------------------------------
// Stage 5: topology, the host recursion of kernels/CUDA_buildMeshTreeLBVH.cu:309-455.
//  * morton_node (:360-411): leaf if the range is smaller than min_leaf, if the
//    level is tree_depth, or if the level's split pointer sits exactly at the
//    start of the next level's list; otherwise the pointer advances past every
//    split <= the range start (it can run into the next levels' lists); the
//    split found ends the range (leaf) or cuts it (internal node, axis = level % 3).
//  * leaf (:341-358): with tree_complete, a range larger than max_leaf becomes
//    a median node instead.
//  * median_node (:314-339): leaf if smaller than max_leaf, else split at
//    (a+b)>>1.
//  * Node numbering: the k-th internal node in pre-order gets children 2k+1, 2k+2.
// ---------------------------------------------------------------------------
struct TopoStats {
  u32 node_count, leaf_count, real_depth, split_count;
  u32 overrun_visits;   // visits whose split search left the level's own list
  u32 nondet_reads;     // visits whose scan stopped in a list deeper than tree_depth (unsorted in the reference)
  u32 past_end_reads;   // visits whose scan ran past the end of the split list (undefined in the reference)
  u32 error;            // 1 = node capacity exceeded
};

struct Topo {
  const SplitLists* sl;
  u32 ptr[33];
  u32 D, min_leaf, max_leaf; bool complete;
  Node* nodes; u32 cap; u32 count; u32 real_depth;
  TopoStats st;
};

static void put_node(Topo& t, u32 id, const Node& nd) {
  if (id < t.cap) t.nodes[id] = nd; else t.st.error = 1;
}

static Node make_internal(u32 axis, u32 child) {
  Node n; n.w0 = (axis & 3u) << 1; n.w1 = child;
  for (int i = 0; i < 3; ++i) { n.bmin[i] = kHuge; n.bmax[i] = -kHuge; }
  return n;
}
static Node make_leaf(u32 first, u32 count) {
  Node n; n.w0 = 1u | (count << 1); n.w1 = first;
  for (int i = 0; i < 3; ++i) { n.bmin[i] = kHuge; n.bmax[i] = -kHuge; }
  return n;
}

static void median_node(Topo& t, u32 a, u32 b, u32 lvl, u32 id);

static void leaf_node(Topo& t, u32 a, u32 b, u32 lvl, u32 id) {
  if (t.complete && b - a > t.max_leaf) { median_node(t, a, b, lvl, id); return; }
  if (lvl > t.real_depth) t.real_depth = lvl;
  put_node(t, id, make_leaf(a, b - a));
  t.st.leaf_count++;
}

static void median_node(Topo& t, u32 a, u32 b, u32 lvl, u32 id) {
  if (b - a < t.max_leaf) { leaf_node(t, a, b, lvl, id); return; }
  u32 mid = (a + b) >> 1;
  u32 left = ++t.count, right = ++t.count;
  put_node(t, id, make_internal(lvl % 3, left));
  median_node(t, a, mid, lvl + 1, left);
  median_node(t, mid, b, lvl + 1, right);
}

static void morton_node(Topo& t, u32 a, u32 b, u32 lvl, u32 id) {
  const SplitLists& sl = *t.sl;
  const u32 S = sl.start[32];
  if (b - a < t.min_leaf || lvl == t.D || t.ptr[lvl] == sl.start[lvl + 1]) { leaf_node(t, a, b, lvl, id); return; }
  u32 s;
  bool left_own_list = false;
  for (;;) {
    u32 j = t.ptr[lvl];
    if (j >= sl.start[lvl + 1]) left_own_list = true;
    if (j >= S) s = 0xFFFFFFFFu;
    else s = sl.C[j];
    if (s >= b || s > a) break;
    t.ptr[lvl]++;
  }
  {
    // per-visit statistics on the index where the scan stopped
    u32 j = t.ptr[lvl];
    if (left_own_list) t.st.overrun_visits++;
    if (j >= S) t.st.past_end_reads++;
    else if (sl.start[t.D + 1] < S && j >= sl.start[t.D + 1]) t.st.nondet_reads++;
  }
  if (s >= b) { leaf_node(t, a, b, lvl, id); return; }
  u32 left = ++t.count, right = ++t.count;
  put_node(t, id, make_internal(lvl % 3, left));
  morton_node(t, a, s, lvl + 1, left);
  morton_node(t, s, b, lvl + 1, right);
}

// Builds the topology from sorted codes. Returns the node count; stats in st_out (8 x u32).
OR_API u32 or_build_topology(const u32* sorted_codes, u32 n, u32 tree_depth, int tree_complete,
                             u32 min_leaf, u32 max_leaf, float* nodes_out, u32 node_cap, u32* st_out) {
  SplitLists sl;
  find_splits(sorted_codes, n, sl);
  Topo t;
  t.sl = &sl;
  if (tree_depth > 32) tree_depth = 32;
  for (u32 L = 0; L <= 32; ++L) t.ptr[L] = sl.start[L];
  t.D = tree_depth; t.min_leaf = min_leaf ? min_leaf : kMinLeafDefault; t.max_leaf = max_leaf ? max_leaf : kMaxLeafDefault;
  t.complete = tree_complete != 0;
  t.nodes = (Node*)nodes_out; t.cap = node_cap; t.count = 0; t.real_depth = 0;
  memset(&t.st, 0, sizeof(t.st));
  t.st.split_count = sl.start[32];
  if (n > 0) morton_node(t, 0, n, 0, 0);
  else { put_node(t, 0, make_leaf(0, 0)); t.st.leaf_count = 1; }
  t.st.node_count = t.count + 1;
  t.st.real_depth = t.real_depth + 1;
  if (st_out) memcpy(st_out, &t.st, sizeof(t.st));
  return t.st.node_count;
}

// ---------------------------------------------------------------------------
// Stage 6: node boxes (kernels/CUDA_buildMeshTreeLBVH.cu:235-303,620-649).
// Leaf: merge of the triangle boxes of its range (through indices). Internal:
// min/max of its children once both children have a positive z extent; a
// child whose z extent is not positive (a flat z leaf, or an ancestor of one)
// leaves the parent at its initial inverted box, which is what the reference's
// "done" test produces after real_depth passes. Children ids exceed their
// parent's id, so one sweep in decreasing id order is bottom-up.
// ---------------------------------------------------------------------------
OR_API void or_node_boxes(float* nodes_io, u32 node_count, const float* boxes, const u32* indices) {
  Node* nd = (Node*)nodes_io;
  const Box* bx = (const Box*)boxes;
#pragma omp parallel for schedule(dynamic, 64)
  for (long k = 0; k < (long)node_count; ++k) {
    Node& q = nd[k];
    if (!(q.w0 & 1u)) continue;
    u32 first = q.w1, cnt = q.w0 >> 1;
    F4 mn = {kHuge, kHuge, kHuge, kHuge}, mx = {-kHuge, -kHuge, -kHuge, -kHuge};
    for (u32 i = first; i < first + cnt; ++i) { const Box& b = bx[indices[i]]; mn = f4min(mn, b.mn); mx = f4max(mx, b.mx); }
    q.bmin[0] = mn.x; q.bmin[1] = mn.y; q.bmin[2] = mn.z;
    q.bmax[0] = mx.x; q.bmax[1] = mx.y; q.bmax[2] = mx.z;
  }
  for (long k = (long)node_count - 1; k >= 0; --k) {
    Node& q = nd[k];
    if (q.w0 & 1u) continue;
    const Node& l = nd[q.w1];
    const Node& r = nd[q.w1 + 1];
    if (l.bmax[2] - l.bmin[2] > 0.0f && r.bmax[2] - r.bmin[2] > 0.0f) {
      for (int i = 0; i < 3; ++i) { q.bmin[i] = fmin_sel(l.bmin[i], r.bmin[i]); q.bmax[i] = fmax_sel(l.bmax[i], r.bmax[i]); }
    }
  }
}

// kernels/CUDA_reorderMeshFaces.cu:26-38 -- faces_out[i] = faces[indices[i]]
OR_API void or_reorder_faces(const u32* faces, const u32* indices, u32 n, u32* faces_out) {
  const U4* f = (const U4*)faces; U4* o = (U4*)faces_out;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i) o[i] = f[indices[i]];
}

// Triangles in position order as {v0, e1 = v1 - v0, e2 = v2 - v0} with w = 0,
// computed as kernels/CUDA_raytraceMeshTree.cu:168-176 does per test.
OR_API void or_pack_tris(const float* vertices, const u32* faces_reordered, u32 n, float* tris_out) {
  const F4* v = (const F4*)vertices; const U4* f = (const U4*)faces_reordered; F4* o = (F4*)tris_out;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i) {
    U4 face = f[i];
    F4 v0 = v[face.x];
    F4 e1 = f4sub(v[face.y], v0);
    F4 e2 = f4sub(v[face.z], v0);
    v0.w = 0.0f; e1.w = 0.0f; e2.w = 0.0f;
    o[3 * i + 0] = v0; o[3 * i + 1] = e1; o[3 * i + 2] = e2;
  }
}

// Whole build: boxes, Morton, sort, topology, node boxes, reorder, pack.
// info_out: node_count, leaf_count, real_depth, split_count, overrun_visits,
// nondet_reads, past_end_reads, error.
OR_API u32 or_lbvh_build(const float* vertices, u32 vertex_count, const u32* faces, u32 n,
                         const float* hitbox_or_null, u32 tree_depth, int tree_complete, int layout,
                         float* boxes_out, u32* indices_out, u32* codes_out,
                         float* nodes_out, u32 node_cap, u32* faces_out, float* tris_out, u32* info_out) {
  float hit[8];
  if (hitbox_or_null) memcpy(hit, hitbox_or_null, 32); else or_hitbox(vertices, vertex_count, hit);
  or_mesh_boxes(vertices, faces, n, boxes_out, indices_out);
  or_morton(boxes_out, n, hit, layout, codes_out);
  or_sort_pairs(codes_out, indices_out, n, 32, 0);
  u32 st[8];
  u32 nc = or_build_topology(codes_out, n, tree_depth, tree_complete, kMinLeafDefault, kMaxLeafDefault, nodes_out, node_cap, st);
  if (nc <= node_cap) or_node_boxes(nodes_out, nc, boxes_out, indices_out);
  if (tree_complete) {
    if (faces_out) or_reorder_faces(faces, indices_out, n, faces_out);
    if (tris_out && faces_out) or_pack_tris(vertices, faces_out, n, tris_out);
  }
  if (info_out) memcpy(info_out, st, sizeof(st));
  return nc;
}

// ---------------------------------------------------------------------------
// SAH / Hybrid build (kernels/CUDA_buildMeshTreeSAH.cu:224-789,
// CUDAMeshTree.cpp:93-103). The reference keeps a global stack of work items
// (node id, node box, face range); each launch runs one 32-thread block per
// stacked item and every block pops one item, bins its faces' centroids on the
// longest axis of their bounds into 32 bins, and either writes a leaf or
// allocates two child ids with atomicAdd and pushes (right, left). Executed
// serially (one block at a time), pops are depth first, left child first, so a
// node is split in pre-order and the k-th split of a subtree whose root was
// popped when the node counter stood at B gets children B + 2k, B + 2k + 1.
// That serial order is the contract here (the GPU's concurrent blocks number
// nodes in a racy order). One departure: a node of >= 224 faces for which no
// bin boundary separates two non-empty sides (every centroid in one bin, or a
// degenerate parent box) becomes a leaf; the reference never terminates there.
// Arithmetic as written (no contraction); box min / max as omin / omax below.
// ---------------------------------------------------------------------------
namespace sah {
const int kBins = 32;                      // SM_BIN_COUNT, :48
const float kTriCost = 0.125f;             // TRI_RAY_COST, :52
const float kBoxCost = 1.0f;               // BOX_RAY_COST, :53
const u32 kMinLeaf = 16, kMaxLeaf = 224;   // :55-56

struct Item { F4 mn, mx; u32 node, first, bound; };
struct Bin { float bmin[3], bmax[3]; int count, lcount, rcount; float larea, rarea; };

// min / max in the order of the floats' bit patterns read as sign-magnitude
// (-0 < +0; the reference's fminf leaves that tie unspecified), as the GPU's
// ordered-key atomics compute them
static inline u32 ordkey(float f) { u32 u; memcpy(&u, &f, 4); return (u & 0x80000000u) ? ~u : (u | 0x80000000u); }
static inline float omin(float a, float b) { return ordkey(b) < ordkey(a) ? b : a; }
static inline float omax(float a, float b) { return ordkey(b) > ordkey(a) ? b : a; }
static inline F4 f4fmin(F4 a, F4 b) { return {omin(a.x, b.x), omin(a.y, b.y), omin(a.z, b.z), omin(a.w, b.w)}; }
static inline F4 f4fmax(F4 a, F4 b) { return {omax(a.x, b.x), omax(a.y, b.y), omax(a.z, b.z), omax(a.w, b.w)}; }
// aabox::getArea (CUDABox.h:35-45)
static inline float area(F4 mn, F4 mx) {
  const F4 v = f4sub(mx, mn);
  return 2.f * (v.x * v.y + v.x * v.z + v.y * v.z);
}
// (int) of a float inside a kernel: round toward zero, saturating, NaN -> 0
static inline int f2i_rz_sat(float x) {
  if (x != x) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (int)0x80000000u;
  return (int)x;
}
static inline float comp(F4 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

static void write_leaf(Node* nodes, u32 id, F4 mn, F4 mx, u32 first, u32 count) {
  Node& o = nodes[id];
  o.w0 = 1u | (count << 1);
  o.w1 = first;
  o.bmin[0] = mn.x; o.bmin[1] = mn.y; o.bmin[2] = mn.z;
  o.bmax[0] = mx.x; o.bmax[1] = mx.y; o.bmax[2] = mx.z;
}
static void write_node(Node* nodes, u32 id, F4 mn, F4 mx, int axis, u32 child) {
  Node& o = nodes[id];
  o.w0 = (u32)axis << 1;
  o.w1 = child;
  o.bmin[0] = mn.x; o.bmin[1] = mn.y; o.bmin[2] = mn.z;
  o.bmax[0] = mx.x; o.bmax[1] = mx.y; o.bmax[2] = mx.z;
}
}  // namespace sah

// boxes: aabox per original face; indices: face ids in position order (in/out);
// nodes_in / node_count_in: an existing tree whose leaves are refined (Hybrid),
// or node_count_in = 0 for a full SAH build from root_box. Returns 0 or 2 when
// the node capacity would be exceeded. stats[0] = leaves made because no bin
// boundary splits a node of >= 224 faces.
OR_API int or_sah_build(const float* boxes_f, const float* root_box, u32* indices, u32 n, const float* nodes_in, u32 node_count_in,
                        float* nodes_out, u32 capacity, u32* node_count_out, u32* stats) {
  using namespace sah;
  const Box* boxes = (const Box*)boxes_f;
  Node* nodes = (Node*)nodes_out;
  std::vector<Item> stack;
  std::vector<u32> tmp(n);
  u32 node_count = 0, no_split = 0;
  if (node_count_in == 0) {
    Item it;
    memcpy(&it.mn, root_box, 16);
    memcpy(&it.mx, root_box + 4, 16);
    it.node = 0; it.first = 0; it.bound = n;
    stack.push_back(it);
    node_count = 1;
  } else {
    if (node_count_in > capacity) return 2;
    memcpy(nodes, nodes_in, (size_t)node_count_in * sizeof(Node));
    node_count = node_count_in;
    for (u32 k = 0; k < node_count_in; ++k) {  // kernel_initStack (:647-666), threads in order
      const Node& b = nodes[k];
      if (!(b.w0 & 1u)) continue;
      Item it;
      it.mn = {b.bmin[0], b.bmin[1], b.bmin[2], 0.0f};
      it.mx = {b.bmax[0], b.bmax[1], b.bmax[2], 0.0f};
      it.node = k; it.first = b.w1; it.bound = b.w1 + (b.w0 >> 1);
      stack.push_back(it);
    }
  }
  while (!stack.empty()) {
    const Item it = stack.back();
    stack.pop_back();
    const u32 cnt = it.bound - it.first;
    if (cnt <= kMinLeaf) { write_leaf(nodes, it.node, it.mn, it.mx, it.first, cnt); continue; }
    // centroid bounds and the longest axis (:275-345)
    F4 cmn = {kHuge, kHuge, kHuge, kHuge}, cmx = {-kHuge, -kHuge, -kHuge, -kHuge};
    for (u32 l = it.first; l < it.bound; ++l) {
      const Box& b = boxes[indices[l]];
      const F4 c = f4scale(f4add(b.mn, b.mx), 0.5f);
      cmn = f4fmin(cmn, c);
      cmx = f4fmax(cmx, c);
    }
    const F4 ext = f4sub(cmx, cmn);
    int axis;
    if (ext.x > ext.y) axis = ext.x > ext.z ? 0 : 2;
    else axis = ext.y > ext.z ? 1 : 2;
    const float scale = (float)(kBins - 1) / comp(ext, axis);
    const float bmin = comp(cmn, axis);
    // binning (:356-409)
    Bin bins[kBins];
    for (int m = 0; m < kBins; ++m) {
      for (int k = 0; k < 3; ++k) { bins[m].bmin[k] = kHuge; bins[m].bmax[k] = -kHuge; }
      bins[m].count = bins[m].lcount = bins[m].rcount = 0;
      bins[m].larea = bins[m].rarea = 0.f;
    }
    std::vector<unsigned char> bin_of(cnt);
    for (u32 l = it.first; l < it.bound; ++l) {
      const Box& b = boxes[indices[l]];
      const F4 c = f4scale(f4add(b.mn, b.mx), 0.5f);
      int m = f2i_rz_sat((comp(c, axis) - bmin) * scale);
      if (m < 0) m = 0;
      else if (m >= kBins - 1) m = kBins - 1;
      bin_of[l - it.first] = (unsigned char)m;
      Bin& q = bins[m];
      q.bmin[0] = omin(q.bmin[0], b.mn.x); q.bmin[1] = omin(q.bmin[1], b.mn.y); q.bmin[2] = omin(q.bmin[2], b.mn.z);
      q.bmax[0] = omax(q.bmax[0], b.mx.x); q.bmax[1] = omax(q.bmax[1], b.mx.y); q.bmax[2] = omax(q.bmax[2], b.mx.z);
      q.count++;
    }
    // sweeps and the cost of every boundary (:423-474, bvbin::getSAH CUDABin.h:104-111)
    F4 lmn = {kHuge, kHuge, kHuge, kHuge}, lmx = {-kHuge, -kHuge, -kHuge, -kHuge};
    int lcount = 0;
    for (int m = 0; m < kBins - 1; ++m) {
      lcount += bins[m].count;
      lmn = {omin(lmn.x, bins[m].bmin[0]), omin(lmn.y, bins[m].bmin[1]), omin(lmn.z, bins[m].bmin[2]), lmn.w};
      lmx = {omax(lmx.x, bins[m].bmax[0]), omax(lmx.y, bins[m].bmax[1]), omax(lmx.z, bins[m].bmax[2]), lmx.w};
      bins[m].larea += area(lmn, lmx);
      bins[m].lcount += lcount;
    }
    const float parent_area = area(it.mn, it.mx);
    float t_min = kHuge;
    int m_min = -1;
    F4 rmn = {kHuge, kHuge, kHuge, kHuge}, rmx = {-kHuge, -kHuge, -kHuge, -kHuge};
    int rcount = 0;
    for (int m = kBins - 1; m > 0; --m) {
      rcount += bins[m].count;
      rmn = {omin(rmn.x, bins[m].bmin[0]), omin(rmn.y, bins[m].bmin[1]), omin(rmn.z, bins[m].bmin[2]), rmn.w};
      rmx = {omax(rmx.x, bins[m].bmax[0]), omax(rmx.y, bins[m].bmax[1]), omax(rmx.z, bins[m].bmax[2]), rmx.w};
      Bin& q = bins[m - 1];
      q.rarea += area(rmn, rmx);
      q.rcount += rcount;
      const float t = kBoxCost * 2.f + kTriCost * ((q.larea / parent_area) * q.lcount + (q.rarea / parent_area) * q.rcount);
      if (t < t_min) { t_min = t; m_min = m - 1; }
    }
    // leaf by cost (:479-496); no usable boundary -> leaf (departure, see above)
    if ((cnt < kMaxLeaf && t_min > (float)(cnt + 1) * kTriCost) || m_min < 0) {
      if (m_min < 0 && cnt >= kMaxLeaf) ++no_split;
      write_leaf(nodes, it.node, it.mn, it.mx, it.first, cnt);
      continue;
    }
    // child boxes and the stable partition (:498-613)
    F4 a_mn = {kHuge, kHuge, kHuge, kHuge}, a_mx = {-kHuge, -kHuge, -kHuge, -kHuge};
    F4 b_mn = a_mn, b_mx = a_mx;
    u32 nl = 0;
    for (int m = 0; m < kBins; ++m) {
      F4& mn = m <= m_min ? a_mn : b_mn;
      F4& mx = m <= m_min ? a_mx : b_mx;
      mn = {omin(mn.x, bins[m].bmin[0]), omin(mn.y, bins[m].bmin[1]), omin(mn.z, bins[m].bmin[2]), mn.w};
      mx = {omax(mx.x, bins[m].bmax[0]), omax(mx.y, bins[m].bmax[1]), omax(mx.z, bins[m].bmax[2]), mx.w};
      if (m <= m_min) nl += (u32)bins[m].count;
    }
    u32 li = it.first, ri = it.first + nl;
    for (u32 l = it.first; l < it.bound; ++l) {
      if (bin_of[l - it.first] <= m_min) tmp[li++] = indices[l];
      else tmp[ri++] = indices[l];
    }
    memcpy(indices + it.first, tmp.data() + it.first, (size_t)cnt * 4);
    if (node_count + 2 > capacity) return 2;
    const u32 c = node_count;
    node_count += 2;
    write_node(nodes, it.node, it.mn, it.mx, axis, c);
    stack.push_back(Item{b_mn, b_mx, c + 1, it.first + nl, it.bound});
    stack.push_back(Item{a_mn, a_mx, c, it.first, it.first + nl});
  }
  *node_count_out = node_count;
  if (stats) stats[0] = no_split;
  return 0;
}

// ---------------------------------------------------------------------------
// Rasteriser (kernels/CUDA_rasterizeMeshTree.cu:47-225, camera matrices of
// CUDACamera::update, CUDACamera.cpp:245-266, types/_cuda_float4x4.h).
// Per pixel the faces are tested in face order and the first face with the
// smallest depth t > 0 wins (strict <). The pixel point is the pixel's corner
// (x * 2 / width - 1, 1 - y * 2 / height); a face is tested on the 8 x 4 pixel
// zones of its screen rectangle (start rounded down to an even zone). Face id
// out = the face's index (the reference writes the first index of the face's
// 192-face cache block, see the callers).
// ---------------------------------------------------------------------------
namespace raster {
struct M4 { F4 r0, r1, r2, r3; };
static inline F4 row(const M4& m, int i) { return i == 0 ? m.r0 : (i == 1 ? m.r1 : (i == 2 ? m.r2 : m.r3)); }
static M4 transpose(const M4& m) {
  M4 r;
  r.r0 = {m.r0.x, m.r1.x, m.r2.x, m.r3.x};
  r.r1 = {m.r0.y, m.r1.y, m.r2.y, m.r3.y};
  r.r2 = {m.r0.z, m.r1.z, m.r2.z, m.r3.z};
  r.r3 = {m.r0.w, m.r1.w, m.r2.w, m.r3.w};
  return r;
}
// r_ij = dot(a_i, column j of b)  (matrixMultiply)
static M4 multiply(const M4& a, const M4& b) {
  const M4 t = transpose(b);
  M4 r;
  F4* rr[4] = {&r.r0, &r.r1, &r.r2, &r.r3};
  for (int i = 0; i < 4; ++i) {
    const F4 ai = row(a, i);
    *rr[i] = {dot4(ai, t.r0), dot4(ai, t.r1), dot4(ai, t.r2), dot4(ai, t.r3)};
  }
  return r;
}
static F4 transform(const M4& m, F4 v) { return {dot4(m.r0, v), dot4(m.r1, v), dot4(m.r2, v), dot4(m.r3, v)}; }
// (int) inside a kernel: toward zero, saturating, NaN -> 0
static inline int f2i(float x) {
  if (x != x) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (int)0x80000000u;
  return (int)x;
}
}  // namespace raster

// transpose(view * proj) for a camera at center3 looking along dir3 (the
// normalized lookAt direction), roll angle3[2], fov / ratio; near 1.0, far 1999.999.
OR_API void or_raster_matrix(const float* center3, const float* dir3, const float* angle3, float fov, float ratio, float* out16) {
  using namespace raster;
  const float cx = center3[0], cy = center3[1], cz = center3[2];
  const float dx = dir3[0], dy = dir3[1], dz = dir3[2];
  // target = center + 4999.999 dir; normal = (dir.x, 0, dir.y) (CUDACamera.cpp:247-248)
  const float tx = cx + dx * 4999.999f, ty = cy + dy * 4999.999f, tz = cz + dz * 4999.999f;
  float nx = dx, ny = 0.0f, nz = dy;
  const float ninv = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
  nx = nx * ninv; ny = ny * ninv; nz = nz * ninv;
  // matrixRotationAxis(normal, angle.z) (types/_cuda_float4x4.h:323-350)
  const float u = cosf(angle3[2]), v = sinf(angle3[2]), w = 1.0f - u;
  M4 up_m;
  up_m.r0 = {w * nx * nx + u, w * nx * ny - v * nz, w * nx * nz + v * ny, 0.0f};
  up_m.r1 = {w * ny * nx + v * nz, w * ny * ny + u, w * ny * nz - v * nx, 0.0f};
  up_m.r2 = {w * nz * nx - v * ny, w * nz * ny + v * nx, w * nz * nz + u, 0.0f};
  up_m.r3 = {0.0f, 0.0f, 0.0f, 1.0f};
  const F4 eye = {cx, cy, cz, 0.0f}, at = {tx, ty, tz, 0.0f};
  const F4 up = transform(up_m, {0.0f, 1.0f, 0.0f, 1.0f});
  // matrixLookAt (:412-426)
  const F4 za = normalize4(f4sub(at, eye));
  const F4 xa = normalize4(cross4(up, za));
  const F4 ya = cross4(za, xa);
  const float xf = -dot4(xa, eye), yf = -dot4(ya, eye), zf = -dot4(za, eye);
  M4 view;
  view.r0 = {xa.x, ya.x, za.x, 0.0f};
  view.r1 = {xa.y, ya.y, za.y, 0.0f};
  view.r2 = {xa.z, ya.z, za.z, 0.0f};
  view.r3 = {xf, yf, zf, 1.0f};
  // matrixPerspectiveFov (:398-410)
  const float z_near = 1.000f, z_far = 1999.999f;
  const float ys = 1.0f / tanf(fov * 0.5f);
  const float xs = ys / ratio;
  const float zfac = z_far / (z_far - z_near);
  const float wfac = -z_near * zfac;
  M4 proj;
  proj.r0 = {xs, 0.0f, 0.0f, 0.0f};
  proj.r1 = {0.0f, ys, 0.0f, 0.0f};
  proj.r2 = {0.0f, 0.0f, zfac, 1.0f};
  proj.r3 = {0.0f, 0.0f, wfac, 0.0f};
  const M4 m = transpose(multiply(view, proj));
  memcpy(out16, &m, 64);
}

// faces_id / coords / depths are read (the caller clears them) and updated.
OR_API void or_rasterize(const float* vertices, const u32* faces, u32 face_count, const float* matrix16, int width, int height,
                         u32* faces_id, float* coords, float* depths) {
  using namespace raster;
  M4 m;
  memcpy(&m, matrix16, 64);
  const F4* vtx = (const F4*)vertices;
  const U4* fc = (const U4*)faces;
  const int zcx = 1 + (width - 1) / 8, zcy = 1 + (height - 1) / 4;
  const float zsx = 0.5f * (float)zcx, zsy = 0.5f * (float)zcy;
  const float eps = 0.000001f;
  for (u32 f = 0; f < face_count; ++f) {
    F4 p[3];
    F4 mn = {kHuge, kHuge, kHuge, kHuge}, mx = {-kHuge, -kHuge, -kHuge, -kHuge};
    const u32 vid[3] = {fc[f].x, fc[f].y, fc[f].z};
    for (int k = 0; k < 3; ++k) {
      F4 vi = vtx[vid[k]];
      vi.w = 1.0f;
      F4 vo = transform(m, vi);
      const float inv = 1.0f / fabsf(vo.w);  // operator/= multiplies by the reciprocal
      vo = f4scale(vo, inv);
      vo.w = 0.0f;
      p[k] = vo;
      mn = {fminf(mn.x, vo.x), fminf(mn.y, vo.y), fminf(mn.z, vo.z), fminf(mn.w, vo.w)};
      mx = {fmaxf(mx.x, vo.x), fmaxf(mx.y, vo.y), fmaxf(mx.z, vo.z), fmaxf(mx.w, vo.w)};
    }
    if (!(mn.x < 1.0f && mx.x > -1.0f && mn.y < 1.0f && mx.y > -1.0f)) continue;
    int x0 = f2i(zsx * (mn.x + 1.0f)); x0 = (x0 > 0 ? x0 : 0) / 2 * 2;
    int y0 = f2i(zsy * (1.0f - mx.y)); y0 = (y0 > 0 ? y0 : 0) / 2 * 2;
    int x1 = f2i(zsx * (mx.x + 1.0f)); x1 = x1 < zcx - 1 ? x1 : zcx - 1;
    int y1 = f2i(zsy * (1.0f - mn.y)); y1 = y1 < zcy - 1 ? y1 : zcy - 1;
    const F4 a = p[0], b = p[1], c = p[2];
    for (int j = y0; j <= y1; ++j)
      for (int i = x0; i <= x1; ++i)
        for (int ty = 0; ty < 4; ++ty)
          for (int tx = 0; tx < 8; ++tx) {
            const int x = i * 8 + tx, y = j * 4 + ty;
            const float px = (float)x * 2.0f / (float)width - 1.0f;
            const float py = 1.0f - (float)y * 2.0f / (float)height;
            // intersectTriPoint (:52-71)
            const float det = (b.x - a.x) * (c.y - a.y) - (c.x - a.x) * (b.y - a.y);
            if (det > -eps && det < eps) continue;
            const float inv_det = 1.0f / det;
            const float uu = ((c.x - px) * (a.y - py) - (a.x - px) * (c.y - py)) * inv_det;
            if (uu < 0.0f || uu > 1.0f) continue;
            const float vv = ((a.x - px) * (b.y - py) - (b.x - px) * (a.y - py)) * inv_det;
            if (vv < 0.0f || uu + vv > 1.0f) continue;
            const float t = (1.0f - uu - vv) * a.z + uu * b.z + vv * c.z;
            if (x < 0 || x >= width || y < 0 || y >= height) continue;
            const long l = (long)y * width + x;
            if (t > 0 && t < depths[l]) {
              faces_id[l] = f;
              coords[2 * l] = uu;
              coords[2 * l + 1] = vv;
              depths[l] = t;
            }
          }
  }
}

// ---------------------------------------------------------------------------
// Camera and primary rays.
// lookAt / angleFromDir: CUDACamera.cpp:126-132, 70-88 (float3 normalize uses the
// host rsqrtf = 1/sqrtf). Basis and per-pixel directions:
// kernels/CUDA_calcPrimaryRays.cu:43-55 and :20-32.
// ---------------------------------------------------------------------------
static const float kPi = 3.14159265359f;  // CUDACommon.h:108

OR_API void or_camera_look_at(const float* center3, const float* target3, float* angle3_out) {
  float dx = target3[0] - center3[0], dy = target3[1] - center3[1], dz = target3[2] - center3[2];
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
  angle3_out[0] = ax; angle3_out[1] = ay; angle3_out[2] = 0.0f;
}

// out16: rayOrig, rayDir, rayX, rayY (float4 each)
OR_API void or_camera_basis(const float* center3, const float* angle3, float fov, float ratio, int width, int height, float* out16) {
  float y = tanf(fov * 0.5f);
  float x = y * ratio;
  float p = angle3[0], yw = angle3[1], r = angle3[2];
  F4 camDir = {cosf(p) * cosf(yw), sinf(yw), sinf(p) * cosf(yw), 0.0f};
  F4 camUp = {cosf(p) * sinf(r), cosf(r), 0.0f, 0.0f};
  F4 right = normalize4(cross4(camDir, camUp));
  F4 up = normalize4(cross4(right, camDir));
  F4 rayOrig = {center3[0], center3[1], center3[2], 0.0f};
  F4 rayDir = f4add(f4add(f4scale(up, y), f4scale(right, x)), camDir);
  F4 rayX = f4scale(f4scale(right, 2.0f * x), 1.0f / (float)width);
  F4 rayY = f4scale(f4scale(up, 2.0f * y), 1.0f / (float)height);
  memcpy(out16 + 0, &rayOrig, 16); memcpy(out16 + 4, &rayDir, 16);
  memcpy(out16 + 8, &rayX, 16); memcpy(out16 + 12, &rayY, 16);
}

OR_API void or_primary_rays(const float* basis16, int width, int height, float* orig_out, float* dir_out) {
  F4 o, d, rx, ry;
  memcpy(&o, basis16, 16); memcpy(&d, basis16 + 4, 16); memcpy(&rx, basis16 + 8, 16); memcpy(&ry, basis16 + 12, 16);
  F4* po = (F4*)orig_out; F4* pd = (F4*)dir_out;
#pragma omp parallel for schedule(static)
  for (long yy = 0; yy < height; ++yy)
    for (int xx = 0; xx < width; ++xx) {
      long n = yy * (long)width + xx;
      po[n] = o;
      pd[n] = f4sub(f4sub(d, f4scale(rx, (float)xx)), f4scale(ry, (float)yy));
    }
}

// ---------------------------------------------------------------------------
// Traversal.
// Möller-Trumbore exactly as kernels/CUDA_raytraceMeshTree.cu:57-89 (4-wide dot
// products; vert0/edge1/edge2 have w = 0, so the w products reduce to
// (ray.w * 0) terms which are kept for the sign of zero).
// ---------------------------------------------------------------------------
static inline bool mt_test(F4 o, F4 d, F4 v0, F4 e1, F4 e2, float& t, float& u, float& v) {
  F4 p = cross4(d, e2);
  float det = dot4(e1, p);
  if (det > -0.000001f && det < 0.000001f) return false;
  float inv = 1.0f / det;
  F4 tv = f4sub(o, v0);
  u = dot4(tv, p) * inv;
  if (u < 0.0f || u > 1.0f) return false;
  F4 q = cross4(tv, e1);
  v = dot4(d, q) * inv;
  if (v < 0.0 || u + v > 1.0f) return false;
  t = dot4(e2, q) * inv;
  return t >= 0.0f;
}

// Conservative slab test used by this build's traversal (not the reference's):
// the box is padded by 2^-13 of its largest coordinate magnitude per axis, a
// direction component smaller than 1e-20 in magnitude is replaced by +/-1e-20,
// and the entry distance is compared against 1.000122 x the best t. Identical
// arithmetic runs on the GPU, so visit counts match exactly.
struct RayPre { float ix, iy, iz; };
static inline RayPre ray_pre(F4 d) {
  auto fix = [](float c) { return fabsf(c) < 1e-20f ? copysignf(1e-20f, c) : c; };
  return {1.0f / fix(d.x), 1.0f / fix(d.y), 1.0f / fix(d.z)};
}
static inline bool box_test(const float* bmin, const float* bmax, F4 o, const RayPre& rp, float tbest, float* tnear_out) {
  const float kPad = 1.220703125e-4f;  // 2^-13
  float lo[3], hi[3];
  const float inv[3] = {rp.ix, rp.iy, rp.iz};
  const float oo[3] = {o.x, o.y, o.z};
  for (int a = 0; a < 3; ++a) {
    float m = fmax_sel(fabsf(bmin[a]), fabsf(bmax[a]));
    float pad = m * kPad;
    float t0 = ((bmin[a] - pad) - oo[a]) * inv[a];
    float t1 = ((bmax[a] + pad) - oo[a]) * inv[a];
    lo[a] = fmin_sel(t0, t1); hi[a] = fmax_sel(t0, t1);
  }
  float tn = fmax_sel(fmax_sel(lo[0], lo[1]), lo[2]);
  float tf = fmin_sel(fmin_sel(hi[0], hi[1]), hi[2]);
  *tnear_out = tn;
  return tn <= tf && tf >= 0.0f && tn <= tbest * 1.0001220703125f;
}

struct HitOut { int32_t* id; float* t; float* uv; u32* visits; u32* tests; };

// mode 0: this build's contract -- closest (t, position) over all triangles,
//         DFS in the reference order (pop, test node box, push far then near),
//         with the conservative box test above.
// mode 1: the reference's own traversal semantics, kernels/CUDA_raytraceMeshTree.cu:111-219:
//         box test with invdir = normalize(1/d) (rsqrtf taken as 1/sqrtf), CUDA
//         fminf/fmaxf (NaN-ignoring), first strictly smaller t wins in DFS order.
// id_mode 0: id = position in the reordered faces; 1: original triangle id via indices.
// Rays with depth_in <= 0 (or NaN) are misses. A miss returns id -1, t = depth_in, u = v = 0.
static void trace_one(long r, const Node* nodes, const F4* tris, const u32* indices, const F4* orig, const F4* dir,
                      const float* depth_in, int mode, int id_mode, HitOut out) {
  F4 o = orig[r], d = dir[r];
  float depth = depth_in ? depth_in[r] : kHuge;
  float tmax0 = depth;
  int32_t best = -1; float bu = 0.0f, bv = 0.0f;
  u32 visits = 0, tests = 0;
  if (depth > 0.0f) {
    RayPre rp = ray_pre(d);
    F4 invn = {0, 0, 0, 0};
    if (mode == 1) invn = normalize4(F4{1.0f / d.x, 1.0f / d.y, 1.0f / d.z, 0.0f});
    u32 stack[256]; int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      u32 nid = stack[--sp];
      const Node& nd = nodes[nid];
      visits++;
      if (nd.w0 & 1u) {
        u32 first = nd.w1, cnt = nd.w0 >> 1;
        for (u32 k = 0; k < cnt; ++k) {
          u32 pos = first + k;
          float t, u, v;
          tests++;
          if (!mt_test(o, d, tris[3 * pos], tris[3 * pos + 1], tris[3 * pos + 2], t, u, v)) continue;
          if (mode == 1) {
            if (t < depth) { best = (int32_t)pos; bu = u; bv = v; depth = t; }
          } else {
            if (!(t < tmax0)) continue;
            if (t < depth || (t == depth && best >= 0 && (int32_t)pos < best) || (t == depth && best < 0)) {
              best = (int32_t)pos; bu = u; bv = v; depth = t;
            }
          }
        }
      } else {
        bool pass; float tn;
        if (mode == 1) {
          F4 v1 = {(nd.bmin[0] - o.x) * invn.x, (nd.bmin[1] - o.y) * invn.y, (nd.bmin[2] - o.z) * invn.z, 0};
          F4 v2 = {(nd.bmax[0] - o.x) * invn.x, (nd.bmax[1] - o.y) * invn.y, (nd.bmax[2] - o.z) * invn.z, 0};
          float mnx = fminf(v1.x, v2.x), mny = fminf(v1.y, v2.y), mnz = fminf(v1.z, v2.z);
          float mxx = fmaxf(v1.x, v2.x), mxy = fmaxf(v1.y, v2.y), mxz = fmaxf(v1.z, v2.z);
          float tmin = fmaxf(mnz, fmaxf(mnx, mny));
          float tmx = fminf(mxz, fminf(mxx, mxy));
          pass = (tmx >= tmin) && (tmx >= 0.0f) && (tmin < depth);
          tn = tmin;
        } else {
          pass = box_test(nd.bmin, nd.bmax, o, rp, depth, &tn);
        }
        if (pass) {
          u32 axis = (nd.w0 >> 1) & 3u;
          float da = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
          u32 near_c = nd.w1, far_c = nd.w1 + 1;
          if (da < 0.f) { near_c = nd.w1 + 1; far_c = nd.w1; }
          if (sp + 2 <= 256) { stack[sp++] = far_c; stack[sp++] = near_c; }
        }
      }
    }
  }
  if (best >= 0) {
    out.id[r] = id_mode == 1 ? (int32_t)indices[best] : best;
    out.t[r] = depth; out.uv[2 * r] = bu; out.uv[2 * r + 1] = bv;
  } else {
    out.id[r] = -1; out.t[r] = tmax0; out.uv[2 * r] = 0.0f; out.uv[2 * r + 1] = 0.0f;
  }
  if (out.visits) out.visits[r] = visits;
  if (out.tests) out.tests[r] = tests;
}

OR_API void or_trace(const float* nodes, const float* tris, const u32* indices, const float* orig, const float* dir,
                     const float* depth_in_or_null, long ray_begin, long ray_end, int mode, int id_mode, int threads,
                     int32_t* id_out, float* t_out, float* uv_out, u32* visits_out, u32* tests_out) {
  HitOut out{id_out, t_out, uv_out, visits_out, tests_out};
#ifdef _OPENMP
  int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt)
#endif
  for (long r = ray_begin; r < ray_end; ++r)
    trace_one(r, (const Node*)nodes, (const F4*)tris, indices, (const F4*)orig, (const F4*)dir, depth_in_or_null, mode, id_mode, out);
}

// Brute force over every triangle: the closest (t, position) with t < depth_in.
OR_API void or_trace_brute(const float* tris, u32 n, const float* orig, const float* dir, const float* depth_in_or_null,
                           long ray_count, int32_t* id_out, float* t_out, float* uv_out) {
  const F4* tr = (const F4*)tris; const F4* po = (const F4*)orig; const F4* pd = (const F4*)dir;
#pragma omp parallel for schedule(dynamic, 64)
  for (long r = 0; r < ray_count; ++r) {
    float tmax0 = depth_in_or_null ? depth_in_or_null[r] : kHuge;
    float best_t = tmax0; int32_t best = -1; float bu = 0, bv = 0;
    if (tmax0 > 0.0f)
      for (u32 k = 0; k < n; ++k) {
        float t, u, v;
        if (!mt_test(po[r], pd[r], tr[3 * k], tr[3 * k + 1], tr[3 * k + 2], t, u, v)) continue;
        if (t < best_t) { best_t = t; best = (int32_t)k; bu = u; bv = v; }
      }
    id_out[r] = best; t_out[r] = best_t; uv_out[2 * r] = bu; uv_out[2 * r + 1] = bv;
  }
}

// ---------------------------------------------------------------------------
// Secondary rays for the incoherent workload: one cosine-weighted diffuse
// bounce per hit. This has no counterpart in the reference; it is input
// generation for the 1M-triangle scene and is restated here so that the GPU
// generator can be checked bit for bit. PCG32 is O'Neill's PCG-XSH-RR 64/32
// (pcg32_srandom_r / pcg32_random_r). The disk sample uses rejection (no
// transcendental functions), the frame is Duff et al. 2017's branchless ONB.
// A miss gives an inactive slot: zero origin and direction, depth -1.
// ---------------------------------------------------------------------------
struct Pcg { u64 state, inc; };
static inline u32 pcg_next(Pcg& g) {
  u64 old = g.state;
  g.state = old * 6364136223846793005ULL + g.inc;
  u32 xs = (u32)(((old >> 18u) ^ old) >> 27u);
  u32 rot = (u32)(old >> 59u);
  return (xs >> rot) | (xs << ((-rot) & 31u));
}
static inline void pcg_seed(Pcg& g, u64 initstate, u64 initseq) {
  g.state = 0u; g.inc = (initseq << 1u) | 1u; pcg_next(g); g.state += initstate; pcg_next(g);
}

OR_API void or_bounce_rays(const float* tris, const float* orig, const float* dir, const int32_t* hit_pos, const float* hit_t,
                           long ray_count, u64 seed, float* orig_out, float* dir_out, float* depth_out) {
  const F4* tr = (const F4*)tris; const F4* po = (const F4*)orig; const F4* pd = (const F4*)dir;
  F4* oo = (F4*)orig_out; F4* od = (F4*)dir_out;
#pragma omp parallel for schedule(static)
  for (long r = 0; r < ray_count; ++r) {
    int32_t pos = hit_pos[r];
    if (pos < 0) { oo[r] = F4{0, 0, 0, 0}; od[r] = F4{0, 0, 0, 0}; depth_out[r] = -1.0f; continue; }
    F4 o = po[r], d = pd[r]; float t = hit_t[r];
    F4 e1 = tr[3 * (long)pos + 1], e2 = tr[3 * (long)pos + 2];
    float nx = e1.y * e2.z - e1.z * e2.y, ny = e1.z * e2.x - e1.x * e2.z, nz = e1.x * e2.y - e1.y * e2.x;
    float inv = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
    nx = nx * inv; ny = ny * inv; nz = nz * inv;
    if (nx * d.x + ny * d.y + nz * d.z > 0.0f) { nx = -nx; ny = -ny; nz = -nz; }
    float px = o.x + t * d.x, py = o.y + t * d.y, pz = o.z + t * d.z;
    const float eps = 1e-4f;
    Pcg g; pcg_seed(g, seed, (u64)r);
    float a = 0.0f, b = 0.0f;
    for (int it = 0; it < 64; ++it) {
      float u1 = (float)(pcg_next(g) >> 8) * 5.9604644775390625e-8f;
      float u2 = (float)(pcg_next(g) >> 8) * 5.9604644775390625e-8f;
      float aa = 2.0f * u1 - 1.0f, bb = 2.0f * u2 - 1.0f;
      if (aa * aa + bb * bb < 1.0f) { a = aa; b = bb; break; }
    }
    float c = sqrtf(1.0f - (a * a + b * b));
    float sgn = copysignf(1.0f, nz);
    float A = -1.0f / (sgn + nz);
    float B = nx * ny * A;
    float t1x = 1.0f + sgn * nx * nx * A, t1y = sgn * B, t1z = -sgn * nx;
    float t2x = B, t2y = sgn + ny * ny * A, t2z = -ny;
    oo[r] = F4{px + nx * eps, py + ny * eps, pz + nz * eps, 0.0f};
    od[r] = F4{t1x * a + t2x * b + nx * c, t1y * a + t2y * b + ny * c, t1z * a + t2z * b + nz * c, 0.0f};
    depth_out[r] = kHuge;
  }
}

// ---------------------------------------------------------------------------
// Attribute interpolation, kernels/CUDA_interpolateData.cu:45-138: weights
// (1 - u - v, u, v), sums left to right, normalize with 1/sqrtf (the reference's
// device rsqrtf is an approximate instruction). A miss (id < 0) gives zeros.
// outputs: points/normals/colors float4, texcoords float2, materials u32; NULL = skip.
// ---------------------------------------------------------------------------
OR_API void or_interpolate(const int32_t* hit_id, const float* hit_uv, long count, const u32* faces, const float* vertices,
                           const float* normals, const float* colors, const float* texcoords,
                           float* out_points, float* out_normals, float* out_colors, float* out_texcoords, u32* out_materials) {
  const U4* f = (const U4*)faces; const F4* v = (const F4*)vertices;
  const F4* nrm = (const F4*)normals; const F4* col = (const F4*)colors;
#pragma omp parallel for schedule(static)
  for (long l = 0; l < count; ++l) {
    int32_t id = hit_id[l];
    if (id < 0) {
      F4 z = {0, 0, 0, 0};
      if (out_points) ((F4*)out_points)[l] = z;
      if (out_normals) ((F4*)out_normals)[l] = z;
      if (out_colors) ((F4*)out_colors)[l] = z;
      if (out_texcoords) { out_texcoords[2 * l] = 0; out_texcoords[2 * l + 1] = 0; }
      if (out_materials) out_materials[l] = 0;
      continue;
    }
    float u = hit_uv[2 * l], w = hit_uv[2 * l + 1];
    U4 face = f[id];
    F4 v0 = v[face.x], v1 = v[face.y], v2 = v[face.z];
    float w0 = 1 - u - w;
    auto lerp = [&](F4 a, F4 b, F4 c) { return f4add(f4add(f4scale(a, w0), f4scale(b, u)), f4scale(c, w)); };
    if (out_points) ((F4*)out_points)[l] = lerp(v0, v1, v2);
    if (out_normals) {
      F4 n = nrm ? normalize4(lerp(nrm[face.x], nrm[face.y], nrm[face.z])) : normalize4(cross4(f4sub(v1, v0), f4sub(v2, v0)));
      ((F4*)out_normals)[l] = n;
    }
    if (out_colors) ((F4*)out_colors)[l] = col ? lerp(col[face.x], col[face.y], col[face.z]) : F4{1.0f, 1.0f, 1.0f, 1.0f};
    if (out_texcoords) {
      if (texcoords) {
        const float* t0 = texcoords + 2 * (size_t)face.x; const float* t1 = texcoords + 2 * (size_t)face.y;
        const float* t2 = texcoords + 2 * (size_t)face.z;
        out_texcoords[2 * l] = t0[0] * w0 + t1[0] * u + t2[0] * w;
        out_texcoords[2 * l + 1] = t0[1] * w0 + t1[1] * u + t2[1] * w;
      } else { out_texcoords[2 * l] = u; out_texcoords[2 * l + 1] = w; }
    }
    if (out_materials) out_materials[l] = face.w;
  }
}

OR_API int or_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Thread count of every parallel oracle loop that takes no explicit count (the
// CPU baseline times the build with one thread and with all of them).
OR_API void or_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
  (void)n;
#endif
}
