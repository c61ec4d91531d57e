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
#include "rt_device.cuh"
#include "../../include/rt_propose.h"

namespace rt {
namespace {

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
  // optional: the packet walks also write each ray's diffuse bounce (bounce_ray / bounce_miss) here
  float4* b_orig;
  float4* b_dir;
  float* b_tmax;
  uint64_t b_seed;
};

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
  const float4* wide;  // 4-wide records
  uint32_t stage = 0;        // shared-memory address of the staged top treelet (0: none; see stage_treelet)
  uint32_t stage_depth = 0;  // levels of 4-wide records a persistent kernel stages (0: none)
  // Batched walks: the ray's mesh's first face position F and first group G. Its records, leaves, groups and
  // triangles are addressed from the batch's base pointers plus these offsets (two 32-bit registers per lane
  // instead of a 64-bit pointer per array); a single mesh has F = G = 0.
  uint32_t F = 0;
  uint32_t G = 0;
};

// Top treelet in shared memory: the 4-wide records of the first `depth` levels below the root (breadth first, at
// most 1 + 4 + 16 + 64 = 85 records, 10.9 KB), copied once per CTA of a persistent kernel. Inside the copy, the
// reference to a child record that is staged as well becomes kStagedBit | slot, so a walk that starts at the
// staged root reads those levels from shared memory and leaves them by an ordinary (global) reference.
// Record indices are below 2^30 and the walk only looks for the bit on internal references.
constexpr uint32_t kStagedBit = 0x40000000u;
constexpr uint32_t kMaxStageDepth = 4;
constexpr uint32_t kMaxStaged = 85;
__host__ __device__ constexpr uint32_t staged_slots(uint32_t depth) {
  return depth == 0 ? 0u : (depth == 1 ? 1u : (depth == 2 ? 5u : (depth == 3 ? 21u : 85u)));
}

__device__ uint32_t stage_treelet(const AccelArgs& C, float4* s_tree, uint32_t* s_rec, uint32_t depth) {
  __shared__ uint32_t s_count;
  if (threadIdx.x == 0) {
    uint32_t n = 0;
    if (__ldg(C.hdr) == 0u) {  // the root is record 0 (a leaf root has nothing to stage)
      s_rec[n++] = 0;
      uint32_t lo = 0;
      for (uint32_t l = 1; l < depth; ++l) {
        const uint32_t hi = n;
        for (uint32_t q = lo; q < hi; ++q) {
          const uint4 refs = __ldg((const uint4*)(C.wide + 8 * (size_t)s_rec[q] + 6));
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const uint32_t rk = u4c(refs, k);
            if (rk != kNoChild && !(rk & 0x80000000u) && n < kMaxStaged) s_rec[n++] = rk;
          }
        }
        lo = hi;
      }
    }
    s_count = n;
  }
  __syncthreads();
  const uint32_t n = s_count;
  for (uint32_t i = threadIdx.x; i < n * 8; i += blockDim.x) {
    const uint32_t q = i >> 3, j = i & 7u;
    float4 v = __ldg(C.wide + 8 * (size_t)s_rec[q] + j);
    if (j == 6) {  // child references: staged children become slot references
      uint32_t rv[4] = {__float_as_uint(v.x), __float_as_uint(v.y), __float_as_uint(v.z), __float_as_uint(v.w)};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (rv[k] == kNoChild || (rv[k] & 0x80000000u)) continue;
        for (uint32_t t = 1; t < n; ++t)
          if (s_rec[t] == rv[k]) { rv[k] = kStagedBit | t; break; }
      }
      v = make_float4(__uint_as_float(rv[0]), __uint_as_float(rv[1]), __uint_as_float(rv[2]), __uint_as_float(rv[3]));
    }
    s_tree[i] = v;
  }
  __syncthreads();
  return n ? (uint32_t)__cvta_generic_to_shared(s_tree) : 0u;
}

// The 128-byte record at shared-memory address a, as wide_test reads a global one.
__device__ __forceinline__ void wide_test_staged(uint32_t a, const float4& oi, float ix, float iy, float iz, float tbest, uint32_t skip,
                                                 float (&t)[4], uint32_t (&r)[4]) {
  float4 w[8];
#pragma unroll
  for (int j = 0; j < 8; ++j)
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(w[j].x), "=f"(w[j].y), "=f"(w[j].z), "=f"(w[j].w) : "r"(a + 16u * j));
  wide_test_regs(w, oi, ix, iy, iz, tbest, skip, t, r);
}

// A 4-wide record's test from global memory (staged == false) or from the staged treelet.
__device__ __forceinline__ void wide_record_test(const AccelArgs& C, uint32_t ref, const float4& oi, float ix, float iy, float iz,
                                                 float tbest, uint32_t skip, float (&t)[4], uint32_t (&r)[4]) {
  if (ref & kStagedBit) wide_test_staged(C.stage + 128u * (ref & ~kStagedBit), oi, ix, iy, iz, tbest, skip, t, r);
  else wide_test(C.wide + 8 * ((size_t)C.F + ref), oi, ix, iy, iz, tbest, skip, t, r);
}

// One ray through the blob. kWW: "while-while" schedule (descend internal
// nodes until the ray holds a leaf, then test the leaf), which keeps the lanes
// of a warp in the same phase more often than the "if-if" schedule.
// Proposal seeding (rt_trace_closest_seeded): the ray first walks the subtree
// `slot_ref[proposal[r]]` (phase 0), then the whole tree with that subtree cut
// out (phase 1), keeping the best hit of phase 0 as its starting best. Phase 0
// finds the exact minimum (t, position) of the subtree, so skipping it in
// phase 1 loses nothing and the final hit is the same as a plain walk's.
struct SeedArgs {
  const int32_t* proposal;
  const int32_t* slot_ref;
  const float4* slot_box;
  uint32_t slot_count;
  int32_t* in_prop;
};
constexpr uint32_t kNoSkip = 0x7FFFFFFFu;  // never a record index or a leaf reference

// A slot reference is walked only when it names a record or leaf of this blob
// (hdr[1] = leaf count; a tree of L leaves has L - 1 two-child records).
__device__ __forceinline__ bool seed_ref_ok(uint32_t q, const AccelArgs& C) {
  const uint32_t leaves = __ldg(C.hdr + 1);
  return (q & 0x80000000u) ? (~q < leaves) : (q + 1u < leaves);
}

// Where a seeded walk starts. With a valid proposal: the proposed subtree
// (phase 0) and that subtree cut out of phase 1. When the ray misses the slot's
// padded box (the same conservative test as every node box), nothing in the
// subtree can be hit, so phase 0 is skipped and the subtree is still cut out.
// Returns false when nothing is left to walk.
template <bool kCount>
__device__ __forceinline__ bool seed_start(uint32_t r, const SeedArgs& S, const AccelArgs& C, const float4& oi, float ix, float iy,
                                           float iz, float bt, uint32_t root, uint32_t& ref, uint32_t& skip, uint32_t& phase,
                                           uint32_t& visits) {
  const int32_t p = __ldg(S.proposal + r);
  if (p < 0 || (uint32_t)p >= S.slot_count) return true;
  const uint32_t q = (uint32_t)__ldg(S.slot_ref + p);
  if (!seed_ref_ok(q, C)) return true;
  skip = q;
  if (S.slot_box) {
    if (kCount) ++visits;
    float tb;
    if (!slab2(ldg4(S.slot_box + 2 * p), ldg4(S.slot_box + 2 * p + 1), oi, ix, iy, iz, bt, tb)) return root != skip;
  }
  ref = q;
  phase = 0;
  return true;
}

template <bool kCount, bool kWW, bool kSeed = false, bool kWide = false>
__device__ __forceinline__ void trace_ray_accel(const uint32_t r, const TraceArgs& A, const AccelArgs& C,
                                                const SeedArgs& S = SeedArgs{}) {
  const float tmax0 = A.tmax ? __ldg(A.tmax + r) : kHuge;
  int32_t best = -1;
  float bt = tmax0, bu = 0.0f, bv = 0.0f;
  uint32_t visits = 0, tests = 0;
  uint32_t phase = 1, best_phase = 1;
  if (tmax0 > 0.0f) {  // an inactive ray (tmax <= 0) reads nothing more
    const float4 o = ldg4(A.orig + r), d = ldg4(A.dir + r);
    const float ix = 1.0f / fix_dir(d.x), iy = 1.0f / fix_dir(d.y), iz = 1.0f / fix_dir(d.z);
    const float4 oi = scaled_origin(o, ix, iy, iz);
    const float zu = o.w * 0.0f, zv = d.w * 0.0f;
    uint32_t st_ref[kStack];
    float st_t[kStack];
    int sp = 0;
    const uint32_t root = C.stage ? kStagedBit : __ldg(C.hdr);
    uint32_t ref = root, skip = kNoSkip;
    bool alive = true;
    if (kSeed) alive = seed_start<kCount>(r, S, C, oi, ix, iy, iz, bt, root, ref, skip, phase, visits);
    // next reference to walk: the nearest stacked subtree still within reach,
    // else (phase 0) the root of phase 1; false when the walk is over
    auto next = [&]() -> bool {
      while (sp > 0) {
        --sp;
        if (st_t[sp] <= bt * kCullSlack) { ref = st_ref[sp]; return true; }
      }
      if (kSeed && phase == 0) {
        phase = 1;
        ref = root;
        return root != skip;
      }
      return false;
    };
    while (alive) {
      // descend internal nodes (kWW: until this ray holds a leaf)
      while (!(ref & 0x80000000u)) {
        if constexpr (kWide) {
          // 4-wide record: up to four children tested at once, nearest first
          float wt[4];
          uint32_t wr[4];
          wide_record_test(C, ref, oi, ix, iy, iz, bt, (kSeed && phase) ? skip : kNoSkip, wt, wr);
          if (kCount) visits += 4;
          if (wt[0] == INFINITY) {
            if (!next()) {
              alive = false;
              break;
            }
          } else {
#pragma unroll
            for (int k = 3; k >= 1; --k) {
              if (wt[k] != INFINITY) {
                if (sp < kStack) {
                  st_ref[sp] = wr[k];
                  st_t[sp] = wt[k];
                  ++sp;
                } else if (A.err) {
                  atomicOr(A.err, (uint32_t)RT_DEVERR_STACK_OVERFLOW);
                }
              }
            }
            ref = wr[0];
          }
        } else {
        const float4* tn = C.tnodes + 4 * ((size_t)C.F + ref);
        float4 a0, a1, b0, b1;
        ldg8(tn, a0, a1);
        ldg8(tn + 2, b0, b1);
        if (kCount) visits += 2;
        float ta, tb;
        bool ha = slab2(a0, a1, oi, ix, iy, iz, bt, ta);
        bool hb = slab2(b0, b1, oi, ix, iy, iz, bt, tb);
        const uint32_t ra = __float_as_uint(a0.w), rb = __float_as_uint(b0.w);
        if (kSeed && phase) {
          if (ra == skip) ha = false;
          if (rb == skip) hb = false;
        }
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
        } else if (ha) {
          ref = ra;
        } else if (hb) {
          ref = rb;
        } else if (!next()) {
          alive = false;
          break;
        }
        }
        if (!kWW && (ref & 0x80000000u)) break;
      }
      if (!alive) break;
      // leaf: group boxes, then the triangles of the groups that pass
      const uint4 L = __ldg(C.leaves + (C.F + ~ref));
      if (kCount) ++visits;
      const uint32_t first = L.x, cnt = L.y, gbase = L.z;
      for (uint32_t g = 0; g * 8 < cnt; ++g) {
        float4 gmn, gmx;
        ldg8(C.groups + 2 * ((size_t)C.G + gbase + g), gmn, gmx);
        if (kCount) ++visits;
        float tg;
        if (!slab2(gmn, gmx, oi, ix, iy, iz, bt, tg)) continue;
        const uint32_t kend = min(cnt, g * 8 + 8);
        for (uint32_t k = g * 8; k < kend; ++k) {
          const uint32_t pos = first + k;
          const float4 v0 = ldg4(A.tris + 3 * ((size_t)C.F + pos));
          const float4 e1 = ldg4(A.tris + 3 * ((size_t)C.F + pos) + 1);
          const float4 e2 = ldg4(A.tris + 3 * ((size_t)C.F + pos) + 2);
          if (kCount) ++tests;
          float t, u, v;
          if (!mt_test(o, d, zu, zv, v0, e1, e2, t, u, v)) continue;
          if (t < bt || (best >= 0 && t == bt && (int32_t)pos < best)) {
            best = (int32_t)pos; bt = t; bu = u; bv = v;
            best_phase = phase;
          }
        }
      }
      // next subtree whose entry is still within reach
      if (!next()) break;
    }
  }
  if (best >= 0) {
    A.hit_id[r] = A.id_mode == 1 ? (int32_t)__ldg(A.indices + C.F + best) : best;
    A.hit_t[r] = bt;
    A.hit_uv[r] = make_float2(bu, bv);
  } else {
    A.hit_id[r] = -1;
    A.hit_t[r] = tmax0;
    A.hit_uv[r] = make_float2(0.0f, 0.0f);
  }
  if (kSeed && S.in_prop) S.in_prop[r] = (best >= 0 && best_phase == 0) ? 1 : 0;
  if (kCount) {
    if (A.visits) A.visits[r] = visits;
    if (A.tests) A.tests[r] = tests;
  }
}

// Warp-cooperative schedule. Each lane descends its own ray until it holds a
// leaf (while-while); then every lane tests its own leaf's group boxes, and the
// (ray, 8-triangle group) items of the whole warp are spread over the 32 lanes:
// a lane tests one group against the ray of the item's owner (fetched by
// shuffles) and merges its best hit into the owner's slot with a 64-bit
// shared-memory atomicMin on (t bits, position), which is the same
// (t, position) rule as the other schedules. The (u, v) of the current best
// are written by the lane whose key is the minimum right after its merge.
constexpr int kCoopWarps = 4;  // 128-thread CTAs

// The triangle tests of one warp-cooperative step. Each lane holds `mask`:
// bit g set = group g of its leaf is to be tested, i.e. positions
// first + kGroup g .. min(cnt, kGroup (g + 1)) - 1 + first of its mesh (whose
// positions start at F in the triangle stream). The (ray, group) items of the
// whole warp are spread over the 32 lanes: a lane tests one group against the
// ray of the item's owner (fetched by shuffles) and merges its best hit into
// the owner's slot with a 64-bit shared-memory atomicMin on (t bits, position),
// the same (t, position) rule as the other schedules. The (u, v) of the
// current best are written by the lane whose key is the minimum right after
// its merge. key0 is this lane's best so far (t bits, position); on return
// s_key[lane] / s_uv[lane] hold the merged best of this lane's ray.
template <uint32_t kGroup>
__device__ __forceinline__ void coop_items(const uint32_t lane, const uint32_t mask, const uint32_t first, const uint32_t cnt,
                                           const uint32_t F, const float4& o, const float4& d, const float zu, const float zv,
                                           const float4* __restrict__ tris, const unsigned long long key0, const float bu,
                                           const float bv, unsigned long long* s_key, float2* s_uv) {
  const uint32_t my_items = __popc(mask);
  uint32_t incl = my_items;
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, k);
    if (lane >= (uint32_t)k) incl += y;
  }
  const uint32_t excl = incl - my_items;
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  s_key[lane] = key0;
  s_uv[lane] = make_float2(bu, bv);
  __syncwarp();
  for (uint32_t base = 0; base < total; base += 32) {
    const uint32_t item = base + lane;
    unsigned long long cand = ~0ull;
    float cu = 0.f, cv = 0.f;
    // owner: last lane whose exclusive offset is <= item
    uint32_t lo = 0, hi = 31;
#pragma unroll
    for (int it = 0; it < 5; ++it) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      const uint32_t off_mid = __shfl_sync(0xffffffffu, excl, mid);
      if (off_mid <= item) lo = mid; else hi = mid - 1;
    }
    const uint32_t owner = lo;
    const float4 oo = make_float4(__shfl_sync(0xffffffffu, o.x, owner), __shfl_sync(0xffffffffu, o.y, owner),
                                  __shfl_sync(0xffffffffu, o.z, owner), 0.0f);
    const float4 od = make_float4(__shfl_sync(0xffffffffu, d.x, owner), __shfl_sync(0xffffffffu, d.y, owner),
                                  __shfl_sync(0xffffffffu, d.z, owner), 0.0f);
    const float ozu = __shfl_sync(0xffffffffu, zu, owner), ozv = __shfl_sync(0xffffffffu, zv, owner);
    const uint32_t omask = __shfl_sync(0xffffffffu, mask, owner);
    const uint32_t oexcl = __shfl_sync(0xffffffffu, excl, owner);
    const uint32_t ofirst = __shfl_sync(0xffffffffu, first, owner);
    const uint32_t ocnt = __shfl_sync(0xffffffffu, cnt, owner);
    // the owner's triangle stream (lanes of a batched launch may trace different meshes)
    const float4* otris = tris + 3 * (size_t)__shfl_sync(0xffffffffu, F, owner);
    if (item < total) {
      const uint32_t g = __fns(omask, 0, (int)(item - oexcl) + 1);
      const uint32_t kend = min(ocnt, g * kGroup + kGroup);
      const unsigned long long cur = s_key[owner];
      unsigned long long mine = ~0ull;
      float mu = 0.f, mv = 0.f;
      for (uint32_t k = g * kGroup; k < kend; ++k) {
        const uint32_t pos = ofirst + k;
        const float4 v0 = ldg4(otris + 3 * (size_t)pos);
        const float4 e1 = ldg4(otris + 3 * (size_t)pos + 1);
        const float4 e2 = ldg4(otris + 3 * (size_t)pos + 2);
        float t, u, v;
        if (!mt_test(oo, od, ozu, ozv, v0, e1, e2, t, u, v)) continue;
        const unsigned long long key = ((unsigned long long)__float_as_uint(t) << 32) | pos;
        if (key < mine) { mine = key; mu = u; mv = v; }
      }
      if (mine < cur) atomicMin(s_key + owner, mine);
      cand = mine;
      cu = mu; cv = mv;
    }
    __syncwarp();
    // (u, v) of the owner's minimum, written by the one lane holding that key
    if (item < total && cand != ~0ull && s_key[owner] == cand) s_uv[owner] = make_float2(cu, cv);
    __syncwarp();
  }
}

template <bool kCount, bool kSeed = false, bool kWide = false>
__device__ __forceinline__ void trace_warp_coop(const uint32_t r, const bool valid, const TraceArgs& A, const AccelArgs& C,
                                                unsigned long long* s_key, float2* s_uv, const SeedArgs& S = SeedArgs{}) {
  const uint32_t lane = lane_id();
  float4 o = make_float4(0.f, 0.f, 0.f, 0.f), d = make_float4(0.f, 0.f, 1.f, 0.f);
  float tmax0 = -1.0f;
  if (valid) {
    tmax0 = A.tmax ? __ldg(A.tmax + r) : kHuge;
    if (tmax0 > 0.0f) {  // an inactive ray (tmax <= 0) reads nothing more
      o = ldg4(A.orig + r);
      d = ldg4(A.dir + r);
    }
  }
  int32_t best = -1;
  float bt = tmax0, bu = 0.0f, bv = 0.0f;
  uint32_t visits = 0, tests = 0;
  const float ix = 1.0f / fix_dir(d.x), iy = 1.0f / fix_dir(d.y), iz = 1.0f / fix_dir(d.z);
  const float4 oi = scaled_origin(o, ix, iy, iz);
  const float zu = o.w * 0.0f, zv = d.w * 0.0f;
  uint32_t st_ref[kStack];
  float st_t[kStack];
  int sp = 0;
  const uint32_t root = C.stage ? kStagedBit : __ldg(C.hdr);
  uint32_t ref = root, skip = kNoSkip;
  uint32_t phase = 1, best_phase = 1;
  bool go = true;
  if (kSeed && valid && tmax0 > 0.0f) go = seed_start<kCount>(r, S, C, oi, ix, iy, iz, bt, root, ref, skip, phase, visits);
  auto next = [&]() -> bool {
    while (sp > 0) {
      --sp;
      if (st_t[sp] <= bt * kCullSlack) { ref = st_ref[sp]; return true; }
    }
    if (kSeed && phase == 0) {
      phase = 1;
      ref = root;
      return root != skip;
    }
    return false;
  };
  bool alive = valid && tmax0 > 0.0f && go;
  while (__any_sync(0xffffffffu, alive)) {
    // 1. descend until this ray holds a leaf
    bool has_leaf = false;
    if (alive) {
      while (!(ref & 0x80000000u)) {
        if constexpr (kWide) {
          // 4-wide record: up to four children tested at once, nearest first
          float wt[4];
          uint32_t wr[4];
          wide_record_test(C, ref, oi, ix, iy, iz, bt, (kSeed && phase) ? skip : kNoSkip, wt, wr);
          if (kCount) visits += 4;
          if (wt[0] == INFINITY) {
            if (!next()) {
              alive = false;
              break;
            }
          } else {
#pragma unroll
            for (int k = 3; k >= 1; --k) {
              if (wt[k] != INFINITY) {
                if (sp < kStack) {
                  st_ref[sp] = wr[k];
                  st_t[sp] = wt[k];
                  ++sp;
                } else if (A.err) {
                  atomicOr(A.err, (uint32_t)RT_DEVERR_STACK_OVERFLOW);
                }
              }
            }
            ref = wr[0];
          }
        } else {
        const float4* tn = C.tnodes + 4 * ((size_t)C.F + ref);
        float4 a0, a1, b0, b1;
        ldg8(tn, a0, a1);
        ldg8(tn + 2, b0, b1);
        if (kCount) visits += 2;
        float ta, tb;
        bool ha = slab2(a0, a1, oi, ix, iy, iz, bt, ta);
        bool hb = slab2(b0, b1, oi, ix, iy, iz, bt, tb);
        const uint32_t ra = __float_as_uint(a0.w), rb = __float_as_uint(b0.w);
        if (kSeed && phase) {
          if (ra == skip) ha = false;
          if (rb == skip) hb = false;
        }
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
        } else if (ha) {
          ref = ra;
        } else if (hb) {
          ref = rb;
        } else if (!next()) {
          alive = false;
          break;
        }
        }
      }
      has_leaf = alive;
    }
    // 2. own leaf: group boxes -> mask of groups to test
    uint32_t mask = 0, first = 0, cnt = 0;
    if (has_leaf) {
      const uint4 L = __ldg(C.leaves + (C.F + ~ref));
      if (kCount) ++visits;
      first = L.x; cnt = L.y;
      const uint32_t gbase = L.z;
      const uint32_t ng = (cnt + 7) >> 3;
      for (uint32_t g = 0; g < ng; ++g) {
        float4 gmn, gmx;
        ldg8(C.groups + 2 * ((size_t)C.G + gbase + g), gmn, gmx);
        if (kCount) ++visits;
        float tg;
        if (slab2(gmn, gmx, oi, ix, iy, iz, bt, tg)) {
          if (g < 32) mask |= 1u << g;
        }
      }
      // the triangles of these groups are tested below, by whichever lanes: count them for this ray
      if (kCount)
        for (uint32_t mm = mask; mm; mm &= mm - 1u) {
          const uint32_t g = __ffs(mm) - 1u;
          tests += min(cnt, g * 8u + 8u) - g * 8u;
        }
      // leaves of more than 256 triangles (tree_complete = 0) keep the groups
      // past 32 to this lane: they are tested below by the owner alone
    }
    // 3. spread the warp's (ray, group) items over the lanes
    // (t bits, position) of the best hit so far; with no hit yet, (tmax bits, 0),
    // which no accepted hit equals (t < tmax is required)
    const unsigned long long key0 = ((unsigned long long)__float_as_uint(bt) << 32) | (uint32_t)(best >= 0 ? best : 0);
    coop_items<8>(lane, mask, first, cnt, C.F, o, d, zu, zv, A.tris, key0, bu, bv, s_key, s_uv);
    // 4. read back the merged best and move on
    if (has_leaf) {
      const unsigned long long k = s_key[lane];
      if (k < key0) {
        bt = __uint_as_float((uint32_t)(k >> 32));
        best = (int32_t)(k & 0xFFFFFFFFu);
        const float2 uv = s_uv[lane];
        bu = uv.x; bv = uv.y;
        best_phase = phase;
      }
      // groups beyond the first 32 (leaves of more than 256 triangles): this lane alone
      for (uint32_t g = 32; g * 8 < cnt; ++g) {
        const uint32_t gbase = __ldg(C.leaves + (C.F + ~ref)).z;
        float4 gmn, gmx;
        ldg8(C.groups + 2 * ((size_t)C.G + gbase + g), gmn, gmx);
        float tg;
        if (!slab2(gmn, gmx, oi, ix, iy, iz, bt, tg)) continue;
        const uint32_t kend = min(cnt, g * 8 + 8);
        for (uint32_t kk = g * 8; kk < kend; ++kk) {
          const uint32_t pos = first + kk;
          const float4 v0 = ldg4(A.tris + 3 * ((size_t)C.F + pos));
          const float4 e1 = ldg4(A.tris + 3 * ((size_t)C.F + pos) + 1);
          const float4 e2 = ldg4(A.tris + 3 * ((size_t)C.F + pos) + 2);
          if (kCount) ++tests;
          float t, u, v;
          if (!mt_test(o, d, zu, zv, v0, e1, e2, t, u, v)) continue;
          if (t < bt || (best >= 0 && t == bt && (int32_t)pos < best)) {
            best = (int32_t)pos; bt = t; bu = u; bv = v;
            best_phase = phase;
          }
        }
      }
      if (!next()) alive = false;
    }
    __syncwarp();
  }
  if (!valid) return;
  if (kSeed && S.in_prop) S.in_prop[r] = (best >= 0 && best_phase == 0) ? 1 : 0;
  if (best >= 0) {
    A.hit_id[r] = A.id_mode == 1 ? (int32_t)__ldg(A.indices + C.F + best) : best;
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

// ---------------------------------------------------------------------------
// Cluster tree walks (RT_TRACE_CLUSTERS; layout in rt_device.cuh)
// ---------------------------------------------------------------------------
struct ClusterArgs {
  const float4* crec;   // cluster records (a batched launch: the batch's, from its base)
  const uint32_t* hdr;  // header words of the ray's mesh
  uint32_t F = 0;       // the mesh's first position (and first record)
  uint32_t n = 0;       // the mesh's face count, as the caller gives it
};

__device__ __forceinline__ void write_hit(const uint32_t r, const TraceArgs& A, const uint32_t F, const int32_t best, const float bt,
                                          const float bu, const float bv, const float tmax0) {
  if (best >= 0) {
    A.hit_id[r] = A.id_mode == 1 ? (int32_t)__ldg(A.indices + F + best) : best;
    A.hit_t[r] = bt;
    A.hit_uv[r] = make_float2(bu, bv);
  } else {
    A.hit_id[r] = -1;
    A.hit_t[r] = tmax0;
    A.hit_uv[r] = make_float2(0.0f, 0.0f);
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

// One diffuse bounce of ray r, which hit the triangle at (global) position pos at distance t: the origin is the hit
// point moved 1e-4 along the triangle's normal turned against the ray, the direction a cosine-weighted sample of
// the hemisphere around that normal (a point of the unit disc by rejection from the PCG stream r of `seed`, lifted
// to the hemisphere, in the orthonormal basis of Duff et al. 2017), tmax huge. Out of line: inlined into the packet
// walk's epilogue it took that kernel to 72 registers (7 CTAs per SM instead of 8).
__device__ __noinline__ void bounce_ray(const float4* __restrict__ tris, uint32_t pos, const float4& o, const float4& d, float t,
                                           uint64_t seed, uint32_t r, float4* __restrict__ orig_out, float4* __restrict__ dir_out,
                                           float* __restrict__ tmax_out) {
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
// A ray that hit nothing has no bounce: zero origin and direction, tmax -1 (an inactive ray).
__device__ __forceinline__ void bounce_miss(uint32_t r, float4* __restrict__ orig_out, float4* __restrict__ dir_out,
                                            float* __restrict__ tmax_out) {
  orig_out[r] = make_float4(0.f, 0.f, 0.f, 0.f);
  dir_out[r] = make_float4(0.f, 0.f, 0.f, 0.f);
  tmax_out[r] = -1.0f;
}

// The header of the ray's mesh describes a cluster tree built for the mesh's face count; root = its record.
__device__ __forceinline__ bool cluster_tree_ok(const ClusterArgs& C, uint32_t& root) {
  root = __ldg(C.hdr + kHdrClusterRoot);
  return __ldg(C.hdr + kHdrClusterValid) == 1u && __ldg(C.hdr + kHdrClusterN) == C.n && C.n > 0 && root < C.n;
}
// A reference inside the mesh (a record index below n, or a cluster whose positions are below n), reached
// within the walk's step bound: a walk of a well-formed tree enters every record and every cluster at most once,
// 2n steps in all. Anything else (a blob written for other sizes, or damaged) ends the walk with
// RT_DEVERR_ACCEL_MISSING instead of reading past the mesh or looping.
__device__ __forceinline__ bool cluster_ref_ok(uint32_t ref, uint32_t n, uint32_t& steps) {
  return ++steps <= 2 * n + 2 && ((ref & kClusterLeaf) ? (ref & kClusterFirstMask) + ((ref >> 28) & 7u) < n : ref < n);
}

// Pops the nearest stacked reference that can still hold a closer hit.
__device__ __forceinline__ bool pop_within(const uint32_t (&st_ref)[kStack], const float (&st_t)[kStack], int& sp, float bt,
                                           uint32_t& ref) {
  while (sp > 0) {
    --sp;
    if (st_t[sp] <= bt * kCullSlack) {
      ref = st_ref[sp];
      return true;
    }
  }
  return false;
}

// One ray, one lane: nearest-first descent through the 4-wide records; a
// cluster is tested when the walk reaches it (entered nearest first, skipped
// once it can no longer hold a closer hit). kWW (while-while): each step first
// descends until the lane holds a cluster, then tests it, so the lanes of a
// warp test triangles together instead of interleaving box and triangle steps.
// kBounce: also write the ray's bounce when A asks for it (the packet kernels' fallback for warps whose rays span
// meshes).
template <bool kCount, bool kWW, bool kBounce = false>
__device__ __forceinline__ void trace_ray_clusters(const uint32_t r, const TraceArgs& A, const ClusterArgs& C) {
  const float tmax0 = A.tmax ? __ldg(A.tmax + r) : kHuge;
  int32_t best = -1;
  float bt = tmax0, bu = 0.0f, bv = 0.0f;
  uint32_t visits = 0, tests = 0;
  uint32_t ref = 0;
  if (tmax0 > 0.0f && !cluster_tree_ok(C, ref)) {
    if (A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
  } else if (tmax0 > 0.0f) {
    const float4 o = ldg4(A.orig + r), d = ldg4(A.dir + r);
    const float ix = 1.0f / fix_dir(d.x), iy = 1.0f / fix_dir(d.y), iz = 1.0f / fix_dir(d.z);
    const float4 oi = scaled_origin(o, ix, iy, iz);
    const float zu = o.w * 0.0f, zv = d.w * 0.0f;
    const float4* tris = A.tris + 3 * (size_t)C.F;
    const float4* recs = C.crec + 8 * (size_t)C.F;
    uint32_t st_ref[kStack];
    float st_t[kStack];
    int sp = 0;
    uint32_t steps = 0;
    // one record step: false when the walk is over (nothing hit and nothing stacked within reach)
    auto record_step = [&]() -> bool {
      float t[4];
      uint32_t k[4];
      cluster_test(recs + 8 * (size_t)ref, oi, ix, iy, iz, bt, t, k);
      if (kCount) visits += 4;
      if (t[0] != INFINITY) {
#pragma unroll
        for (int j = 3; j >= 1; --j) {
          if (t[j] != INFINITY) {
            if (sp < kStack) {
              st_ref[sp] = k[j];
              st_t[sp] = t[j];
              ++sp;
            } else if (A.err) {
              atomicOr(A.err, (uint32_t)RT_DEVERR_STACK_OVERFLOW);
            }
          }
        }
        ref = k[0];
        return true;
      }
      return pop_within(st_ref, st_t, sp, bt, ref);
    };
    auto cluster_step = [&]() {
      const uint32_t p0 = ref & kClusterFirstMask, p1 = p0 + ((ref >> 28) & 7u) + 1u;
      for (uint32_t pos = p0; pos < p1; ++pos) {
        const float4 v0 = ldg4(tris + 3 * (size_t)pos);
        const float4 e1 = ldg4(tris + 3 * (size_t)pos + 1);
        const float4 e2 = ldg4(tris + 3 * (size_t)pos + 2);
        if (kCount) ++tests;
        float th, u, v;
        if (!mt_test(o, d, zu, zv, v0, e1, e2, th, u, v)) continue;
        if (th < bt || (best >= 0 && th == bt && (int32_t)pos < best)) {
          best = (int32_t)pos; bt = th; bu = u; bv = v;
        }
      }
    };
    bool alive = true;
    while (alive) {
      if (!cluster_ref_ok(ref, C.n, steps)) {
        if (A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
        break;
      }
      if constexpr (kWW) {
        while (!(ref & kClusterLeaf)) {
          if (!record_step()) { alive = false; break; }
          if (!cluster_ref_ok(ref, C.n, steps)) {
            if (A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
            alive = false;
            break;
          }
        }
        if (!alive) break;
        cluster_step();
        alive = pop_within(st_ref, st_t, sp, bt, ref);
      } else {
        if (!(ref & kClusterLeaf)) {
          alive = record_step();
        } else {
          cluster_step();
          alive = pop_within(st_ref, st_t, sp, bt, ref);
        }
      }
    }
  }
  write_hit(r, A, C.F, best, bt, bu, bv, tmax0);
  if (kCount) {
    if (A.visits) A.visits[r] = visits;
    if (A.tests) A.tests[r] = tests;
  }
  if (kBounce && A.b_orig) {  // a packet warp's rays span meshes: the bounce as the packet walk would write it
    if (best >= 0) bounce_ray(A.tris, C.F + (uint32_t)best, ldg4(A.orig + r), ldg4(A.dir + r), bt, A.b_seed, r, A.b_orig, A.b_dir, A.b_tmax);
    else bounce_miss(r, A.b_orig, A.b_dir, A.b_tmax);
  }
}

// Warp-cooperative cluster walk: each lane descends its own ray until it holds
// a cluster; then the clusters of all lanes (one item of up to 8 triangles per
// lane) are tested by the whole warp (coop_items), and every lane moves on.
template <bool kCount>
__device__ __forceinline__ void trace_warp_coop_clusters(const uint32_t r, const bool valid, const TraceArgs& A, const ClusterArgs& C,
                                                         unsigned long long* s_key, float2* s_uv) {
  const uint32_t lane = lane_id();
  float4 o = make_float4(0.f, 0.f, 0.f, 0.f), d = make_float4(0.f, 0.f, 1.f, 0.f);
  float tmax0 = -1.0f;
  uint32_t ref = 0;
  bool ok = false;
  if (valid) {
    tmax0 = A.tmax ? __ldg(A.tmax + r) : kHuge;
    if (tmax0 > 0.0f) {  // an inactive ray (tmax <= 0) reads nothing more
      ok = cluster_tree_ok(C, ref);
      if (!ok && A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
      o = ldg4(A.orig + r);
      d = ldg4(A.dir + r);
    }
  }
  int32_t best = -1;
  float bt = tmax0, bu = 0.0f, bv = 0.0f;
  uint32_t visits = 0, tests = 0;
  const float ix = 1.0f / fix_dir(d.x), iy = 1.0f / fix_dir(d.y), iz = 1.0f / fix_dir(d.z);
  const float4 oi = scaled_origin(o, ix, iy, iz);
  const float zu = o.w * 0.0f, zv = d.w * 0.0f;
  const float4* recs = C.crec + 8 * (size_t)C.F;
  uint32_t st_ref[kStack];
  float st_t[kStack];
  int sp = 0;
  uint32_t steps = 0;
  bool alive = ok;
  while (__any_sync(0xffffffffu, alive)) {
    // 1. descend until this ray holds a cluster
    uint32_t mask = 0, first = 0, cnt = 0;
    while (alive) {
      if (!cluster_ref_ok(ref, C.n, steps)) {
        if (A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
        alive = false;
        break;
      }
      if (ref & kClusterLeaf) {
        mask = 1u;
        first = ref & kClusterFirstMask;
        cnt = ((ref >> 28) & 7u) + 1u;
        break;
      }
      float t[4];
      uint32_t k[4];
      cluster_test(recs + 8 * (size_t)ref, oi, ix, iy, iz, bt, t, k);
      if (kCount) visits += 4;
      if (t[0] != INFINITY) {
#pragma unroll
        for (int j = 3; j >= 1; --j) {
          if (t[j] != INFINITY) {
            if (sp < kStack) {
              st_ref[sp] = k[j];
              st_t[sp] = t[j];
              ++sp;
            } else if (A.err) {
              atomicOr(A.err, (uint32_t)RT_DEVERR_STACK_OVERFLOW);
            }
          }
        }
        ref = k[0];
        continue;
      }
      if (!pop_within(st_ref, st_t, sp, bt, ref)) alive = false;
    }
    if (kCount) tests += cnt;
    // 2. the warp's clusters, spread over the lanes
    const unsigned long long key0 = ((unsigned long long)__float_as_uint(bt) << 32) | (uint32_t)(best >= 0 ? best : 0);
    coop_items<kClusterLeafMax>(lane, mask, first, cnt, C.F, o, d, zu, zv, A.tris, key0, bu, bv, s_key, s_uv);
    // 3. read back the merged best and move on
    if (mask) {
      const unsigned long long key = s_key[lane];
      if (key < key0) {
        bt = __uint_as_float((uint32_t)(key >> 32));
        best = (int32_t)(key & 0xFFFFFFFFu);
        const float2 uv = s_uv[lane];
        bu = uv.x; bv = uv.y;
      }
      if (!pop_within(st_ref, st_t, sp, bt, ref)) alive = false;
    }
    __syncwarp();
  }
  if (!valid) return;
  write_hit(r, A, C.F, best, bt, bu, bv, tmax0);
  if (kCount) {
    if (A.visits) A.visits[r] = visits;
    if (A.tests) A.tests[r] = tests;
  }
}

// A float as an unsigned key of the same order (for warp minimum reductions).
__device__ __forceinline__ uint32_t order_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
// Compare-exchange of packet slots on a warp-uniform key, the lane's own entry distance and the reference riding along.
__device__ __forceinline__ void cswap_packet(uint32_t (&key)[4], float (&t)[4], uint32_t (&r)[4], int a, int b) {
  if (key[b] < key[a]) {
    const uint32_t kk = key[a]; key[a] = key[b]; key[b] = kk;
    const float tt = t[a]; t[a] = t[b]; t[b] = tt;
    const uint32_t rr = r[a]; r[a] = r[b]; r[b] = rr;
  }
}

// Packet walk of the cluster tree: the 32 lanes of a warp trace rays of one
// mesh along one node sequence. Every lane tests the same record (one load,
// shared by the warp) against its own ray; a slot is entered when some lane's
// ray enters it within that lane's reach, slots in order of the warp's
// smallest entry distance, and a stacked slot is skipped once no lane can
// still find a closer hit in it (each lane keeps its own entry distances).
// At a cluster the lanes whose ray enters it test its triangles. Lanes whose
// ray is idle (no ray, or tmax <= 0) ride along without tests. For coherent
// rays (pixel tiles) the warp stays converged where per-lane walks diverge.
// min_lanes > 0: once fewer lanes than that want the node the packet is at,
// the warp leaves the packet walk and every lane walks on alone from its own
// copy of the stack (which already holds its own entry distances).
// kBounce: also write each ray's bounce (A.b_*); a separate instantiation, since the bounce code alone (taken or
// not) costs the walk about 3% in a kernel that does not write bounces.
template <bool kCount, bool kBounce = false>
__device__ __forceinline__ void trace_warp_packet_clusters(const uint32_t r, const bool valid, const TraceArgs& A, const ClusterArgs& C,
                                                           const uint32_t min_lanes) {
  float4 o = make_float4(0.f, 0.f, 0.f, 0.f), d = make_float4(0.f, 0.f, 1.f, 0.f);
  float tmax0 = -1.0f;
  if (valid) {
    tmax0 = A.tmax ? __ldg(A.tmax + r) : kHuge;
    if (tmax0 > 0.0f) {
      o = ldg4(A.orig + r);
      d = ldg4(A.dir + r);
    }
  }
  const bool live = valid && tmax0 > 0.0f;
  int32_t best = -1;
  float bt = tmax0, bu = 0.0f, bv = 0.0f;
  uint32_t visits = 0, tests = 0;
  uint32_t ref = 0;
  const bool ok = cluster_tree_ok(C, ref);  // the same header for every lane
  if (!ok) {
    if (live && A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
  } else if (__any_sync(0xffffffffu, live)) {
    const float ix = 1.0f / fix_dir(d.x), iy = 1.0f / fix_dir(d.y), iz = 1.0f / fix_dir(d.z);
    const float4 oi = scaled_origin(o, ix, iy, iz);
    const float zu = o.w * 0.0f, zv = d.w * 0.0f;
    const float4* tris = A.tris + 3 * (size_t)C.F;
    const float4* recs = C.crec + 8 * (size_t)C.F;
    uint32_t st_ref[kStack];
    float st_t[kStack];
    int sp = 0;
    uint32_t steps = 0;
    const uint32_t kMiss = order_key(INFINITY);
    float cur_t = live ? 0.0f : INFINITY;  // this lane's entry distance of the node at hand
    auto push = [&](uint32_t sref, float st) {
      if (sp < kStack) {
        st_ref[sp] = sref;
        st_t[sp] = st;
        ++sp;
      } else if (A.err) {
        atomicOr(A.err, (uint32_t)RT_DEVERR_STACK_OVERFLOW);
      }
    };
    auto test_cluster = [&]() {
      const uint32_t p0 = ref & kClusterFirstMask, p1 = p0 + ((ref >> 28) & 7u) + 1u;
      for (uint32_t pos = p0; pos < p1; ++pos) {
        const float4 v0 = ldg4(tris + 3 * (size_t)pos);
        const float4 e1 = ldg4(tris + 3 * (size_t)pos + 1);
        const float4 e2 = ldg4(tris + 3 * (size_t)pos + 2);
        if (kCount) ++tests;
        float th, u, v;
        if (!mt_test(o, d, zu, zv, v0, e1, e2, th, u, v)) continue;
        if (th < bt || (best >= 0 && th == bt && (int32_t)pos < best)) {
          best = (int32_t)pos; bt = th; bu = u; bv = v;
        }
      }
    };
    bool alone = false;  // this warp left the packet walk
    for (;;) {
      if (!cluster_ref_ok(ref, C.n, steps)) {
        if (live && A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
        break;
      }
      const bool want = live && cur_t <= bt * kCullSlack;
      if (min_lanes && (uint32_t)__popc(__ballot_sync(0xffffffffu, want)) < min_lanes) {
        if (want) push(ref, cur_t);
        alone = true;
        break;
      }
      bool next = false;
      if (!(ref & kClusterLeaf)) {
        float t[4];
        uint32_t k[4], key[4];
        cluster_slots(recs + 8 * (size_t)ref, oi, ix, iy, iz, bt, t, k);
        if (kCount && want) visits += 4;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (!want) t[q] = INFINITY;
          key[q] = __reduce_min_sync(0xffffffffu, order_key(t[q]));
        }
        cswap_packet(key, t, k, 0, 1);
        cswap_packet(key, t, k, 2, 3);
        cswap_packet(key, t, k, 0, 2);
        cswap_packet(key, t, k, 1, 3);
        cswap_packet(key, t, k, 1, 2);
        if (key[0] != kMiss) {
#pragma unroll
          for (int q = 3; q >= 1; --q)
            if (key[q] != kMiss) push(k[q], t[q]);
          ref = k[0];
          cur_t = t[0];
          next = true;
        }
      } else if (want) {
        test_cluster();
      }
      if (next) continue;
      // the nearest stacked slot some lane can still use
      bool more = false;
      while (sp > 0) {
        --sp;
        if (__any_sync(0xffffffffu, live && st_t[sp] <= bt * kCullSlack)) {
          ref = st_ref[sp];
          cur_t = st_t[sp];
          more = true;
          break;
        }
      }
      if (!more) break;
    }
    if (alone && live) {  // every lane on its own, from its stack
      bool walking = pop_within(st_ref, st_t, sp, bt, ref);
      while (walking) {
        if (!cluster_ref_ok(ref, C.n, steps)) {
          if (A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
          break;
        }
        if (!(ref & kClusterLeaf)) {
          float t[4];
          uint32_t k[4];
          cluster_test(recs + 8 * (size_t)ref, oi, ix, iy, iz, bt, t, k);
          if (kCount) visits += 4;
          if (t[0] != INFINITY) {
#pragma unroll
            for (int q = 3; q >= 1; --q)
              if (t[q] != INFINITY) push(k[q], t[q]);
            ref = k[0];
            continue;
          }
        } else {
          test_cluster();
        }
        walking = pop_within(st_ref, st_t, sp, bt, ref);
      }
    }
  }
  if (!valid) return;
  write_hit(r, A, C.F, best, bt, bu, bv, tmax0);
  if (kCount) {
    if (A.visits) A.visits[r] = visits;
    if (A.tests) A.tests[r] = tests;
  }
  if (kBounce && A.b_orig) {  // the ray's bounce, from the hit at hand (what rt_batch_bounce_rays makes from the written hit)
    if (best >= 0) bounce_ray(A.tris, C.F + (uint32_t)best, o, d, bt, A.b_seed, r, A.b_orig, A.b_dir, A.b_tmax);
    else bounce_miss(r, A.b_orig, A.b_dir, A.b_tmax);
  }
}

// Per-lane cluster walks in warps that refill idle lanes: a lane whose ray is
// done waits until `threshold` lanes of its warp are idle, then those lanes
// take the next rays of the warp's queue and every lane steps its own walk
// again, so a warp no longer waits for its slowest ray. The queue (64 entries
// of shared memory per warp) holds active rays only: the warp takes 32 slots
// at a time with one atomic, reads their tmax together, writes the inactive
// ones (tmax <= 0) as misses at once and appends the others in slot order.
// `slot_ray` maps a slot to a ray (false for a slot without one); `mesh_args`
// sets the cluster-tree arguments of an active ray's mesh.
constexpr uint32_t kRefillQueue = 64;
template <bool kCount, bool kWW, class SlotRay, class MeshArgs>
__device__ __forceinline__ void refill_walks(const TraceArgs& A, uint32_t* counter, const uint32_t slots, const uint32_t threshold,
                                             uint32_t* q_ray, float* q_tmax, const SlotRay& slot_ray, const MeshArgs& mesh_args) {
  const uint32_t lane = lane_id();
  const uint32_t below = (1u << lane) - 1u;
  const uint32_t need = threshold ? min(threshold, 32u) : 16u;
  bool busy = false, exhausted = false;
  uint32_t q_head = 0, q_count = 0;  // warp-uniform
  uint32_t r = 0, ref = 0, visits = 0, tests = 0;
  int32_t best = -1;
  float4 o = make_float4(0.f, 0.f, 0.f, 0.f), d = o, oi = o;
  float ix = 0.f, iy = 0.f, iz = 0.f, zu = 0.f, zv = 0.f, tmax0 = 0.f, bt = 0.f, bu = 0.f, bv = 0.f;
  ClusterArgs C;
  uint32_t st_ref[kStack];
  float st_t[kStack];
  int sp = 0;
  uint32_t steps = 0;
  auto finish = [&]() {
    write_hit(r, A, C.F, best, bt, bu, bv, tmax0);
    if (kCount) {
      if (A.visits) A.visits[r] = visits;
      if (A.tests) A.tests[r] = tests;
    }
    busy = false;
  };
  for (;;) {
    const uint32_t idle = __ballot_sync(0xffffffffu, !busy);
    const uint32_t n_idle = (uint32_t)__popc(idle);
    if (n_idle >= need && (q_count || !exhausted)) {
      // top the queue up to n_idle rays (it never holds more than 31 + 32)
      while (q_count < n_idle && !exhausted) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(counter, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= slots || slots - base <= 32u) exhausted = true;
        const uint32_t slot = base + lane;
        uint32_t sr = 0;
        float st = 0.0f;
        bool act = false;
        if (slot < slots && slot_ray(slot, sr)) {
          st = A.tmax ? __ldg(A.tmax + sr) : kHuge;
          if (st > 0.0f) {
            act = true;
          } else {
            write_hit(sr, A, 0, -1, 0.0f, 0.0f, 0.0f, st);  // an inactive ray: a miss at once
            if (kCount) {
              if (A.visits) A.visits[sr] = 0;
              if (A.tests) A.tests[sr] = 0;
            }
          }
        }
        const uint32_t am = __ballot_sync(0xffffffffu, act);
        if (act) {
          const uint32_t e = (q_head + q_count + (uint32_t)__popc(am & below)) & (kRefillQueue - 1u);
          q_ray[e] = sr;
          q_tmax[e] = st;
        }
        q_count += (uint32_t)__popc(am);
      }
      __syncwarp();
      const uint32_t take = min(q_count, n_idle);
      const uint32_t k = (uint32_t)__popc(idle & below);
      if (!busy && k < take) {
        const uint32_t e = (q_head + k) & (kRefillQueue - 1u);
        r = q_ray[e];
        tmax0 = q_tmax[e];
        mesh_args(r, C);
        best = -1;
        bt = tmax0; bu = bv = 0.0f;
        visits = tests = 0;
        if (cluster_tree_ok(C, ref)) {
          o = ldg4(A.orig + r);
          d = ldg4(A.dir + r);
          ix = 1.0f / fix_dir(d.x); iy = 1.0f / fix_dir(d.y); iz = 1.0f / fix_dir(d.z);
          oi = scaled_origin(o, ix, iy, iz);
          zu = o.w * 0.0f; zv = d.w * 0.0f;
          sp = 0;
          steps = 0;
          busy = true;
        } else {
          if (A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
          finish();  // no cluster tree: a miss
        }
      }
      __syncwarp();
      q_head = (q_head + take) & (kRefillQueue - 1u);
      q_count -= take;
    }
    if (!__any_sync(0xffffffffu, busy)) {
      if (exhausted && !q_count) break;
      continue;
    }
    if (!busy) continue;
    // one step of this lane's walk
    if (!cluster_ref_ok(ref, C.n, steps)) {
      if (A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
      finish();
      continue;
    }
    const float4* recs = C.crec + 8 * (size_t)C.F;
    const bool was_cluster = (ref & kClusterLeaf) != 0;
    bool done_walk = false;  // the descent found nothing more to walk
    while (!(ref & kClusterLeaf)) {  // one record (if-if), or records until a cluster is held (while-while)
      float t[4];
      uint32_t k[4];
      cluster_test(recs + 8 * (size_t)ref, oi, ix, iy, iz, bt, t, k);
      if (kCount) visits += 4;
      if (t[0] != INFINITY) {
#pragma unroll
        for (int q = 3; q >= 1; --q) {
          if (t[q] != INFINITY) {
            if (sp < kStack) {
              st_ref[sp] = k[q];
              st_t[sp] = t[q];
              ++sp;
            } else if (A.err) {
              atomicOr(A.err, (uint32_t)RT_DEVERR_STACK_OVERFLOW);
            }
          }
        }
        ref = k[0];
      } else if (!pop_within(st_ref, st_t, sp, bt, ref)) {
        done_walk = true;
        break;
      }
      if (!kWW) break;
      if (!cluster_ref_ok(ref, C.n, steps)) {
        if (A.err) atomicOr(A.err, (uint32_t)RT_DEVERR_ACCEL_MISSING);
        done_walk = true;
        break;
      }
    }
    if (done_walk) {
      finish();
      continue;
    }
    if (!kWW && !was_cluster) continue;  // if-if: a step is one record or one cluster
    {
      // the cluster's triangles in position order; the next triangle's loads are issued before the test of the one
      // at hand, so a cluster of two or three waits for memory once
      const float4* tp = A.tris + 3 * ((size_t)C.F + (ref & kClusterFirstMask));
      const uint32_t p0 = ref & kClusterFirstMask, cnt = ((ref >> 28) & 7u) + 1u;
      auto test_tri = [&](const float4& v0, const float4& e1, const float4& e2, uint32_t pos) {
        if (kCount) ++tests;
        float th, u, v;
        if (mt_test(o, d, zu, zv, v0, e1, e2, th, u, v) && (th < bt || (best >= 0 && th == bt && (int32_t)pos < best))) {
          best = (int32_t)pos; bt = th; bu = u; bv = v;
        }
      };
      float4 a0 = ldg4(tp), a1 = ldg4(tp + 1), a2 = ldg4(tp + 2);
      float4 b0 = a0, b1 = a1, b2 = a2;
      if (cnt > 1) { b0 = ldg4(tp + 3); b1 = ldg4(tp + 4); b2 = ldg4(tp + 5); }
      test_tri(a0, a1, a2, p0);
      for (uint32_t i = 1; i < cnt; i += 2) {
        if (i + 1 < cnt) { a0 = ldg4(tp + 3 * i + 3); a1 = ldg4(tp + 3 * i + 4); a2 = ldg4(tp + 3 * i + 5); }
        test_tri(b0, b1, b2, p0 + i);
        if (i + 1 >= cnt) break;
        if (i + 2 < cnt) { b0 = ldg4(tp + 3 * i + 6); b1 = ldg4(tp + 3 * i + 7); b2 = ldg4(tp + 3 * i + 8); }
        test_tri(a0, a1, a2, p0 + i + 1);
      }
    }
    if (!pop_within(st_ref, st_t, sp, bt, ref)) finish();
  }
}

// Slot -> ray. With an image width, slots walk 8x4 pixel tiles of the
// row-major image (a warp traces one tile); otherwise slots are ray indices.
struct SlotMap {
  uint32_t width, height, tiles_x, slots;
  const uint32_t* order;  // optional slot -> ray permutation (rt_ray_order)
  __device__ __forceinline__ bool ray_of(uint32_t s, uint32_t& r) const {
    if (order) { r = __ldg(order + s); return s < slots; }
    if (!width) { r = s; return s < slots; }
    const uint32_t tile = s >> 5, w = s & 31u;
    const uint32_t x = (tile % tiles_x) * 8 + (w & 7u), y = (tile / tiles_x) * 4 + (w >> 3);
    r = y * width + x;
    return x < width && y < height;
  }
};

template <bool kCount, bool kWW, bool kSeed, bool kWide>
__global__ __launch_bounds__(128) void k_trace_accel(TraceArgs A, AccelArgs C, SlotMap M, SeedArgs S) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t r;
  C.F = C.G = 0;  // one mesh: no offsets (known to the compiler)
  if (s < M.slots && M.ray_of(s, r)) trace_ray_accel<kCount, kWW, kSeed, kWide>(r, A, C, S);
}

template <bool kCount, bool kSeed, bool kWide>
__global__ __launch_bounds__(128, kSeed ? 6 : 0) void k_trace_coop(TraceArgs A, AccelArgs C, SlotMap M, SeedArgs S) {
  __shared__ unsigned long long s_key[kCoopWarps][32];
  __shared__ float2 s_uv[kCoopWarps][32];
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t r = 0;
  const bool valid = s < M.slots && M.ray_of(s, r);
  const uint32_t w = threadIdx.x >> 5;
  C.F = C.G = 0;
  trace_warp_coop<kCount, kSeed, kWide>(r, valid, A, C, s_key[w], s_uv[w], S);
}

template <bool kCount, bool kSeed, bool kWide>
__global__ __launch_bounds__(128, kSeed ? 6 : (kCount ? 0 : 7)) void k_trace_coop_persistent(TraceArgs A, AccelArgs C, SlotMap M, uint32_t* counter,
                                                                          SeedArgs S) {
  __shared__ unsigned long long s_key[kCoopWarps][32];
  __shared__ float2 s_uv[kCoopWarps][32];
  __shared__ uint32_t s_rec[kMaxStaged];
  extern __shared__ float4 s_tree[];
  C.F = C.G = 0;
  if (kWide && C.stage_depth) C.stage = stage_treelet(C, s_tree, s_rec, C.stage_depth);
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= M.slots) break;
    uint32_t r = 0;
    const uint32_t s = base + lane;
    const bool valid = s < M.slots && M.ray_of(s, r);
    trace_warp_coop<kCount, kSeed, kWide>(r, valid, A, C, s_key[w], s_uv[w], S);
  }
}

// Persistent warps: each warp takes 32 slots at a time from a global counter
// until the slots run out (the counter is zeroed before the launch).
template <bool kCount, bool kWW, bool kSeed, bool kWide>
__global__ __launch_bounds__(128) void k_trace_accel_persistent(TraceArgs A, AccelArgs C, SlotMap M, uint32_t* counter, SeedArgs S) {
  __shared__ uint32_t s_rec[kMaxStaged];
  extern __shared__ float4 s_tree[];
  C.F = C.G = 0;
  if (kWide && C.stage_depth) C.stage = stage_treelet(C, s_tree, s_rec, C.stage_depth);
  const uint32_t lane = lane_id();
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= M.slots) break;
    uint32_t r;
    const uint32_t s = base + lane;
    if (s < M.slots && M.ray_of(s, r)) trace_ray_accel<kCount, kWW, kSeed, kWide>(r, A, C, S);
  }
}

// Batched traversal: one launch for the rays of all meshes of rt_batch_build;
// each ray finds its mesh by binary search over ray_offsets and traverses that
// mesh's part of the blob with the single-mesh per-ray code.
struct BatchTraceArgs {
  uint32_t M;
  const uint32_t* foff;
  const uint32_t* roff;
  BatchAccel acc;
  const uint32_t* order;  // optional slot -> ray permutation (rt_batch_ray_order, rt_image_tile_order)
  __device__ __forceinline__ uint32_t ray_of(uint32_t s) const { return order ? __ldg(order + s) : s; }
};

// Seeded: the slot tables of mesh m start at m slot_count entries.
template <bool kCount, bool kWW, bool kSeed, bool kWide>
__device__ __forceinline__ void batch_trace_ray(uint32_t r, const TraceArgs& A, const BatchTraceArgs& B, const SeedArgs& S) {
  const uint32_t m = find_seg(B.roff, B.M, r);
  const uint32_t F = __ldg(B.foff + m);
  AccelArgs C;
  C.hdr = B.acc.hdr + 64 * (size_t)m;
  C.tnodes = B.acc.tnodes;
  C.leaves = B.acc.leaves;
  C.groups = B.acc.groups;
  C.wide = B.acc.wide;
  C.F = F;
  C.G = group_base(F, m);
  if constexpr (kSeed) {
    SeedArgs Sm = S;
    Sm.slot_ref = S.slot_ref + (size_t)m * S.slot_count;
    if (S.slot_box) Sm.slot_box = S.slot_box + 2 * (size_t)m * S.slot_count;
    trace_ray_accel<kCount, kWW, true, kWide>(r, A, C, Sm);
  } else {
    trace_ray_accel<kCount, kWW, false, kWide>(r, A, C);
  }
}

template <bool kCount, bool kWW, bool kSeed, bool kWide>
__global__ __launch_bounds__(128) void k_batch_trace(TraceArgs A, BatchTraceArgs B, SeedArgs S) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < A.ray_count) batch_trace_ray<kCount, kWW, kSeed, kWide>(B.ray_of(s), A, B, S);
}

// The per-ray arguments of batched ray r: its mesh's part of the blob, triangle
// stream and indices, and (seeded) slot tables.
template <bool kSeed>
__device__ __forceinline__ void batch_ray_args(uint32_t r, const TraceArgs& A, const BatchTraceArgs& B, const SeedArgs& S, TraceArgs& Am,
                                               AccelArgs& C, SeedArgs& Sm) {
  const uint32_t m = find_seg(B.roff, B.M, r);
  const uint32_t F = __ldg(B.foff + m);
  C.hdr = B.acc.hdr + 64 * (size_t)m;
  C.F = F;
  C.G = group_base(F, m);
  Am = A;
  Sm = S;
  if (kSeed) {
    Sm.slot_ref = S.slot_ref + (size_t)m * S.slot_count;
    if (S.slot_box) Sm.slot_box = S.slot_box + 2 * (size_t)m * S.slot_count;
  }
}

// Warp-cooperative leaf tests over batched rays (persistent warps, 32 rays at a
// time): each lane walks its own mesh; a lane testing another lane's leaf reads
// that lane's triangle stream.
template <bool kCount, bool kSeed, bool kWide>
__global__ __launch_bounds__(128, kSeed ? 6 : (kCount ? 0 : 7)) void k_batch_trace_coop(TraceArgs A, BatchTraceArgs B, SeedArgs S,
                                                                                      uint32_t* counter) {
  __shared__ unsigned long long s_key[kCoopWarps][32];
  __shared__ float2 s_uv[kCoopWarps][32];
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= A.ray_count) break;
    const uint32_t slot = base + lane;
    const bool valid = slot < A.ray_count;
    const uint32_t r = valid ? B.ray_of(slot) : slot;
    TraceArgs Am = A;
    AccelArgs C = {};  // the batch's base pointers (uniform); each lane adds its mesh's offsets
    C.hdr = B.acc.hdr; C.tnodes = B.acc.tnodes; C.leaves = B.acc.leaves; C.groups = B.acc.groups; C.wide = B.acc.wide;
    SeedArgs Sm = S;
    if (valid) batch_ray_args<kSeed>(r, A, B, S, Am, C, Sm);  // idle lanes keep mesh 0's header and zero offsets
    trace_warp_coop<kCount, kSeed, kWide>(r, valid, Am, C, s_key[w], s_uv[w], Sm);
  }
}

// Persistent warps over the batched rays: 32 rays at a time from a global counter.
template <bool kCount, bool kWW, bool kSeed, bool kWide>
__global__ __launch_bounds__(128) void k_batch_trace_persistent(TraceArgs A, BatchTraceArgs B, SeedArgs S, uint32_t* counter) {
  const uint32_t lane = lane_id();
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= A.ray_count) break;
    const uint32_t slot = base + lane;
    if (slot < A.ray_count) batch_trace_ray<kCount, kWW, kSeed, kWide>(B.ray_of(slot), A, B, S);
  }
}

// Cluster tree kernels: single mesh (slots through a SlotMap) and batched (each ray's mesh by binary search).
template <bool kCount, bool kWW>
__global__ __launch_bounds__(128) void k_trace_clusters(TraceArgs A, ClusterArgs C, SlotMap M) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t r;
  C.F = 0;
  if (s < M.slots && M.ray_of(s, r)) trace_ray_clusters<kCount, kWW>(r, A, C);
}
template <bool kCount, bool kWW>
__global__ __launch_bounds__(128) void k_trace_clusters_persistent(TraceArgs A, ClusterArgs C, SlotMap M, uint32_t* counter) {
  const uint32_t lane = lane_id();
  C.F = 0;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= M.slots) break;
    uint32_t r;
    const uint32_t s = base + lane;
    if (s < M.slots && M.ray_of(s, r)) trace_ray_clusters<kCount, kWW>(r, A, C);
  }
}
template <bool kCount>
__global__ __launch_bounds__(128) void k_trace_clusters_coop(TraceArgs A, ClusterArgs C, SlotMap M, uint32_t* counter) {
  __shared__ unsigned long long s_key[kCoopWarps][32];
  __shared__ float2 s_uv[kCoopWarps][32];
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  C.F = 0;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= M.slots) break;
    uint32_t r = 0;
    const uint32_t s = base + lane;
    const bool valid = s < M.slots && M.ray_of(s, r);
    trace_warp_coop_clusters<kCount>(r, valid, A, C, s_key[w], s_uv[w]);
  }
}

template <bool kCount>
__global__ __launch_bounds__(128) void k_trace_clusters_packet(TraceArgs A, ClusterArgs C, SlotMap M, uint32_t* counter,
                                                                uint32_t min_lanes) {
  const uint32_t lane = lane_id();
  C.F = 0;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= M.slots) break;
    uint32_t r = 0;
    const uint32_t s = base + lane;
    const bool valid = s < M.slots && M.ray_of(s, r);
    trace_warp_packet_clusters<kCount>(r, valid, A, C, min_lanes);
  }
}

// Refill walks are latency-bound: eight CTAs (32 warps) per SM, 64 registers, outrun seven CTAs at the 72 registers
// the compiler would take for the pipelined triangle loads.
template <bool kCount, bool kWW>
__global__ __launch_bounds__(128, 8) void k_trace_clusters_refill(TraceArgs A, ClusterArgs C, SlotMap M, uint32_t* counter,
                                                                uint32_t threshold) {
  __shared__ uint32_t q_ray[4][kRefillQueue];
  __shared__ float q_tmax[4][kRefillQueue];
  C.F = 0;
  const uint32_t w = threadIdx.x >> 5;
  refill_walks<kCount, kWW>(
      A, counter, M.slots, threshold, q_ray[w], q_tmax[w], [&](uint32_t slot, uint32_t& r) { return M.ray_of(slot, r); },
      [&](uint32_t, ClusterArgs& Cl) { Cl = C; });
}

__device__ __forceinline__ void batch_cluster_args(uint32_t r, const BatchTraceArgs& B, ClusterArgs& C) {
  const uint32_t m = find_seg(B.roff, B.M, r);
  const uint32_t F = __ldg(B.foff + m);
  C.hdr = B.acc.hdr + 64 * (size_t)m;
  C.F = F;
  C.n = __ldg(B.foff + m + 1) - F;
}
template <bool kCount, bool kWW>
__global__ __launch_bounds__(128) void k_batch_trace_clusters(TraceArgs A, BatchTraceArgs B) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= A.ray_count) return;
  const uint32_t r = B.ray_of(s);
  ClusterArgs C;
  C.crec = B.acc.crec;
  batch_cluster_args(r, B, C);
  trace_ray_clusters<kCount, kWW>(r, A, C);
}
template <bool kCount, bool kWW>
__global__ __launch_bounds__(128) void k_batch_trace_clusters_persistent(TraceArgs A, BatchTraceArgs B, uint32_t* counter) {
  const uint32_t lane = lane_id();
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= A.ray_count) break;
    const uint32_t slot = base + lane;
    if (slot < A.ray_count) {
      const uint32_t r = B.ray_of(slot);
      ClusterArgs C;
      C.crec = B.acc.crec;
      batch_cluster_args(r, B, C);
      trace_ray_clusters<kCount, kWW>(r, A, C);
    }
  }
}
template <bool kCount, bool kWW>
__global__ __launch_bounds__(128, 8) void k_batch_trace_clusters_refill(TraceArgs A, BatchTraceArgs B, uint32_t* counter,
                                                                      uint32_t threshold) {
  __shared__ uint32_t q_ray[4][kRefillQueue];
  __shared__ float q_tmax[4][kRefillQueue];
  const uint32_t w = threadIdx.x >> 5;
  refill_walks<kCount, kWW>(
      A, counter, A.ray_count, threshold, q_ray[w], q_tmax[w],
      [&](uint32_t slot, uint32_t& r) {
        r = B.ray_of(slot);
        return true;
      },
      [&](uint32_t r, ClusterArgs& C) {
        C.crec = B.acc.crec;
        batch_cluster_args(r, B, C);
      });
}

// Packet walks over batched rays: a warp whose valid rays all belong to one mesh walks it as a packet; a warp
// spanning meshes falls back to per-lane walks.
template <bool kCount, bool kBounce>
__global__ __launch_bounds__(128) void k_batch_trace_clusters_packet(TraceArgs A, BatchTraceArgs B, uint32_t* counter,
                                                                      uint32_t min_lanes) {
  const uint32_t lane = lane_id();
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= A.ray_count) break;
    const uint32_t slot = base + lane;
    const bool valid = slot < A.ray_count;
    const uint32_t r = valid ? B.ray_of(slot) : 0u;
    ClusterArgs C;
    C.crec = B.acc.crec;
    C.hdr = B.acc.hdr;
    if (valid) batch_cluster_args(r, B, C);
    // lane 0 always holds a valid slot (base < ray_count); its mesh is the packet's
    const uint32_t F0 = __shfl_sync(0xffffffffu, C.F, 0);
    if (__all_sync(0xffffffffu, !valid || C.F == F0)) {
      ClusterArgs P;
      P.crec = B.acc.crec;
      P.hdr = (const uint32_t*)__shfl_sync(0xffffffffu, (unsigned long long)C.hdr, 0);
      P.F = F0;
      P.n = __shfl_sync(0xffffffffu, C.n, 0);
      trace_warp_packet_clusters<kCount, kBounce>(r, valid, A, P, min_lanes);
    } else if (valid) {
      trace_ray_clusters<kCount, false, kBounce>(r, A, C);
    }
  }
}

template <bool kCount>
__global__ __launch_bounds__(128) void k_batch_trace_clusters_coop(TraceArgs A, BatchTraceArgs B, uint32_t* counter) {
  __shared__ unsigned long long s_key[kCoopWarps][32];
  __shared__ float2 s_uv[kCoopWarps][32];
  const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= A.ray_count) break;
    const uint32_t slot = base + lane;
    const bool valid = slot < A.ray_count;
    const uint32_t r = valid ? B.ray_of(slot) : slot;
    ClusterArgs C;  // idle lanes: mesh 0's header, no walk
    C.crec = B.acc.crec;
    C.hdr = B.acc.hdr;
    if (valid) batch_cluster_args(r, B, C);
    trace_warp_coop_clusters<kCount>(r, valid, A, C, s_key[w], s_uv[w]);
  }
}

// Sort key of a ray: direction octant (3 bits) above a 21-bit Morton code of
// its origin in the given box (128 cells per axis); inactive rays (tmax <= 0)
// sort last.
__global__ __launch_bounds__(256) void k_ray_keys(const float4* __restrict__ orig, const float4* __restrict__ dir,
                                                 const float* __restrict__ tmax, uint32_t count, float3 lo, float3 scale,
                                                 uint32_t* __restrict__ keys, uint32_t* __restrict__ idx) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < count; r += gridDim.x * blockDim.x) {
    idx[r] = r;
    if (tmax && !(__ldg(tmax + r) > 0.0f)) { keys[r] = 0xFFFFFFu; continue; }
    const float4 o = ldg4(orig + r), d = ldg4(dir + r);
    const uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    uint32_t q[3];
    const float c[3] = {(o.x - lo.x) * scale.x, (o.y - lo.y) * scale.y, (o.z - lo.z) * scale.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) q[a] = min(__float2uint_rz(fmaxf(c[a], 0.0f)), 511u) >> 2;  // 7 bits per axis
    uint32_t m = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b) m |= ((q[0] >> b) & 1u) << (3 * b + 2) | ((q[1] >> b) & 1u) << (3 * b + 1) | ((q[2] >> b) & 1u) << (3 * b);
    // 3 + 21 bits: three radix passes (a finer code sorts slower than it gains). 0xFFFFFF is kept for the
    // inactive rays, so an octant-7 ray in the top cell on all three axes shares the key of its neighbour cell.
    keys[r] = min((oct << 21) | m, 0xFFFFFEu);
  }
}

// Sort key of a batched ray: its mesh id (found in ray_offsets) above its direction octant above the top
// `mbits` bits (a multiple of 3) of the 21-bit Morton code of its origin in `box`; inactive rays get the key of
// a mesh id one past the last, so that they sort after every active ray.
__global__ __launch_bounds__(256) void k_batch_ray_keys(const float4* __restrict__ orig, const float4* __restrict__ dir,
                                                       const float* __restrict__ tmax, uint32_t count, const uint32_t* __restrict__ roff,
                                                       uint32_t M, uint32_t mbits, float3 lo, float3 scale, uint32_t* __restrict__ keys,
                                                       uint32_t* __restrict__ idx) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < count; r += gridDim.x * blockDim.x) {
    idx[r] = r;
    if (tmax && !(__ldg(tmax + r) > 0.0f)) { keys[r] = M << (3 + mbits); continue; }
    const uint32_t m = find_seg(roff, M, r);
    const float4 o = ldg4(orig + r), d = ldg4(dir + r);
    const uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    uint32_t mc = 0;
    if (mbits) {
      uint32_t q[3];
      const float c[3] = {(o.x - lo.x) * scale.x, (o.y - lo.y) * scale.y, (o.z - lo.z) * scale.z};
#pragma unroll
      for (int a = 0; a < 3; ++a) q[a] = min(__float2uint_rz(fmaxf(c[a], 0.0f)), 511u) >> 2;  // 7 bits per axis
#pragma unroll
      for (int b = 0; b < 7; ++b)
        mc |= ((q[0] >> b) & 1u) << (3 * b + 2) | ((q[1] >> b) & 1u) << (3 * b + 1) | ((q[2] >> b) & 1u) << (3 * b);
      mc >>= 21 - mbits;
    }
    keys[r] = (m << (3 + mbits)) | (oct << mbits) | mc;
  }
}

// Slot -> ray of `images` row-major width x height images stored one after the other: a warp's 32 slots are
// an 8 x 4 pixel tile of one image, tiles in row-major order (width % 8 == 0, height % 4 == 0).
__global__ __launch_bounds__(256) void k_image_tile_order(uint32_t total, uint32_t width, uint32_t height, uint32_t* __restrict__ order) {
  const uint32_t per = width * height, tiles_x = width / 8;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < total; s += gridDim.x * blockDim.x) {
    const uint32_t img = s / per, k = s - img * per, tile = k >> 5, w = k & 31u;
    const uint32_t x = (tile % tiles_x) * 8 + (w & 7u), y = (tile / tiles_x) * 4 + (w >> 3);
    order[s] = img * per + y * width + x;
  }
}

// kernels/CUDA_calcPrimaryRays.cu:20-32
// The rays of `count` cameras, camera c's rows at c w h: the arithmetic of k_primary with camera c's basis
// (origin, direction, x step, y step) read from `bases` (four float4 per camera).
__global__ __launch_bounds__(256) void k_batch_primary(const float4* __restrict__ bases, uint32_t count, uint32_t w, uint32_t h,
                                                       float4* __restrict__ orig, float4* __restrict__ dir) {
  const uint32_t per = w * h;
  const size_t total = (size_t)count * per;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
    const uint32_t c = (uint32_t)(g / per), n = (uint32_t)(g % per);
    const float4 ro = __ldg(bases + 4 * c), rd = __ldg(bases + 4 * c + 1), rx = __ldg(bases + 4 * c + 2), ry = __ldg(bases + 4 * c + 3);
    const float x = (float)(n % w), y = (float)(n / w);
    orig[g] = ro;
    dir[g] = make_float4((rd.x - x * rx.x) - y * ry.x, (rd.y - x * rx.y) - y * ry.y, (rd.z - x * rx.z) - y * ry.z,
                         (rd.w - x * rx.w) - y * ry.w);
  }
}
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

// kBatch: hit_pos is a position inside the ray's own mesh of a batched build (the rays of mesh m are
// ray_off[m] .. ray_off[m + 1]); the mesh's first face position face_off[m] is added before the triangle
// is read. The PCG stream is the ray index either way.
template <bool kBatch>
__global__ __launch_bounds__(256) void k_bounce(const float4* __restrict__ tris, const float4* __restrict__ orig,
                                               const float4* __restrict__ dir, const int32_t* __restrict__ hit_pos,
                                               const float* __restrict__ hit_t, uint32_t count, uint64_t seed,
                                               float4* __restrict__ orig_out, float4* __restrict__ dir_out, float* __restrict__ tmax_out,
                                               const uint32_t* __restrict__ ray_off, const uint32_t* __restrict__ face_off, uint32_t M) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < count; r += gridDim.x * blockDim.x) {
    int32_t pos = hit_pos[r];
    if (kBatch && pos >= 0) {
      uint32_t lo = 0, hi = M;  // largest m with ray_off[m] <= r
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(ray_off + mid) <= r) lo = mid; else hi = mid;
      }
      pos += (int32_t)__ldg(face_off + lo);
    }
    if (pos < 0) {
      bounce_miss(r, orig_out, dir_out, tmax_out);
      continue;
    }
    bounce_ray(tris, (uint32_t)pos, orig[r], dir[r], hit_t[r], seed, r, orig_out, dir_out, tmax_out);
  }
}

// A tracing order with the active rays (tmax > 0) first: each warp takes a run of 1024 consecutive rays, counts
// its active ones, reserves one contiguous stretch for them (and one, from the end backwards, for the inactive
// ones) and writes them in ray order, so that neighbouring rays stay together in the order. ctr: 2 zeroed words.
constexpr uint32_t kOrderRun = 1024;
__global__ __launch_bounds__(256) void k_active_first_order(const float* __restrict__ tmax, uint32_t count, uint32_t* __restrict__ order,
                                                            uint32_t* __restrict__ ctr) {
  const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t run = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); (size_t)run * kOrderRun < count; run += warps) {
    const uint32_t r0 = run * kOrderRun, r1 = min(count, r0 + kOrderRun);
    uint32_t na = 0, ni = 0;
    for (uint32_t b = r0; b < r1; b += 32) {
      const bool in = b + lane < r1;
      const bool act = in && __ldg(tmax + b + lane) > 0.0f;
      na += __popc(__ballot_sync(0xffffffffu, act));
      ni += __popc(__ballot_sync(0xffffffffu, in && !act));
    }
    uint32_t ab = 0, ib = 0;
    if (lane == 0) {
      if (na) ab = atomicAdd(ctr, na);
      if (ni) ib = atomicAdd(ctr + 1, ni);
    }
    ab = __shfl_sync(0xffffffffu, ab, 0);
    ib = __shfl_sync(0xffffffffu, ib, 0);
    for (uint32_t b = r0; b < r1; b += 32) {
      const uint32_t r = b + lane;
      const bool in = r < r1;
      const bool act = in && __ldg(tmax + r) > 0.0f;
      const uint32_t am = __ballot_sync(0xffffffffu, act), im = __ballot_sync(0xffffffffu, in && !act);
      if (act) order[ab + __popc(am & lt)] = r;
      else if (in) order[count - 1u - (ib + __popc(im & lt))] = r;
      ab += __popc(am);
      ib += __popc(im);
    }
  }
}

// SM count of the current device (cached per device).
int sms() {
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

}  // namespace
// Hit packing for download: blocks of kPackRays rays (256 threads x 8 consecutive rays); one pass counts each
// block's hits, a scan turns the counts into block offsets (and the total), a second pass writes (t, u, v) of
// every hit at its block offset plus its rank in the block.
constexpr uint32_t kPackRays = 2048;
__global__ __launch_bounds__(256) void k_pack_count(const int32_t* __restrict__ id, uint32_t n, uint32_t* __restrict__ block_hits) {
  __shared__ uint32_t s_w[8];
  const uint32_t base = blockIdx.x * kPackRays + threadIdx.x * 8u;
  uint32_t c = 0;
#pragma unroll
  for (uint32_t k = 0; k < 8; ++k) c += (base + k < n && __ldg(id + base + k) >= 0) ? 1u : 0u;
  uint32_t total;
  block_excl_scan_nt<256>(c, s_w, total);
  if (threadIdx.x == 0) block_hits[blockIdx.x] = total;
}
__global__ __launch_bounds__(256) void k_pack_write(const int32_t* __restrict__ id, const float* __restrict__ t,
                                                    const float2* __restrict__ uv, uint32_t n, const uint32_t* __restrict__ block_base,
                                                    float* __restrict__ packed) {
  __shared__ uint32_t s_w[8];
  const uint32_t base = blockIdx.x * kPackRays + threadIdx.x * 8u;
  uint32_t m = 0;
#pragma unroll
  for (uint32_t k = 0; k < 8; ++k)
    if (base + k < n && __ldg(id + base + k) >= 0) m |= 1u << k;
  uint32_t total;
  uint32_t o = block_base[blockIdx.x] + block_excl_scan_nt<256>((uint32_t)__popc(m), s_w, total);
#pragma unroll
  for (uint32_t k = 0; k < 8; ++k) {
    if (!((m >> k) & 1u)) continue;
    const float2 w = __ldg(uv + base + k);
    packed[3 * (size_t)o] = __ldg(t + base + k);
    packed[3 * (size_t)o + 1] = w.x;
    packed[3 * (size_t)o + 2] = w.y;
    ++o;
  }
}

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

namespace {

// Thread slots of a single-mesh launch: a given ray order, 8x4 pixel tiles of an image, or the rays in order.
SlotMap slot_map(const rt_trace_desc* d) {
  SlotMap M;
  M.order = d->ray_order;
  const uint32_t R = d->ray_count;
  if (d->ray_order) {
    M.width = 0; M.height = 0; M.tiles_x = 0; M.slots = R;
  } else if (d->image_width && R % d->image_width == 0) {
    M.width = d->image_width;
    M.height = R / d->image_width;
    M.tiles_x = (M.width + 7) / 8;
    M.slots = M.tiles_x * ((M.height + 3) / 4) * 32;
  } else {
    M.width = 0; M.height = 0; M.tiles_x = 0; M.slots = R;
  }
  return M;
}

// Cluster tree launch (RT_TRACE_CLUSTERS): per-lane walks (a grid, or persistent warps with a work counter) or
// the warp-cooperative walk (RT_TRACE_COOP, persistent warps; without a work counter the per-lane grid).
rt_status launch_clusters(const rt_trace_desc* d, const TraceArgs& A, cudaStream_t st) {
  const bool count = d->ray_visits || d->ray_tests;
  const bool ww = (d->schedule & RT_TRACE_WHILE_WHILE) != 0;
  ClusterArgs C;
  {
    Carve c((void*)d->accel, ~(size_t)0);
    AccelLayout AL;
    carve_accel(c, AL, d->face_count_hint);
    C.crec = AL.crec;
    C.hdr = AL.hdr;
  }
  C.n = d->face_count_hint;
  const SlotMap M = slot_map(d);
  if (d->work_counter) {
    if (cudaMemsetAsync(d->work_counter, 0, 4, st) != cudaSuccess) return RT_ERR_CUDA;
    const uint32_t blocks = (uint32_t)hmin<uint64_t>((uint64_t)sms() * (d->persistent_blocks_per_sm ? d->persistent_blocks_per_sm : 8u),
                                                     ((uint64_t)M.slots + 127) / 128);
    if (d->schedule & RT_TRACE_PACKET) {
      if (count) k_trace_clusters_packet<true><<<blocks, 128, 0, st>>>(A, C, M, d->work_counter, d->lane_threshold);
      else k_trace_clusters_packet<false><<<blocks, 128, 0, st>>>(A, C, M, d->work_counter, d->lane_threshold);
    } else if (d->schedule & RT_TRACE_REFILL) {
#define RT_LAUNCH_CR(CNT, WW) k_trace_clusters_refill<CNT, WW><<<blocks, 128, 0, st>>>(A, C, M, d->work_counter, d->lane_threshold)
      if (count) { if (ww) RT_LAUNCH_CR(true, true); else RT_LAUNCH_CR(true, false); }
      else { if (ww) RT_LAUNCH_CR(false, true); else RT_LAUNCH_CR(false, false); }
#undef RT_LAUNCH_CR
    } else if (d->schedule & RT_TRACE_COOP) {
      if (count) k_trace_clusters_coop<true><<<blocks, 128, 0, st>>>(A, C, M, d->work_counter);
      else k_trace_clusters_coop<false><<<blocks, 128, 0, st>>>(A, C, M, d->work_counter);
    } else {
#define RT_LAUNCH_CP(CNT, WW) k_trace_clusters_persistent<CNT, WW><<<blocks, 128, 0, st>>>(A, C, M, d->work_counter)
      if (count) { if (ww) RT_LAUNCH_CP(true, true); else RT_LAUNCH_CP(true, false); }
      else { if (ww) RT_LAUNCH_CP(false, true); else RT_LAUNCH_CP(false, false); }
#undef RT_LAUNCH_CP
    }
  } else {
    const uint32_t blocks = (M.slots + 127) / 128;
#define RT_LAUNCH_CS(CNT, WW) k_trace_clusters<CNT, WW><<<blocks, 128, 0, st>>>(A, C, M)
    if (count) { if (ww) RT_LAUNCH_CS(true, true); else RT_LAUNCH_CS(true, false); }
    else { if (ww) RT_LAUNCH_CS(false, true); else RT_LAUNCH_CS(false, false); }
#undef RT_LAUNCH_CS
  }
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

// Blob traversal launch for every schedule of rt_trace_desc.
template <bool kSeed, bool kWide>
rt_status launch_accel_w(const rt_trace_desc* d, const TraceArgs& A, const SeedArgs& S, cudaStream_t st) {
  const bool count = d->ray_visits || d->ray_tests;
  // blob layout of rt_lbvh_build / rt_sah_build
  const size_t n = d->face_count_hint;
  AccelArgs C;
  {
    Carve c((void*)d->accel, ~(size_t)0);
    AccelLayout AL;
    carve_accel(c, AL, (uint32_t)n);
    C.hdr = AL.hdr; C.tnodes = AL.tnodes; C.leaves = AL.leaves; C.groups = AL.groups; C.wide = AL.wide;
  }
  // the top treelet is staged by the persistent kernels of the 4-wide walk only (one copy per CTA)
  C.stage_depth = (kWide && d->work_counter) ? (d->treelet_depth < kMaxStageDepth ? d->treelet_depth : kMaxStageDepth) : 0u;
  const size_t stage_smem = (size_t)staged_slots(C.stage_depth) * 128;
  const SlotMap M = slot_map(d);
  const bool ww = (d->schedule & RT_TRACE_WHILE_WHILE) != 0;
  const uint32_t pblocks = (uint32_t)sms() * (d->persistent_blocks_per_sm ? d->persistent_blocks_per_sm : 8u);
  const uint32_t sblocks = (M.slots + 127) / 128;
  if (d->work_counter && cudaMemsetAsync(d->work_counter, 0, 4, st) != cudaSuccess) return RT_ERR_CUDA;
  if (d->schedule & RT_TRACE_COOP) {
    if (d->work_counter) {
      if (count) k_trace_coop_persistent<true, kSeed, kWide><<<pblocks, 128, stage_smem, st>>>(A, C, M, d->work_counter, S);
      else k_trace_coop_persistent<false, kSeed, kWide><<<pblocks, 128, stage_smem, st>>>(A, C, M, d->work_counter, S);
    } else {
      if (count) k_trace_coop<true, kSeed, kWide><<<sblocks, 128, 0, st>>>(A, C, M, S);
      else k_trace_coop<false, kSeed, kWide><<<sblocks, 128, 0, st>>>(A, C, M, S);
    }
  } else if (d->work_counter) {
#define RT_LAUNCH_P(CNT, WW) \
  k_trace_accel_persistent<CNT, WW, kSeed, kWide><<<pblocks, 128, stage_smem, st>>>(A, C, M, d->work_counter, S)
    if (count) { if (ww) RT_LAUNCH_P(true, true); else RT_LAUNCH_P(true, false); }
    else { if (ww) RT_LAUNCH_P(false, true); else RT_LAUNCH_P(false, false); }
#undef RT_LAUNCH_P
  } else {
#define RT_LAUNCH_S(CNT, WW) k_trace_accel<CNT, WW, kSeed, kWide><<<sblocks, 128, 0, st>>>(A, C, M, S)
    if (count) { if (ww) RT_LAUNCH_S(true, true); else RT_LAUNCH_S(true, false); }
    else { if (ww) RT_LAUNCH_S(false, true); else RT_LAUNCH_S(false, false); }
#undef RT_LAUNCH_S
  }
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

template <bool kSeed>
rt_status launch_accel(const rt_trace_desc* d, const TraceArgs& A, const SeedArgs& S, cudaStream_t st) {
  if (d->schedule & RT_TRACE_CLUSTERS) return kSeed ? RT_ERR_UNSUPPORTED : launch_clusters(d, A, st);
  if (d->schedule & RT_TRACE_WIDE) return launch_accel_w<kSeed, true>(d, A, S, st);
  return launch_accel_w<kSeed, false>(d, A, S, st);
}

rt_status trace_args(const rt_trace_desc* d, TraceArgs& A) {
  if (!d || !d->nodes || !d->orig || !d->dir || !d->hit_id || !d->hit_t || !d->hit_uv) return RT_ERR_INVALID_ARGUMENT;
  if (!d->tris && (!d->vertices || !d->faces)) return RT_ERR_INVALID_ARGUMENT;
  if (d->id_mode == 1 && !d->indices) return RT_ERR_INVALID_ARGUMENT;
  if (d->ray_count > RT_MAX_RAYS) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  A.nodes = (const uint4*)d->nodes; A.tris = (const float4*)d->tris; A.verts = (const float4*)d->vertices;
  A.faces = (const uint4*)d->faces; A.indices = d->indices; A.orig = (const float4*)d->orig; A.dir = (const float4*)d->dir;
  A.tmax = d->tmax; A.ray_count = d->ray_count; A.id_mode = d->id_mode; A.hit_id = d->hit_id; A.hit_t = d->hit_t;
  A.hit_uv = (float2*)d->hit_uv; A.visits = d->ray_visits; A.tests = d->ray_tests; A.err = d->error_word;
  A.b_orig = nullptr; A.b_dir = nullptr; A.b_tmax = nullptr; A.b_seed = 0;
  return RT_OK;
}

}  // namespace

extern "C" rt_status rt_trace_closest(const rt_trace_desc* d, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_trace_closest");
  TraceArgs A = {};
  const rt_status s = trace_args(d, A);
  if (s != RT_OK) return s;
  if (d->ray_count == 0) return RT_OK;
  const bool count = d->ray_visits || d->ray_tests;
  const uint32_t blocks = (d->ray_count + 127) / 128;
  cudaStream_t st = (cudaStream_t)stream;
  if (d->accel) {
    if (!d->tris) return RT_ERR_INVALID_ARGUMENT;
    return launch_accel<false>(d, A, SeedArgs{}, st);
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

extern "C" rt_status rt_trace_closest_seeded(const rt_trace_desc* d, const rt_seed_desc* sd, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_trace_closest_seeded");
  TraceArgs A = {};
  const rt_status s = trace_args(d, A);
  if (s != RT_OK) return s;
  if (!sd || !sd->proposal || !sd->slot_ref || !d->accel || !d->tris) return RT_ERR_INVALID_ARGUMENT;
  if (d->ray_count == 0) return RT_OK;
  SeedArgs S;
  S.proposal = sd->proposal; S.slot_ref = sd->slot_ref; S.slot_box = (const float4*)sd->slot_box; S.slot_count = sd->slot_count;
  S.in_prop = sd->in_proposal;
  return launch_accel<true>(d, A, S, (cudaStream_t)stream);
}

extern "C" rt_status rt_ray_order_scratch_bytes(uint32_t count, size_t* bytes) {
  if (!bytes) return RT_ERR_INVALID_ARGUMENT;
  Carve c(nullptr, 0);
  c.take<uint32_t>(count);
  *bytes = c.off + radix_scratch_bytes(count) + 512;
  return RT_OK;
}

extern "C" rt_status rt_ray_order(const float* orig, const float* dir, const float* tmax, uint32_t count, const float box[6],
                                  uint32_t* order, void* scratch, size_t scratch_bytes, rt_stream stream) {
  if (!orig || !dir || !order || !box) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (count == 0) return RT_OK;
  size_t need = 0;
  rt_ray_order_scratch_bytes(count, &need);
  if (!scratch || scratch_bytes < need) return RT_ERR_SCRATCH_TOO_SMALL;
  Carve c(scratch, scratch_bytes);
  uint32_t* keys = c.take<uint32_t>(count);
  void* sort_scratch = c.take<char>(radix_scratch_bytes(count));
  const float3 lo = make_float3(box[0], box[1], box[2]);
  const float3 sc = make_float3(511.0f / fmaxf(box[3] - box[0], 1e-30f), 511.0f / fmaxf(box[4] - box[1], 1e-30f),
                                511.0f / fmaxf(box[5] - box[2], 1e-30f));
  const uint32_t blocks = (uint32_t)hmin<size_t>((count + 255) / 256, (size_t)sms() * 16);
  cudaStream_t st = (cudaStream_t)stream;
  k_ray_keys<<<blocks, 256, 0, st>>>((const float4*)orig, (const float4*)dir, tmax, count, lo, sc, keys, order);
  note_launch();
  RT_CHECK_LAUNCH();
  return radix_sort_pairs(keys, order, count, 0, 24, 0, sort_scratch, radix_scratch_bytes(count), st, nullptr);
}

extern "C" rt_status rt_batch_ray_order_scratch_bytes(uint32_t count, size_t* bytes) { return rt_ray_order_scratch_bytes(count, bytes); }

extern "C" rt_status rt_batch_ray_order(const float* orig, const float* dir, const float* tmax, uint32_t count, const uint32_t* ray_offsets,
                                        uint32_t mesh_count, const float box[6], uint32_t morton_bits, uint32_t* order, void* scratch,
                                        size_t scratch_bytes, rt_stream stream) {
  if (!orig || !dir || !order || !box || !ray_offsets || mesh_count == 0 || mesh_count > (1u << 20)) return RT_ERR_INVALID_ARGUMENT;
  if (morton_bits > 21 || morton_bits % 3) return RT_ERR_INVALID_ARGUMENT;
  uint32_t mesh_bits = 1;
  while ((1u << mesh_bits) <= mesh_count) ++mesh_bits;  // ids 0 .. mesh_count (the inactive rays' id)
  if (mesh_bits + 3 + morton_bits > 32) morton_bits = (29 - mesh_bits) / 3 * 3;  // as many Morton bits as fit in 32
  const uint32_t key_bits = mesh_bits + 3 + morton_bits;
  size_t need = 0;
  rt_ray_order_scratch_bytes(count, &need);
  if (count && (!scratch || scratch_bytes < need)) return RT_ERR_SCRATCH_TOO_SMALL;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (count == 0) return RT_OK;
  Carve c(scratch, scratch_bytes);
  uint32_t* keys = c.take<uint32_t>(count);
  void* sort_scratch = c.take<char>(radix_scratch_bytes(count));
  const float3 lo = make_float3(box[0], box[1], box[2]);
  const float3 sc = make_float3(511.0f / fmaxf(box[3] - box[0], 1e-30f), 511.0f / fmaxf(box[4] - box[1], 1e-30f),
                                511.0f / fmaxf(box[5] - box[2], 1e-30f));
  const uint32_t blocks = (uint32_t)hmin<size_t>((count + 255) / 256, (size_t)sms() * 16);
  cudaStream_t st = (cudaStream_t)stream;
  k_batch_ray_keys<<<blocks, 256, 0, st>>>((const float4*)orig, (const float4*)dir, tmax, count, ray_offsets, mesh_count, morton_bits, lo, sc,
                                           keys, order);
  note_launch();
  RT_CHECK_LAUNCH();
  return radix_sort_pairs(keys, order, count, 0, (key_bits + 7) / 8 * 8, 0, sort_scratch, radix_scratch_bytes(count), st, nullptr);
}

extern "C" rt_status rt_image_tile_order(uint32_t images, uint32_t width, uint32_t height, uint32_t* order, rt_stream stream) {
  if (!order || width == 0 || height == 0 || width % 8 || height % 4) return RT_ERR_INVALID_ARGUMENT;
  const uint64_t total = (uint64_t)images * width * height;
  if (total > 0xFFFFFFFFull) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (total == 0) return RT_OK;
  const uint32_t blocks = (uint32_t)hmin<uint64_t>((total + 255) / 256, (uint64_t)sms() * 16);
  k_image_tile_order<<<blocks, 256, 0, (cudaStream_t)stream>>>((uint32_t)total, width, height, order);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_primary_rays(const rt_camera* cam, uint32_t w, uint32_t h, float* orig, float* dir, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_primary_rays");
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

extern "C" rt_status rt_batch_primary_rays(const float* bases, uint32_t count, uint32_t w, uint32_t h, float* orig, float* dir,
                                           rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_batch_primary_rays");
  if (count == 0) return RT_OK;
  if (!bases || !orig || !dir || w == 0 || h == 0) return RT_ERR_INVALID_ARGUMENT;
  if ((uint64_t)count * w * h > 0xFFFFFFFFull) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  const size_t total = (size_t)count * w * h;
  const uint32_t blocks = (uint32_t)hmin<size_t>((total + 255) / 256, (size_t)sms() * 16);
  k_batch_primary<<<blocks, 256, 0, (cudaStream_t)stream>>>((const float4*)bases, count, w, h, (float4*)orig, (float4*)dir);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_bounce_rays(const float* tris, const float* orig, const float* dir, const int32_t* hit_pos, const float* hit_t,
                                    uint32_t count, uint64_t seed, float* orig_out, float* dir_out, float* tmax_out, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_bounce_rays");
  if (count == 0) return RT_OK;
  if (!tris || !orig || !dir || !hit_pos || !hit_t || !orig_out || !dir_out || !tmax_out) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  const uint32_t blocks = (uint32_t)hmin<size_t>((count + 255) / 256, (size_t)sms() * 16);
  k_bounce<false><<<blocks, 256, 0, (cudaStream_t)stream>>>((const float4*)tris, (const float4*)orig, (const float4*)dir, hit_pos, hit_t,
                                                            count, seed, (float4*)orig_out, (float4*)dir_out, tmax_out, nullptr, nullptr, 0);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_batch_bounce_rays(const float* tris, const uint32_t* face_offsets, const uint32_t* ray_offsets, uint32_t mesh_count,
                                          const float* orig, const float* dir, const int32_t* hit_pos, const float* hit_t, uint32_t count,
                                          uint64_t seed, float* orig_out, float* dir_out, float* tmax_out, uint32_t* order_out,
                                          uint32_t* order_counters, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_batch_bounce_rays");
  if (count == 0) return RT_OK;
  if (!tris || !face_offsets || !ray_offsets || mesh_count == 0 || !orig || !dir || !hit_pos || !hit_t || !orig_out || !dir_out ||
      !tmax_out || (order_out && !order_counters))
    return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (order_out && cudaMemsetAsync(order_counters, 0, 8, (cudaStream_t)stream) != cudaSuccess) return RT_ERR_CUDA;
  const uint32_t blocks = (uint32_t)hmin<size_t>((count + 255) / 256, (size_t)sms() * 16);
  k_bounce<true><<<blocks, 256, 0, (cudaStream_t)stream>>>((const float4*)tris, (const float4*)orig, (const float4*)dir, hit_pos, hit_t,
                                                           count, seed, (float4*)orig_out, (float4*)dir_out, tmax_out, ray_offsets,
                                                           face_offsets, mesh_count);
  note_launch();
  RT_CHECK_LAUNCH();
  if (order_out) {
    const uint32_t runs = (count + kOrderRun - 1) / kOrderRun;
    const uint32_t oblocks = (uint32_t)hmin<size_t>((runs + 7) / 8, (size_t)sms() * 16);
    k_active_first_order<<<oblocks, 256, 0, (cudaStream_t)stream>>>(tmax_out, count, order_out, order_counters);
    note_launch();
    RT_CHECK_LAUNCH();
  }
  return RT_OK;
}

namespace {
template <bool kSeed, bool kWide>
rt_status batch_launch_w(const rt_batch_trace_desc* d, const TraceArgs& A, const BatchTraceArgs& B, const SeedArgs& S, cudaStream_t st,
                         bool count, bool ww) {
  if (d->work_counter && (d->schedule & RT_TRACE_COOP)) {
    if (cudaMemsetAsync(d->work_counter, 0, 4, st) != cudaSuccess) return RT_ERR_CUDA;
    const uint32_t per_sm = d->persistent_blocks_per_sm ? d->persistent_blocks_per_sm : 8u;
    const uint32_t blocks = (uint32_t)hmin<uint64_t>((uint64_t)sms() * per_sm, (d->ray_count + 127) / 128);
    if (count) k_batch_trace_coop<true, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S, d->work_counter);
    else k_batch_trace_coop<false, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S, d->work_counter);
  } else if (d->work_counter) {
    if (cudaMemsetAsync(d->work_counter, 0, 4, st) != cudaSuccess) return RT_ERR_CUDA;
    const uint32_t per_sm = d->persistent_blocks_per_sm ? d->persistent_blocks_per_sm : 8u;
    const uint32_t blocks = (uint32_t)hmin<uint64_t>((uint64_t)sms() * per_sm, (d->ray_count + 127) / 128);
    if (count) {
      if (ww) k_batch_trace_persistent<true, true, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S, d->work_counter);
      else k_batch_trace_persistent<true, false, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S, d->work_counter);
    } else {
      if (ww) k_batch_trace_persistent<false, true, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S, d->work_counter);
      else k_batch_trace_persistent<false, false, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S, d->work_counter);
    }
  } else {
    const uint32_t blocks = (d->ray_count + 127) / 128;
    if (count) {
      if (ww) k_batch_trace<true, true, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S);
      else k_batch_trace<true, false, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S);
    } else {
      if (ww) k_batch_trace<false, true, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S);
      else k_batch_trace<false, false, kSeed, kWide><<<blocks, 128, 0, st>>>(A, B, S);
    }
  }
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

// Bounce rays asked of a batched trace: the packet walk writes them itself; every other schedule (and the seeded
// trace) leaves them to one k_bounce launch after the trace, over the hits it wrote.
bool bounce_fused(const rt_batch_trace_desc* d) {
  return d->bounce_orig && (d->schedule & RT_TRACE_CLUSTERS) && (d->schedule & RT_TRACE_PACKET) && d->work_counter;
}
rt_status bounce_after(const rt_batch_trace_desc* d, bool fused, cudaStream_t st) {
  if (!d->bounce_orig || fused) return RT_OK;
  const uint32_t count = d->ray_count;
  const uint32_t blocks = (uint32_t)hmin<size_t>((count + 255) / 256, (size_t)sms() * 16);
  k_bounce<true><<<blocks, 256, 0, st>>>((const float4*)d->tris, (const float4*)d->orig, (const float4*)d->dir, d->hit_id, d->hit_t,
                                         count, d->bounce_seed, (float4*)d->bounce_orig, (float4*)d->bounce_dir, d->bounce_tmax,
                                         d->ray_offsets, d->face_offsets, d->mesh_count);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

rt_status batch_launch_clusters(const rt_batch_trace_desc* d, const TraceArgs& A, const BatchTraceArgs& B, cudaStream_t st, bool count) {
  const bool ww = (d->schedule & RT_TRACE_WHILE_WHILE) != 0;
  if (d->work_counter) {
    if (cudaMemsetAsync(d->work_counter, 0, 4, st) != cudaSuccess) return RT_ERR_CUDA;
    const uint32_t per_sm = d->persistent_blocks_per_sm ? d->persistent_blocks_per_sm : 8u;
    const uint32_t blocks = (uint32_t)hmin<uint64_t>((uint64_t)sms() * per_sm, ((uint64_t)d->ray_count + 127) / 128);
    if (d->schedule & RT_TRACE_PACKET) {
#define RT_LAUNCH_BCK(CNT, BNC) k_batch_trace_clusters_packet<CNT, BNC><<<blocks, 128, 0, st>>>(A, B, d->work_counter, d->lane_threshold)
      if (A.b_orig) { if (count) RT_LAUNCH_BCK(true, true); else RT_LAUNCH_BCK(false, true); }
      else { if (count) RT_LAUNCH_BCK(true, false); else RT_LAUNCH_BCK(false, false); }
#undef RT_LAUNCH_BCK
    } else if (d->schedule & RT_TRACE_REFILL) {
#define RT_LAUNCH_BCR(CNT, WW) k_batch_trace_clusters_refill<CNT, WW><<<blocks, 128, 0, st>>>(A, B, d->work_counter, d->lane_threshold)
      if (count) { if (ww) RT_LAUNCH_BCR(true, true); else RT_LAUNCH_BCR(true, false); }
      else { if (ww) RT_LAUNCH_BCR(false, true); else RT_LAUNCH_BCR(false, false); }
#undef RT_LAUNCH_BCR
    } else if (d->schedule & RT_TRACE_COOP) {
      if (count) k_batch_trace_clusters_coop<true><<<blocks, 128, 0, st>>>(A, B, d->work_counter);
      else k_batch_trace_clusters_coop<false><<<blocks, 128, 0, st>>>(A, B, d->work_counter);
    } else {
#define RT_LAUNCH_BCP(CNT, WW) k_batch_trace_clusters_persistent<CNT, WW><<<blocks, 128, 0, st>>>(A, B, d->work_counter)
      if (count) { if (ww) RT_LAUNCH_BCP(true, true); else RT_LAUNCH_BCP(true, false); }
      else { if (ww) RT_LAUNCH_BCP(false, true); else RT_LAUNCH_BCP(false, false); }
#undef RT_LAUNCH_BCP
    }
  } else {
    const uint32_t blocks = (d->ray_count + 127) / 128;
#define RT_LAUNCH_BCS(CNT, WW) k_batch_trace_clusters<CNT, WW><<<blocks, 128, 0, st>>>(A, B)
    if (count) { if (ww) RT_LAUNCH_BCS(true, true); else RT_LAUNCH_BCS(true, false); }
    else { if (ww) RT_LAUNCH_BCS(false, true); else RT_LAUNCH_BCS(false, false); }
#undef RT_LAUNCH_BCS
  }
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

template <bool kSeed>
rt_status batch_launch(const rt_batch_trace_desc* d, const SeedArgs& S, cudaStream_t st) {
  TraceArgs A = {};
  A.tris = (const float4*)d->tris; A.indices = d->indices; A.orig = (const float4*)d->orig; A.dir = (const float4*)d->dir;
  A.tmax = d->tmax; A.ray_count = d->ray_count; A.id_mode = d->id_mode; A.hit_id = d->hit_id; A.hit_t = d->hit_t;
  A.hit_uv = (float2*)d->hit_uv; A.visits = d->ray_visits; A.tests = d->ray_tests; A.err = d->error_word;
  if (!kSeed && bounce_fused(d)) {
    A.b_orig = (float4*)d->bounce_orig; A.b_dir = (float4*)d->bounce_dir; A.b_tmax = d->bounce_tmax; A.b_seed = d->bounce_seed;
  }
  BatchTraceArgs B;
  B.M = d->mesh_count; B.foff = d->face_offsets; B.roff = d->ray_offsets; B.order = d->ray_order;
  Carve c((void*)d->accel, ~(size_t)0);
  carve_batch_accel_layout(c, B.acc, d->mesh_count, d->face_count);
  const bool count = d->ray_visits || d->ray_tests;
  const bool ww = (d->schedule & RT_TRACE_WHILE_WHILE) != 0;
  if (d->schedule & RT_TRACE_CLUSTERS) return kSeed ? RT_ERR_UNSUPPORTED : batch_launch_clusters(d, A, B, st, count);
  if (d->schedule & RT_TRACE_WIDE) return batch_launch_w<kSeed, true>(d, A, B, S, st, count, ww);
  return batch_launch_w<kSeed, false>(d, A, B, S, st, count, ww);
}

// Two device ranges [a, a + an) and [b, b + bn) share a byte.
bool ranges_overlap(const void* a, size_t an, const void* b, size_t bn) {
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return a && b && an && bn && x < y + bn && y < x + an;
}

rt_status batch_check(const rt_batch_trace_desc* d) {
  if (!d || d->mesh_count == 0 || !d->face_offsets || !d->ray_offsets || !d->accel || !d->tris || !d->orig || !d->dir ||
      !d->hit_id || !d->hit_t || !d->hit_uv || d->face_count < d->mesh_count)
    return RT_ERR_INVALID_ARGUMENT;
  if (d->id_mode == 1 && !d->indices) return RT_ERR_INVALID_ARGUMENT;
  if (d->ray_count > RT_MAX_RAYS) return RT_ERR_INVALID_ARGUMENT;
  const bool any_bounce = d->bounce_orig || d->bounce_dir || d->bounce_tmax;
  if (any_bounce && (!d->bounce_orig || !d->bounce_dir || !d->bounce_tmax || d->id_mode != 0)) return RT_ERR_INVALID_ARGUMENT;
  if (any_bounce) {  // the bounce rays are written while the call still reads its rays and writes its hits: no shared bytes
    const size_t R = d->ray_count;
    const void* bufs[9] = {d->bounce_orig, d->bounce_dir, d->bounce_tmax, d->orig, d->dir, d->tmax, d->hit_id, d->hit_t, d->hit_uv};
    const size_t bytes[9] = {16 * R, 16 * R, 4 * R, 16 * R, 16 * R, 4 * R, 4 * R, 4 * R, 8 * R};
    for (int i = 0; i < 3; ++i)  // each bounce output against every other buffer of the call
      for (int j = i + 1; j < 9; ++j)
        if (ranges_overlap(bufs[i], bytes[i], bufs[j], bytes[j])) return RT_ERR_INVALID_ARGUMENT;
  }
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  return RT_OK;
}
}  // namespace

extern "C" rt_status rt_batch_trace(const rt_batch_trace_desc* d, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_batch_trace");
  const rt_status s = batch_check(d);
  if (s != RT_OK || d->ray_count == 0) return s;
  const rt_status t = batch_launch<false>(d, SeedArgs{}, (cudaStream_t)stream);
  if (t != RT_OK) return t;
  return bounce_after(d, bounce_fused(d), (cudaStream_t)stream);
}

extern "C" rt_status rt_batch_trace_seeded(const rt_batch_trace_desc* d, const rt_seed_desc* sd, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_batch_trace_seeded");
  const rt_status s = batch_check(d);
  if (s != RT_OK) return s;
  if (!sd || !sd->proposal || !sd->slot_ref) return RT_ERR_INVALID_ARGUMENT;
  if (d->ray_count == 0) return RT_OK;
  SeedArgs S;
  S.proposal = sd->proposal; S.slot_ref = sd->slot_ref; S.slot_box = (const float4*)sd->slot_box; S.slot_count = sd->slot_count;
  S.in_prop = sd->in_proposal;
  const rt_status t = batch_launch<true>(d, S, (cudaStream_t)stream);
  if (t != RT_OK) return t;
  return bounce_after(d, false, (cudaStream_t)stream);
}

namespace {
// Scratch of rt_pack_hits: the block counts (scanned in place into block offsets), then the scan's block sums.
size_t pack_scratch(uint32_t count, uint32_t** counts, uint32_t** sums, void* base) {
  const uint32_t nb = (count + kPackRays - 1) / kPackRays;
  Carve c(base, ~(size_t)0);
  uint32_t* a = c.take<uint32_t>((size_t)nb + 1);
  uint32_t* b = c.take<uint32_t>((size_t)(nb + 1023) / 1024 + 1);
  if (counts) *counts = a;
  if (sums) *sums = b;
  return c.off;
}
}  // namespace

extern "C" rt_status rt_pack_hits_scratch_bytes(uint32_t count, size_t* scratch_bytes) {
  if (!scratch_bytes) return RT_ERR_INVALID_ARGUMENT;
  *scratch_bytes = pack_scratch(count, nullptr, nullptr, nullptr);
  return RT_OK;
}

extern "C" rt_status rt_pack_hits(const int32_t* hit_id, const float* hit_t, const float* hit_uv, uint32_t count, float* packed,
                                  uint32_t* packed_count, void* scratch, size_t scratch_bytes, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_pack_hits");
  if (!packed_count) return RT_ERR_INVALID_ARGUMENT;
  if (count && (!hit_id || !hit_t || !hit_uv || !packed || !scratch)) return RT_ERR_INVALID_ARGUMENT;
  if (count > RT_MAX_RAYS) return RT_ERR_INVALID_ARGUMENT;
  if (count && scratch_bytes < pack_scratch(count, nullptr, nullptr, nullptr)) return RT_ERR_SCRATCH_TOO_SMALL;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  cudaStream_t st = (cudaStream_t)stream;
  if (count == 0) return cudaMemsetAsync(packed_count, 0, 4, st) == cudaSuccess ? RT_OK : RT_ERR_CUDA;
  uint32_t *counts = nullptr, *sums = nullptr;
  pack_scratch(count, &counts, &sums, scratch);
  const uint32_t nb = (count + kPackRays - 1) / kPackRays;
  k_pack_count<<<nb, 256, 0, st>>>(hit_id, count, counts);
  note_launch();
  RT_CHECK_LAUNCH();
  excl_scan(counts, nb, sums, packed_count, st);
  RT_CHECK_LAUNCH();
  k_pack_write<<<nb, 256, 0, st>>>(hit_id, hit_t, (const float2*)hit_uv, count, counts, packed);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}
