// rt_clusters.cu -- the cluster tree of the traversal blob (layout in rt_device.cuh).
//
// The node tree of an LBVH build stops at the build's tree depth (12 levels
// by default), so its leaves hold about N / 4096 triangles each: a quarter of
// a million triangles per mesh gives leaves of ~100 triangles, which a walk
// tests in 8-triangle groups. The cluster tree is a second, independent
// traversal tree over the same positions that goes down to leaf_max (4)
// triangles per leaf. Hits never depend on it: the closest hit is the minimum
// (t, position) over all triangles whatever tree prunes the search.
//
// Construction: the binary radix tree of the keys (Morton code << 32 |
// position), which are distinct and sorted, built bottom-up by the
// agglomerative scheme of Apetrei (Fast and Simple Agglomerative LBVH
// Construction, 2014): the boundary between positions b and b + 1 carries the
// value key(b) xor key(b + 1); a node covering positions l .. r merges with the
// neighbour across the flanking boundary of smaller value, and that boundary is
// the index of the parent (the internal node splitting between b and b + 1).
// One thread starts at each position and climbs; at each parent the first of
// the two children to arrive leaves (an atomic exchange on the parent's word
// hands over its far end of the range), the second completes the parent
// (box, 4-wide record) and climbs on, so no thread ever waits.
//
// Three launches keep almost all of that in shared memory:
//   k_cluster_chunk     one CTA per chunk of 512 positions of one mesh: the
//                       climb through the parents whose boundary lies inside
//                       the chunk, in rounds over a compacted list of the
//                       nodes moving up, with shared-memory arrival words,
//                       child references and boxes (every node completed here
//                       has both children inside the chunk), then the records
//                       of those nodes. A node whose parent boundary lies
//                       outside the chunk (at most one per side) is left in the
//                       chunk's frontier; the CTA writes all its arrival words
//                       and, for the next passes, the few nodes they read.
//   k_cluster_frontier  one thread per frontier node: the rest of the climb
//                       through global memory; an arriving child stores its
//                       reference and box in its side of the parent's slots,
//                       then exchanges the parent's word (acquire-release), so
//                       the second arrival reads the sibling's box at once.
//   k_cluster_records   the records of the nodes the frontier pass completed
//                       (each frontier thread lists the nodes it completed).
#include <cuda/atomic>

#include "rt_common.cuh"
#include "rt_device.cuh"

namespace rt {
namespace {

struct ClusterBuild {
  const float4* tris;    // {v0, e1, e2} per position, all meshes
  const uint32_t* codes; // sorted Morton codes per position (mesh-local order)
  const uint32_t* foff;  // batched: face offsets (M + 1 entries); single mesh: nullptr
  uint32_t M;            // meshes (1 for a single mesh)
  uint32_t N;            // positions, all meshes
  uint32_t leaf_max;     // largest cluster
  ClusterTemps T;
  uint32_t* hdr;         // header words, 64 per mesh
  float4* crec;          // records, all meshes
};

__device__ __forceinline__ void mesh_of_chunk(const ClusterBuild& B, uint32_t b, uint32_t& m, uint32_t& F, uint32_t& n, uint32_t& j) {
  if (!B.foff) {
    m = 0; F = 0; n = B.N; j = b;
    return;
  }
  uint32_t lo = 0, hi = B.M - 1;  // largest m with cluster_chunk_base(F_m, m) <= b
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (cluster_chunk_base(__ldg(B.foff + mid), mid) <= b) lo = mid; else hi = mid - 1;
  }
  m = lo;
  F = __ldg(B.foff + m);
  n = __ldg(B.foff + m + 1) - F;
  j = b - cluster_chunk_base(F, m);
}

__device__ __forceinline__ unsigned long long key_xor(uint32_t c0, uint32_t c1, uint32_t b) {
  return ((unsigned long long)(c0 ^ c1) << 32) | (b ^ (b + 1u));
}

__device__ __forceinline__ void tri_box(const float4* tr, float3& mn, float3& mx) {
  const float4 v0 = ldg4(tr), e1 = ldg4(tr + 1), e2 = ldg4(tr + 2);
  const float ax = __fadd_rn(v0.x, e1.x), ay = __fadd_rn(v0.y, e1.y), az = __fadd_rn(v0.z, e1.z);
  const float bx = __fadd_rn(v0.x, e2.x), by = __fadd_rn(v0.y, e2.y), bz = __fadd_rn(v0.z, e2.z);
  mn = make_float3(fminf(v0.x, fminf(ax, bx)), fminf(v0.y, fminf(ay, by)), fminf(v0.z, fminf(az, bz)));
  mx = make_float3(fmaxf(v0.x, fmaxf(ax, bx)), fmaxf(v0.y, fmaxf(ay, by)), fmaxf(v0.z, fmaxf(az, bz)));
  pad_box(mn, mx);
}

// Where a pass reads the child references and child boxes of completed nodes: shared memory for the chunk pass
// (the chunk's positions and inner boundaries), global memory (through L2) for the record pass.
struct SmemNodes {
  const float (*lbox)[kClusterChunk];
  const float (*ibox)[kClusterChunk];
  const uint32_t* child;
  uint32_t s;  // the chunk's first position
  __device__ __forceinline__ void box(uint32_t ref, float3& mn, float3& mx) const {
    const float(*b)[kClusterChunk] = (ref & kClusterLeaf) ? lbox : ibox;
    const uint32_t k = (ref & ~kClusterLeaf) - s;
    mn = make_float3(b[0][k], b[1][k], b[2][k]);
    mx = make_float3(b[3][k], b[4][k], b[5][k]);
  }
  __device__ __forceinline__ uint32_t kid(uint32_t p, uint32_t side) const { return child[2 * (p - s) + side]; }
  __device__ __forceinline__ void kid_box(uint32_t p, uint32_t side, float3& mn, float3& mx) const { box(kid(p, side), mn, mx); }
};
struct GlobalNodes {
  const ClusterTemps* T;
  uint32_t F;
  __device__ __forceinline__ uint32_t kid(uint32_t p, uint32_t side) const { return __ldcg(T->child + 2 * ((size_t)F + p) + side); }
  __device__ __forceinline__ void kid_box(uint32_t p, uint32_t side, float3& mn, float3& mx) const {
    const float4* q = T->cbox + 4 * ((size_t)F + p) + 2 * side;
    const float4 a = __ldcg(q), b = __ldcg(q + 1);
    mn = make_float3(a.x, a.y, a.z);
    mx = make_float3(b.x, b.y, b.z);
  }
};

// The 4-wide record of a completed internal node p (positions l .. r, children l .. p and p + 1 .. r): child 0
// fills slots 0 and 1, child 1 slots 2 and 3 -- a child that is a cluster (at most leaf_max positions) its first
// slot (the second keeps NaN bounds), any other child one slot for each of its two children.
template <class Nodes>
__device__ __forceinline__ void write_record(const ClusterBuild& B, const Nodes& Nd, float4* rec, uint32_t p, uint32_t l, uint32_t r) {
  const float qnan = __int_as_float(0x7fffffff);
  float3 mn[4], mx[4];
  uint32_t ref[4];
  auto child = [&](const int k, uint32_t lo, uint32_t hi) {
    const uint32_t c = Nd.kid(p, (uint32_t)(k >> 1));
    if (hi - lo + 1 <= B.leaf_max) {
      Nd.kid_box(p, (uint32_t)(k >> 1), mn[k], mx[k]);
      ref[k] = cluster_leaf_ref(lo, hi - lo + 1);
      mn[k + 1] = mx[k + 1] = make_float3(qnan, qnan, qnan);
      ref[k + 1] = kNoChild;
    } else {  // an internal node (more than leaf_max >= 1 positions); its split is its own index
      Nd.kid_box(c, 0, mn[k], mx[k]);
      Nd.kid_box(c, 1, mn[k + 1], mx[k + 1]);
      ref[k] = (c - lo + 1 <= B.leaf_max) ? cluster_leaf_ref(lo, c - lo + 1) : Nd.kid(c, 0);
      ref[k + 1] = (hi - c <= B.leaf_max) ? cluster_leaf_ref(c + 1, hi - c) : Nd.kid(c, 1);
    }
  };
  child(0, l, p);
  child(2, p + 1, r);
  rec[0] = make_float4(mn[0].x, mn[1].x, mn[2].x, mn[3].x);
  rec[1] = make_float4(mn[0].y, mn[1].y, mn[2].y, mn[3].y);
  rec[2] = make_float4(mn[0].z, mn[1].z, mn[2].z, mn[3].z);
  rec[3] = make_float4(mx[0].x, mx[1].x, mx[2].x, mx[3].x);
  rec[4] = make_float4(mx[0].y, mx[1].y, mx[2].y, mx[3].y);
  rec[5] = make_float4(mx[0].z, mx[1].z, mx[2].z, mx[3].z);
  rec[6] = make_float4(__uint_as_float(ref[0]), __uint_as_float(ref[1]), __uint_as_float(ref[2]), __uint_as_float(ref[3]));
  rec[7] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// The root (positions 0 .. n - 1, box mn / mx, reference cur) is complete: header words, and a one-slot record
// at index n - 1 when the whole mesh is one cluster.
__device__ __forceinline__ void finish_root(const ClusterBuild& B, uint32_t m, uint32_t F, uint32_t n, uint32_t cur, const float3& mn,
                                            const float3& mx) {
  uint32_t root = cur;
  if (n <= B.leaf_max) {
    const float qnan = __int_as_float(0x7fffffff);
    float4* rec = B.crec + 8 * ((size_t)F + n - 1);
    rec[0] = make_float4(mn.x, qnan, qnan, qnan);
    rec[1] = make_float4(mn.y, qnan, qnan, qnan);
    rec[2] = make_float4(mn.z, qnan, qnan, qnan);
    rec[3] = make_float4(mx.x, qnan, qnan, qnan);
    rec[4] = make_float4(mx.y, qnan, qnan, qnan);
    rec[5] = make_float4(mx.z, qnan, qnan, qnan);
    rec[6] = make_float4(__uint_as_float(cluster_leaf_ref(0, n)), __uint_as_float(kNoChild), __uint_as_float(kNoChild),
                         __uint_as_float(kNoChild));
    rec[7] = make_float4(0.f, 0.f, 0.f, 0.f);
    root = n - 1;
  }
  uint32_t* hdr = B.hdr + 64 * (size_t)m;
  hdr[kHdrClusterN] = n;
  hdr[kHdrClusterRoot] = root;
  __threadfence();
  hdr[kHdrClusterValid] = 1u;
}

// The chunk pass climbs in rounds: the nodes to move up (all positions first) sit in a compacted shared-memory
// list; in a round every listed node arrives at its parent, and the second arrival at a parent completes it
// (range and box, in shared memory) and lists it for the next round, so the threads of a warp work on listed
// nodes side by side. After the last round the CTA writes, with coalesced stores, every position's box, every
// inner boundary's child references, box and arrival word, and the records of the nodes completed here.
__global__ __launch_bounds__(kClusterChunk, 4) void k_cluster_chunk(ClusterBuild B) {
  __shared__ uint32_t s_other[kClusterChunk];
  __shared__ uint32_t s_child[2 * kClusterChunk];
  __shared__ uint32_t s_range[2][kClusterChunk];  // first and last position of a node completed here (else last = 0)
  __shared__ float s_ibox[6][kClusterChunk];
  __shared__ float s_lbox[6][kClusterChunk];
  __shared__ uint32_t s_code[kClusterChunk + 2];  // codes of positions s - 1 .. s + 512
  __shared__ uint32_t s_list[3][kClusterChunk];   // round r reads list r % 3 and fills list (r + 1) % 3
  __shared__ uint32_t s_count[3];
  const uint32_t t = threadIdx.x;
  uint32_t m, F, n, j;
  if (B.foff && B.M <= kClusterChunk) {
    // the chunk's mesh in one step: the number of meshes whose first chunk is at or before this one, less one
    const bool before = t < B.M && cluster_chunk_base(__ldg(B.foff + t), t) <= blockIdx.x;
    m = (uint32_t)__syncthreads_count(before) - 1u;
    F = __ldg(B.foff + m);
    n = __ldg(B.foff + m + 1) - F;
    j = blockIdx.x - cluster_chunk_base(F, m);
  } else {
    mesh_of_chunk(B, blockIdx.x, m, F, n, j);
  }
  const uint32_t s = j * kClusterChunk;
  if (t < 2) B.T.frontier[2 * (size_t)blockIdx.x + t] = make_uint4(0, 0, 0, 0);
  if (s >= n) return;  // a gap in the batched grid (the whole CTA)
  const uint32_t e = min(n, s + kClusterChunk) - 1;  // the chunk's last position; inner boundaries s .. e - 1
  s_other[t] = 0;
  s_range[1][t] = 0;
  for (uint32_t q = t; q < kClusterChunk + 2; q += blockDim.x) {
    const long long pos = (long long)s - 1 + q;
    if (pos >= 0 && pos < (long long)n) s_code[q] = __ldg(B.codes + F + pos);
  }
  const uint32_t i = s + t;
  if (i <= e) {
    float3 mn, mx;
    tri_box(B.tris + 3 * ((size_t)F + i), mn, mx);
    s_lbox[0][t] = mn.x; s_lbox[1][t] = mn.y; s_lbox[2][t] = mn.z; s_lbox[3][t] = mx.x; s_lbox[4][t] = mx.y; s_lbox[5][t] = mx.z;
    s_list[0][t] = kClusterLeaf | i;
  }
  if (t == 0) {
    s_count[0] = e - s + 1;
    s_count[1] = 0;
  }
  __syncthreads();
  const SmemNodes Nd{s_lbox, s_ibox, s_child, s};
  for (uint32_t round = 0;; ++round) {
    // one barrier per round: the list after next (read two rounds ago) is emptied during this round
    const uint32_t cb = round % 3u, nb = (round + 1u) % 3u;
    const uint32_t count = s_count[cb];
    if (count == 0) break;
    if (t < count) {
      const uint32_t cur = s_list[cb][t];
      uint32_t l, r;
      if (cur & kClusterLeaf) {
        l = r = cur & ~kClusterLeaf;
      } else {
        l = s_range[0][cur - s];
        r = s_range[1][cur - s];
      }
      if (l == 0 && r == n - 1) {
        float3 mn, mx;
        Nd.box(cur, mn, mx);
        finish_root(B, m, F, n, cur, mn, mx);
      } else {
        // boundary b's codes are s_code[b - s + 1] and s_code[b - s + 2] (b in s - 1 .. e)
        const bool left_child = (l == 0) || (r != n - 1 && key_xor(s_code[r - s + 1], s_code[r - s + 2], r) <
                                                             key_xor(s_code[l - s], s_code[l - s + 1], l - 1));
        const uint32_t p = left_child ? r : l - 1;
        if (p < s || p >= e) {  // the parent's boundary is not inside the chunk: the frontier pass goes on from here
          B.T.frontier[2 * (size_t)blockIdx.x + (p < s ? 0 : 1)] = make_uint4(cur, l, r, 1u);
        } else {
          const uint32_t k = p - s;
          s_child[2 * k + (left_child ? 0u : 1u)] = cur;
          __threadfence_block();
          const uint32_t old = atomicExch(s_other + k, (left_child ? l : r) + 1u);
          if (old != 0) {  // second arrival: this thread completes the parent
            __threadfence_block();
            if (left_child) r = old - 1u; else l = old - 1u;
            float3 amn, amx, bmn, bmx;
            Nd.box(s_child[2 * k], amn, amx);
            Nd.box(s_child[2 * k + 1], bmn, bmx);
            s_ibox[0][k] = fminf(amn.x, bmn.x); s_ibox[1][k] = fminf(amn.y, bmn.y); s_ibox[2][k] = fminf(amn.z, bmn.z);
            s_ibox[3][k] = fmaxf(amx.x, bmx.x); s_ibox[4][k] = fmaxf(amx.y, bmx.y); s_ibox[5][k] = fmaxf(amx.z, bmx.z);
            s_range[0][k] = l;
            s_range[1][k] = r;
            // append to the next list, one shared-memory atomic per warp
            const uint32_t am = __activemask();
            const uint32_t lane = t & 31u, leader = __ffs(am) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(s_count + nb, (uint32_t)__popc(am));
            base = __shfl_sync(am, base, leader);
            s_list[nb][base + __popc(am & ((1u << lane) - 1u))] = p;
          }
        }
      }
    }
    if (t == 0) s_count[(round + 2u) % 3u] = 0;
    __syncthreads();
  }
  // Write-out. Every boundary's arrival word (coalesced; e's is zero: its children are never both inside one chunk),
  // the record of each node completed here with more than leaf_max positions, and
  // for the global pass and its records the nodes they read: the frontier nodes and the first child to arrive at
  // each parent still pending, each with its box and, when internal, its child references and their boxes.
  auto put_box = [&](float4* dst, uint32_t ref) {
    float3 mn, mx;
    Nd.box(ref, mn, mx);
    dst[0] = make_float4(mn.x, mn.y, mn.z, 0.f);
    dst[1] = make_float4(mx.x, mx.y, mx.z, 0.f);
  };
  auto export_kids = [&](uint32_t ref) {
    if (ref & kClusterLeaf) return;
    const uint32_t k0 = Nd.kid(ref, 0), k1 = Nd.kid(ref, 1);
    *(uint2*)(B.T.child + 2 * ((size_t)F + ref)) = make_uint2(k0, k1);
    put_box(B.T.cbox + 4 * ((size_t)F + ref), k0);
    put_box(B.T.cbox + 4 * ((size_t)F + ref) + 2, k1);
  };
  if (i < e) {
    const uint32_t word = s_other[t];
    B.T.other[(size_t)F + i] = word;
    const uint32_t l = s_range[0][t], r = s_range[1][t];
    if (r != 0) {
      if (r - l + 1 > B.leaf_max) write_record(B, Nd, B.crec + 8 * ((size_t)F + i), i, l, r);
    } else if (word != 0) {  // one child arrived: a left child stored its first position (<= i), a right one its last
      const uint32_t side = (word - 1u <= i) ? 0u : 1u;
      const uint32_t c = s_child[2 * t + side];
      B.T.child[2 * ((size_t)F + i) + side] = c;
      put_box(B.T.cbox + 4 * ((size_t)F + i) + 2 * side, c);
      export_kids(c);
    }
  } else if (i == e && i + 1 < n) {
    B.T.other[(size_t)F + i] = 0u;
  }
  if (t < 2) {
    const uint4 fr = B.T.frontier[2 * (size_t)blockIdx.x + t];
    if (fr.w) {
      put_box(B.T.fbox + 4 * (size_t)blockIdx.x + 2 * t, fr.x);
      export_kids(fr.x);
    }
  }
}

// The rest of the climb, from the frontier nodes, through global memory. Each arriving child stores its
// reference and box in its side of the parent's slots, then exchanges the parent's arrival word with
// acquire-release order at device scope; the second arrival reads the sibling's box, completes the parent and
// marks it (its range) for k_cluster_records.
__global__ __launch_bounds__(128) void k_cluster_frontier(ClusterBuild B) {
  const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= 2 * cluster_chunks(B.N, B.M)) return;
  const uint4 fr = B.T.frontier[f];
  if (fr.w == 0) {
    B.T.chain[(size_t)f * (kClusterChain + 1) + kClusterChain] = 0;
    return;
  }
  uint32_t m, F, n, j;
  mesh_of_chunk(B, f >> 1, m, F, n, j);
  const uint32_t* codes = B.codes + F;
  uint32_t cur = fr.x, l = fr.y, r = fr.z;
  const float4 b0 = B.T.fbox[2 * (size_t)f], b1 = B.T.fbox[2 * (size_t)f + 1];
  float3 mn = make_float3(b0.x, b0.y, b0.z), mx = make_float3(b1.x, b1.y, b1.z);
  uint32_t* chain = B.T.chain + (size_t)f * (kClusterChain + 1);
  uint32_t done = 0;  // nodes completed by this climb (listed in chain for k_cluster_records)
  for (;;) {
    if (l == 0 && r == n - 1) {
      finish_root(B, m, F, n, cur, mn, mx);
      break;
    }
    const bool left_child = (l == 0) || (r != n - 1 && key_xor(__ldg(codes + r), __ldg(codes + r + 1), r) <
                                                         key_xor(__ldg(codes + l - 1), __ldg(codes + l), l - 1));
    const uint32_t p = left_child ? r : l - 1;
    const uint32_t side = left_child ? 0u : 1u;
    float4* slot = B.T.cbox + 4 * ((size_t)F + p);
    B.T.child[2 * ((size_t)F + p) + side] = cur;
    slot[2 * side] = make_float4(mn.x, mn.y, mn.z, 0.f);
    slot[2 * side + 1] = make_float4(mx.x, mx.y, mx.z, 0.f);
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> word(B.T.other[(size_t)F + p]);
    const uint32_t old = word.exchange((left_child ? l : r) + 1u, cuda::memory_order_acq_rel);
    if (old == 0) break;  // the sibling completes the parent
    if (left_child) r = old - 1u; else l = old - 1u;
    const float4 s0 = __ldcg(slot + 2 * (1 - side)), s1 = __ldcg(slot + 2 * (1 - side) + 1);
    mn = make_float3(fminf(mn.x, s0.x), fminf(mn.y, s0.y), fminf(mn.z, s0.z));
    mx = make_float3(fmaxf(mx.x, s1.x), fmaxf(mx.y, s1.y), fmaxf(mx.z, s1.z));
    B.T.prange[(size_t)F + p] = make_uint2(l, r + 1u);
    if (done < kClusterChain) chain[done++] = p;
    cur = p;
  }
  chain[kClusterChain] = done;
}

// Records of the nodes the frontier pass completed: one warp per frontier node, a lane per node of its climb.
__global__ __launch_bounds__(256) void k_cluster_records(ClusterBuild B) {
  const uint32_t f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
  if (f >= 2 * cluster_chunks(B.N, B.M)) return;
  const uint32_t* chain = B.T.chain + (size_t)f * (kClusterChain + 1);
  const uint32_t done = chain[kClusterChain];
  if (done == 0) return;
  uint32_t m, F, n, j;
  mesh_of_chunk(B, f >> 1, m, F, n, j);
  for (uint32_t k = lane; k < done; k += 32) {
    const uint32_t p = chain[k];
    const uint2 pr = B.T.prange[(size_t)F + p];
    const uint32_t l = pr.x, r = pr.y - 1u;
    if (r - l + 1 > B.leaf_max) write_record(B, GlobalNodes{&B.T, F}, B.crec + 8 * ((size_t)F + p), p, l, r);
  }
}

}  // namespace

rt_status build_cluster_tree(const float4* tris, const uint32_t* codes, uint32_t n, uint32_t leaf_max, const ClusterTemps& T,
                             uint32_t* hdr, float4* crec, cudaStream_t st) {
  return batch_build_cluster_tree(tris, codes, nullptr, 1, n, leaf_max, T, hdr, crec, st);
}

rt_status batch_build_cluster_tree(const float4* tris, const uint32_t* codes, const uint32_t* foff, uint32_t M, uint32_t N,
                                   uint32_t leaf_max, const ClusterTemps& T, uint32_t* hdr, float4* crec, cudaStream_t st) {
  if (N == 0) return RT_OK;
  if (N > kClusterFirstMask || leaf_max < 1 || leaf_max > kClusterLeafMax) return RT_ERR_UNSUPPORTED;
  ClusterBuild B;
  B.tris = tris; B.codes = codes; B.foff = foff; B.M = M; B.N = N; B.leaf_max = leaf_max; B.T = T; B.hdr = hdr; B.crec = crec;
  const uint32_t chunks = cluster_chunks(N, M);
  k_cluster_chunk<<<chunks, kClusterChunk, 0, st>>>(B);
  k_cluster_frontier<<<(2 * chunks + 127) / 128, 128, 0, st>>>(B);
  k_cluster_records<<<(2 * chunks * 32 + 255) / 256, 256, 0, st>>>(B);
  note_launch(3);
  RT_CHECK_LAUNCH();
  return RT_OK;
}

}  // namespace rt
