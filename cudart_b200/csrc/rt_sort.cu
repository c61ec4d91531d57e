// rt_sort.cu -- stable LSD radix sort of 32-bit keys with optional 32-bit
// values, 8-bit digits, one launch per digit pass (onesweep).
//
// Replaces the reference's sort family (CUDA_radixSortGeneral, CUDA_radixSort,
// CUDA_bitonicSort*, CUDA_bubbleSort512; kernels/CUDA_radixSortGeneral.cu:397-482
// etc.), which serialises its shared histogram 256 ways and ranks keys with
// warp-synchronous code that is undefined on Volta and later. Here:
//   * one histogram launch reads the keys once and counts the digits of every
//     pass (so each pass knows where every digit's run starts);
//   * per pass, one launch over tiles of 4096 keys (512 threads x 8 keys).
//     A CTA takes the next tile index from a counter, ranks its keys stably
//     (the lanes of equal digit found by one ballot per digit bit, plus
//     per-warp counters), publishes its per-digit counts, and finds how many
//     keys of each digit the earlier tiles hold by reading
//     their published counts backwards until it meets a tile that already
//     published its inclusive prefix (decoupled look-back, after Merrill and
//     Adinets, "Onesweep: a faster least significant digit radix sort for
//     GPUs", 2022). It then publishes its own inclusive prefix, stages the
//     tile in shared memory in sorted order and writes it out so that
//     consecutive threads write consecutive addresses of each digit run.
//     Traffic per pass: keys (and values) read once and written once.
//   * n <= 4096: a single CTA does every pass in shared memory (one launch).
// The look-back waits only on tiles whose index was taken earlier, by CTAs that
// were already running and publish their counts before they wait on anything,
// so every wait ends; each is still bounded (an iteration limit, after which
// RT_DEVERR_WAIT_TIMEOUT is OR-ed into the caller's error word and the CTA goes
// on with what it has).
#include "rt_common.cuh"

namespace rt {
namespace {

// single-CTA sort of up to one tile
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096
constexpr int kRadix = 256;

// onesweep passes
constexpr int kOsThreads = 512;
constexpr int kOsWarps = kOsThreads / 32;
constexpr int kOsItems = 8;
constexpr int kOsTile = kOsThreads * kOsItems;  // 4096
static_assert(kOsTile == kTile, "both sorts use 4096-key tiles");
constexpr uint32_t kFlagAggregate = 1u << 30;  // the tile's own count of the digit is published
constexpr uint32_t kFlagPrefix = 2u << 30;     // the count of all keys of the digit up to and including the tile
constexpr uint32_t kCountMask = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 22;      // look-back reads of one status word before giving up (seconds)
constexpr int kMaxPasses = 4;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Block-wide exclusive scan of one value per thread (NT threads).
template <int NT>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
  constexpr int NW = NT / 32;
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
    uint32_t w = lane < NW ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < NW) s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t warp_prefix = warp ? s_warp[warp - 1] : 0u;
  total = s_warp[NW - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

// Digit counts of every pass in one read of the keys: counts[p * 256 + d] = keys whose digit p is d.
__global__ __launch_bounds__(256) void k_sort_hist(const uint32_t* __restrict__ keys, uint32_t n, uint32_t begin_bit, uint32_t passes,
                                                   uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[kMaxPasses][kRadix];
  for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += 256) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint32_t n4 = n >> 2;
  const uint4* k4 = reinterpret_cast<const uint4*>(keys);
  const bool vec = ((uintptr_t)keys & 15u) == 0;
  auto count = [&](uint32_t k) {
    for (uint32_t p = 0; p < passes; ++p) atomicAdd(&h[p][(k >> (begin_bit + 8 * p)) & 255u], 1u);
  };
  if (vec) {
    for (uint32_t i = blockIdx.x * 256 + threadIdx.x; i < n4; i += gridDim.x * 256) {
      const uint4 k = __ldg(k4 + i);
      count(k.x); count(k.y); count(k.z); count(k.w);
    }
    for (uint32_t i = 4 * n4 + blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) count(__ldg(keys + i));
  } else {
    for (uint32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) count(__ldg(keys + i));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (int)passes * kRadix; i += 256) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(counts + i, c);
  }
}

// The lanes of the warp whose 9-bit digit equals this lane's (digits 0..255, 256 for a lane without a key): one
// ballot per bit, each lane keeping the lanes that agree with it on that bit -- the mask __match_any_sync gives.
__device__ __forceinline__ uint32_t match_digit(uint32_t d) {
  uint32_t m = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const bool bit = (d >> b) & 1u;
    const uint32_t v = __ballot_sync(0xffffffffu, bit);
    m &= bit ? v : ~v;
  }
  return m;
}

// Optional epilogue of a pass: out[position] = the segment of the value written there (largest m with
// off[m] <= value, m < count), for a caller that needs each sorted value's segment next.
struct SegOut {
  const uint32_t* off;
  uint32_t count;
  uint32_t* out;
};
__device__ __forceinline__ uint32_t find_seg(const uint32_t* __restrict__ off, uint32_t M, uint32_t x) {
  uint32_t lo = 0, hi = M - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// One digit pass. status[tile * 256 + d] holds a flag (bits 30-31) and a count (bits 0-29); all zero at the start.
// vals_in == nullptr with kVals: the values are the keys' input positions (first pass of an index sort).
template <bool kVals>
__global__ __launch_bounds__(kOsThreads, 3) void k_onesweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                                            uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n,
                                                            uint32_t shift, const uint32_t* __restrict__ digit_counts,
                                                            uint32_t* __restrict__ status, uint32_t* __restrict__ tile_counter,
                                                            uint32_t* __restrict__ digit_totals_out, uint32_t* __restrict__ err,
                                                            SegOut seg) {
  __shared__ uint32_t s_keys[kOsTile];
  __shared__ uint32_t s_vals[kVals ? kOsTile : 1];
  __shared__ uint16_t s_cnt[kOsWarps][kRadix];  // per warp and digit: count, then the warp's offset in the tile's run (<= 4096)
  __shared__ uint32_t s_tile_start[kRadix];
  __shared__ uint32_t s_glob[kRadix];
  __shared__ uint32_t s_warp[kOsWarps];
  __shared__ uint32_t s_tile;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tid = threadIdx.x;
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  for (int i = tid; i < kOsWarps * kRadix; i += kOsThreads) (&s_cnt[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const size_t base = (size_t)tile * kOsTile;

  // stable ranks inside the tile: warp w owns keys [w * 256, w * 256 + 256), 32 consecutive keys per round
  uint32_t key[kOsItems], val[kOsItems], rank[kOsItems];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < kOsItems; ++r) {
    const size_t idx = base + (size_t)warp * (kOsItems * 32) + r * 32 + lane;
    const bool valid = idx < n;
    key[r] = valid ? __ldg(keys_in + idx) : 0u;
    if (kVals) val[r] = valid ? (vals_in ? __ldg(vals_in + idx) : (uint32_t)idx) : 0u;
    const uint32_t d = valid ? ((key[r] >> shift) & 255u) : (uint32_t)kRadix;
    const uint32_t peers = match_digit(d);
    uint32_t pre = 0;
    if (d < (uint32_t)kRadix) pre = s_cnt[warp][d];
    rank[r] = pre + __popc(peers & lt);
    __syncwarp();
    if (d < (uint32_t)kRadix && (peers & lt) == 0) s_cnt[warp][d] = (uint16_t)(pre + __popc(peers));
    __syncwarp();
  }
  __syncthreads();

  // per digit (threads 0..255): warp offsets inside the tile's digit run, the tile's count, published at once
  uint32_t tile_count = 0;
  if (tid < kRadix) {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kOsWarps; ++w) {
      const uint32_t c = s_cnt[w][tid];
      s_cnt[w][tid] = (uint16_t)run;
      run += c;
    }
    tile_count = run;
    st_relaxed(status + (size_t)tile * kRadix + tid, (tile == 0 ? kFlagPrefix : kFlagAggregate) | run);
  }
  uint32_t total;
  const uint32_t start = block_excl_scan<kOsThreads>(tile_count, s_warp, total);
  const uint32_t dc = tid < kRadix ? digit_counts[tid] : 0u;
  const uint32_t dbase = block_excl_scan<kOsThreads>(dc, s_warp, total);
  if (tid < kRadix) {
    s_tile_start[tid] = start;
    // keys of this digit in the tiles before this one: the look-back reads four earlier tiles' words at a time
    // (independent loads, one round trip) and walks them nearest first; a word not yet published is read again
    uint32_t excl = 0, spins = 0;
    for (int64_t j = (int64_t)tile - 1; j >= 0;) {
      uint32_t w4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) w4[q] = (j - q >= 0) ? ld_relaxed(status + (size_t)(j - q) * kRadix + tid) : kFlagPrefix;
      bool done = false;
      int q = 0;
      for (; q < 4; ++q) {
        const uint32_t flag = w4[q] & ~kCountMask;
        if (flag == 0u) break;  // tile j - q has published nothing yet
        excl += w4[q] & kCountMask;
        if (flag == kFlagPrefix) { done = true; break; }
      }
      if (done) break;
      j -= q;
      if (q == 0 && ++spins > kSpinLimit) {
        if (err) atomicOr(err, (uint32_t)RT_DEVERR_WAIT_TIMEOUT);
        break;
      }
    }
    if (tile > 0) st_relaxed(status + (size_t)tile * kRadix + tid, kFlagPrefix | (excl + tile_count));
    s_glob[tid] = dbase + excl;
    if (digit_totals_out && tile == 0) digit_totals_out[tid] = dc;
  }
  __syncthreads();

#pragma unroll
  for (int r = 0; r < kOsItems; ++r) {
    const size_t idx = base + (size_t)warp * (kOsItems * 32) + r * 32 + lane;
    if (idx < n) {
      const uint32_t d = (key[r] >> shift) & 255u;
      const uint32_t pos = s_tile_start[d] + s_cnt[warp][d] + rank[r];
      s_keys[pos] = key[r];
      if (kVals) s_vals[pos] = val[r];
    }
  }
  __syncthreads();
  const uint32_t tile_n = (uint32_t)min((size_t)kOsTile, (size_t)n - base);
  for (uint32_t i = tid; i < tile_n; i += kOsThreads) {
    const uint32_t k = s_keys[i];
    const uint32_t d = (k >> shift) & 255u;
    const size_t out = (size_t)s_glob[d] + (i - s_tile_start[d]);
    keys_out[out] = k;
    if (kVals) {
      vals_out[out] = s_vals[i];
      if (seg.out) seg.out[out] = find_seg(seg.off, seg.count, s_vals[i]);
    }
  }
}

// n <= kTile: every pass in shared memory, one CTA. Dynamic shared memory:
// 2 x kTile keys (+ 2 x kTile values).
template <bool kVals>
__global__ __launch_bounds__(kThreads) void k_radix_small(uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t n,
                                                         uint32_t begin_bit, uint32_t passes, int init_vals,
                                                         uint32_t* __restrict__ digit_totals_out, SegOut seg) {
  extern __shared__ uint32_t dyn[];
  uint32_t* kbuf[2] = {dyn, dyn + kTile};
  uint32_t* vbuf[2] = {dyn + 2 * kTile, dyn + 3 * kTile};
  __shared__ uint32_t s_cnt[kWarps][kRadix + 1];
  __shared__ uint32_t s_tile_start[kRadix];
  __shared__ uint32_t s_warp[kWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt = lanemask_lt();
  for (uint32_t i = threadIdx.x; i < n; i += kThreads) {
    kbuf[0][i] = keys[i];
    if (kVals) vbuf[0][i] = init_vals ? i : vals[i];
  }
  __syncthreads();
  int cur = 0;
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t shift = begin_bit + 8 * p;
    for (int i = threadIdx.x; i < kWarps * (kRadix + 1); i += kThreads) (&s_cnt[0][0])[i] = 0;
    __syncthreads();
    uint32_t rank[kItems];
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
      uint32_t idx = warp * (kItems * 32) + r * 32 + lane;
      uint32_t d = idx < n ? ((kbuf[cur][idx] >> shift) & 255u) : (uint32_t)kRadix;
      uint32_t peers = match_digit(d);
      uint32_t pre = s_cnt[warp][d];
      rank[r] = pre + __popc(peers & lt);
      __syncwarp();
      if ((peers & lt) == 0) s_cnt[warp][d] = pre + __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      uint32_t c = s_cnt[w][threadIdx.x];
      s_cnt[w][threadIdx.x] = run;
      run += c;
    }
    if (digit_totals_out && p + 1 == passes) digit_totals_out[threadIdx.x] = run;
    uint32_t total;
    s_tile_start[threadIdx.x] = block_excl_scan<kThreads>(run, s_warp, total);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
      uint32_t idx = warp * (kItems * 32) + r * 32 + lane;
      if (idx < n) {
        uint32_t k = kbuf[cur][idx];
        uint32_t d = (k >> shift) & 255u;
        uint32_t pos = s_tile_start[d] + s_cnt[warp][d] + rank[r];
        kbuf[cur ^ 1][pos] = k;
        if (kVals) vbuf[cur ^ 1][pos] = vbuf[cur][idx];
      }
    }
    __syncthreads();
    cur ^= 1;
  }
  for (uint32_t i = threadIdx.x; i < n; i += kThreads) {
    keys[i] = kbuf[cur][i];
    if (kVals) {
      vals[i] = vbuf[cur][i];
      if (seg.out) seg.out[i] = find_seg(seg.off, seg.count, vbuf[cur][i]);
    }
  }
}

__global__ void k_iota(uint32_t* v, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

constexpr size_t kSmallSmem = 4 * kTile * sizeof(uint32_t);

// The single-block sort's 64 KB of dynamic shared memory, allowed once per device.
bool small_smem_ready() {
  static PerDeviceOnce once;
  return once.run([] {
    cudaError_t a = cudaFuncSetAttribute(k_radix_small<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem);
    cudaError_t b = cudaFuncSetAttribute(k_radix_small<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem);
    return a == cudaSuccess && b == cudaSuccess;
  });
}

// Scratch regions of an n-key sort (n > one tile), in carve order: the other key and value buffers, then one
// zero-initialised block of every pass's tile status words, tile counters and digit counts.
struct SortLayout {
  uint32_t *kalt, *valt, *status, *counters, *counts;
  size_t zero_bytes;
};
SortLayout carve_sort(Carve& c, uint32_t n) {
  SortLayout L;
  const size_t tiles = (n + kOsTile - 1) / kOsTile;
  L.kalt = c.take<uint32_t>(n);
  L.valt = c.take<uint32_t>(n);
  L.status = c.take<uint32_t>((size_t)kMaxPasses * tiles * kRadix + (size_t)kMaxPasses * 64 + (size_t)kMaxPasses * kRadix);
  L.counters = L.status ? L.status + (size_t)kMaxPasses * tiles * kRadix : nullptr;  // one word per pass, 256 B apart
  L.counts = L.counters ? L.counters + (size_t)kMaxPasses * 64 : nullptr;
  L.zero_bytes = ((size_t)kMaxPasses * tiles * kRadix + (size_t)kMaxPasses * 64 + (size_t)kMaxPasses * kRadix) * 4;
  return L;
}

}  // namespace

size_t radix_scratch_bytes(uint32_t n) {
  if (n <= (uint32_t)kTile) return 256;
  return radix_scratch_bytes_of(n);
}

rt_status radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t begin_bit, uint32_t end_bit, int init_vals,
                           void* scratch, size_t scratch_bytes, cudaStream_t stream, uint32_t* digit_totals_out, uint32_t* err,
                           const uint32_t* digit_counts_in, const uint32_t* seg_off, uint32_t seg_count, uint32_t* seg_out) {
  if (n == 0) return RT_OK;
  if (end_bit <= begin_bit || end_bit > 32) return RT_ERR_INVALID_ARGUMENT;
  if (n > kCountMask) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t passes = (end_bit - begin_bit + 7) / 8;
  if (n <= (uint32_t)kTile) {
    if (!small_smem_ready()) return RT_ERR_CUDA;
    if (vals)
      k_radix_small<true><<<1, kThreads, kSmallSmem, stream>>>(keys, vals, n, begin_bit, passes, init_vals, digit_totals_out,
                                                               SegOut{seg_off, seg_count, (seg_off && seg_count) ? seg_out : nullptr});
    else
      k_radix_small<false><<<1, kThreads, kSmallSmem, stream>>>(keys, nullptr, n, begin_bit, passes, 0, digit_totals_out, SegOut{});
    note_launch();
    RT_CHECK_LAUNCH();
    return RT_OK;
  }
  if (!scratch || scratch_bytes < radix_scratch_bytes(n)) return RT_ERR_SCRATCH_TOO_SMALL;
  const uint32_t tiles = (n + kOsTile - 1) / kOsTile;
  Carve c(scratch, scratch_bytes);
  const SortLayout L = carve_sort(c, n);
  if (!c.ok()) return RT_ERR_SCRATCH_TOO_SMALL;
  if (cudaMemsetAsync(L.status, 0, L.zero_bytes, stream) != cudaSuccess) return RT_ERR_CUDA;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    sms = 148;
  const uint32_t* counts = digit_counts_in;
  if (!counts) {  // one read of the keys for every pass's digit counts, unless the keys' producer counted them
    const uint32_t hist_blocks = (uint32_t)hmin<size_t>((n / 4 + 255) / 256, (size_t)sms * 4);
    k_sort_hist<<<hist_blocks ? hist_blocks : 1, 256, 0, stream>>>(keys, n, begin_bit, passes, L.counts);
    note_launch();
    RT_CHECK_LAUNCH();
    counts = L.counts;
  }
  uint32_t *ks = keys, *vs = vals, *kd = L.kalt, *vd = L.valt;
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t shift = begin_bit + 8 * p;
    uint32_t* st = L.status + (size_t)p * tiles * kRadix;
    uint32_t* ctr = L.counters + (size_t)p * 64;
    const uint32_t* dc = counts + (size_t)p * kRadix;
    uint32_t* dto = p + 1 == passes ? digit_totals_out : nullptr;
    const SegOut seg{seg_off, seg_count, (p + 1 == passes && seg_off && seg_count) ? seg_out : nullptr};
    if (vals)
      k_onesweep<true><<<tiles, kOsThreads, 0, stream>>>(ks, (p == 0 && init_vals) ? nullptr : vs, kd, vd, n, shift, dc, st, ctr, dto, err,
                                                          seg);
    else
      k_onesweep<false><<<tiles, kOsThreads, 0, stream>>>(ks, nullptr, kd, nullptr, n, shift, dc, st, ctr, dto, err, SegOut{});
    note_launch();
    RT_CHECK_LAUNCH();
    uint32_t* t;
    t = ks; ks = kd; kd = t;
    t = vs; vs = vd; vd = t;
  }
  if (ks != keys) {
    if (cudaMemcpyAsync(keys, ks, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream) != cudaSuccess) return RT_ERR_CUDA;
    if (vals && cudaMemcpyAsync(vals, vs, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream) != cudaSuccess) return RT_ERR_CUDA;
  }
  return RT_OK;
}

}  // namespace rt

using namespace rt;

extern "C" rt_status rt_sort_scratch_bytes(uint32_t n, size_t* bytes) {
  if (!bytes) return RT_ERR_INVALID_ARGUMENT;
  *bytes = radix_scratch_bytes(n);
  return RT_OK;
}

static uint32_t bits_of(uint32_t bit_depth) {
  uint32_t bytes = bit_depth == 0 ? 1 : 1 + (bit_depth - 1) / 8;
  return 8 * (bytes > 4 ? 4 : bytes);
}

extern "C" rt_status rt_radix_sort_pairs(uint32_t* keys, uint32_t* values, uint32_t n, uint32_t bit_depth, int init_values,
                                         void* scratch, size_t scratch_bytes, rt_stream stream) {
  const rt::NvtxRange nvtx_range("rt_radix_sort_pairs");
  if (n && (!keys || !values)) return RT_ERR_INVALID_ARGUMENT;
  if (n > (uint32_t)kTile && (!scratch || scratch_bytes < radix_scratch_bytes(n))) return RT_ERR_SCRATCH_TOO_SMALL;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (n == 1 && init_values) {
    k_iota<<<1, 32, 0, (cudaStream_t)stream>>>(values, 1);
    note_launch();
    RT_CHECK_LAUNCH();
    return RT_OK;
  }
  return radix_sort_pairs(keys, values, n, 0, bits_of(bit_depth), init_values, scratch, scratch_bytes, (cudaStream_t)stream, nullptr,
                          nullptr);
}

extern "C" rt_status rt_radix_sort_keys(uint32_t* keys, uint32_t n, uint32_t bit_depth, void* scratch, size_t scratch_bytes, rt_stream stream) {
  if (n && !keys) return RT_ERR_INVALID_ARGUMENT;
  if (n > (uint32_t)kTile && (!scratch || scratch_bytes < radix_scratch_bytes(n))) return RT_ERR_SCRATCH_TOO_SMALL;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  return radix_sort_pairs(keys, nullptr, n, 0, bits_of(bit_depth), 0, scratch, scratch_bytes, (cudaStream_t)stream, nullptr, nullptr);
}
