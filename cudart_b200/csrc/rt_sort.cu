// rt_sort.cu -- stable LSD radix sort of 32-bit keys with optional 32-bit
// values, 8-bit digits.
//
// Replaces the reference's sort family (CUDA_radixSortGeneral, CUDA_radixSort,
// CUDA_bitonicSort*, CUDA_bubbleSort512; kernels/CUDA_radixSortGeneral.cu:397-482
// etc.), which serialises its shared histogram 256 ways and ranks keys with
// warp-synchronous code that is undefined on Volta and later. Here:
//   * tiles of 4096 keys (256 threads x 16 keys);
//   * per pass: tile digit histograms (shared atomics), one CTA per digit to
//     scan its row of tile counts, then a scatter kernel that ranks keys
//     stably inside the tile with __match_any_sync + per-warp counters,
//     stages the tile in shared memory in sorted order and writes it out so
//     that consecutive threads write consecutive addresses of each digit run;
//   * n <= 4096: a single CTA does every pass in shared memory (one launch).
// No kernel waits on another CTA, so nothing here can spin.
#include "rt_common.cuh"

namespace rt {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096
constexpr int kRadix = 256;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Block-wide exclusive scan of one value per thread (kThreads threads).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
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
    uint32_t w = lane < kWarps ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kWarps) s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t warp_prefix = warp ? s_warp[warp - 1] : 0u;
  total = s_warp[kWarps - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

__global__ __launch_bounds__(kThreads) void k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n, uint32_t shift,
                                                        uint32_t num_tiles, uint32_t* __restrict__ tile_hist) {
  __shared__ uint32_t h[kRadix];
  h[threadIdx.x] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kTile;
#pragma unroll 4
  for (int i = threadIdx.x; i < kTile; i += kThreads) {
    size_t idx = base + i;
    if (idx < n) atomicAdd(&h[(__ldg(keys + idx) >> shift) & 255u], 1u);
  }
  __syncthreads();
  tile_hist[(size_t)threadIdx.x * num_tiles + blockIdx.x] = h[threadIdx.x];
}

// One CTA per digit: exclusive scan of that digit's tile counts in place.
__global__ __launch_bounds__(kThreads) void k_radix_scan_digit(uint32_t* __restrict__ tile_hist, uint32_t num_tiles,
                                                              uint32_t* __restrict__ digit_totals) {
  __shared__ uint32_t s_warp[kWarps];
  uint32_t* row = tile_hist + (size_t)blockIdx.x * num_tiles;
  uint32_t running = 0;
  for (uint32_t c = 0; c < num_tiles; c += kThreads) {
    uint32_t i = c + threadIdx.x;
    uint32_t v = i < num_tiles ? row[i] : 0u;
    uint32_t total;
    uint32_t ex = block_excl_scan(v, s_warp, total);
    if (i < num_tiles) row[i] = running + ex;
    running += total;
  }
  if (threadIdx.x == 0) digit_totals[blockIdx.x] = running;
}

// Ranks the tile's keys stably (warp w owns keys [w*512, w*512+512) of the
// tile, 32 consecutive keys per round), then scatters.
template <bool kVals>
__global__ __launch_bounds__(kThreads) void k_radix_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                                                           uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n,
                                                           uint32_t shift, uint32_t num_tiles, const uint32_t* __restrict__ tile_off,
                                                           const uint32_t* __restrict__ digit_totals) {
  __shared__ uint32_t s_keys[kTile];
  __shared__ uint32_t s_vals[kVals ? kTile : 1];
  __shared__ uint32_t s_cnt[kWarps][kRadix + 1];
  __shared__ uint32_t s_tile_start[kRadix];
  __shared__ uint32_t s_glob[kRadix];
  __shared__ uint32_t s_warp[kWarps];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kWarps * (kRadix + 1); i += kThreads) (&s_cnt[0][0])[i] = 0;
  __syncthreads();

  const size_t base = (size_t)blockIdx.x * kTile;
  uint32_t key[kItems], val[kItems], rank[kItems];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    size_t idx = base + (size_t)warp * (kItems * 32) + r * 32 + lane;
    bool valid = idx < n;
    key[r] = valid ? __ldg(keys_in + idx) : 0u;
    if (kVals) val[r] = valid ? (vals_in ? __ldg(vals_in + idx) : (uint32_t)idx) : 0u;
    uint32_t d = valid ? ((key[r] >> shift) & 255u) : (uint32_t)kRadix;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t pre = s_cnt[warp][d];
    rank[r] = pre + __popc(peers & lt);
    __syncwarp();
    if ((peers & lt) == 0) s_cnt[warp][d] = pre + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // per digit: offsets of each warp's run inside the tile's digit run
  uint32_t tile_count = 0;
  {
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      uint32_t c = s_cnt[w][d];
      s_cnt[w][d] = run;
      run += c;
    }
    tile_count = run;
  }
  uint32_t total;
  uint32_t start = block_excl_scan(tile_count, s_warp, total);
  s_tile_start[threadIdx.x] = start;
  uint32_t dg = digit_totals[threadIdx.x];
  uint32_t gex = block_excl_scan(dg, s_warp, total);
  s_glob[threadIdx.x] = gex + tile_off[(size_t)threadIdx.x * num_tiles + blockIdx.x];
  __syncthreads();

#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    size_t idx = base + (size_t)warp * (kItems * 32) + r * 32 + lane;
    if (idx < n) {
      uint32_t d = (key[r] >> shift) & 255u;
      uint32_t pos = s_tile_start[d] + s_cnt[warp][d] + rank[r];
      s_keys[pos] = key[r];
      if (kVals) s_vals[pos] = val[r];
    }
  }
  __syncthreads();
  const uint32_t tile_n = (uint32_t)min((size_t)kTile, (size_t)n - base);
  for (uint32_t i = threadIdx.x; i < tile_n; i += kThreads) {
    uint32_t k = s_keys[i];
    uint32_t d = (k >> shift) & 255u;
    size_t out = (size_t)s_glob[d] + (i - s_tile_start[d]);
    keys_out[out] = k;
    if (kVals) vals_out[out] = s_vals[i];
  }
}

// n <= kTile: every pass in shared memory, one CTA. Dynamic shared memory:
// 2 x kTile keys (+ 2 x kTile values).
template <bool kVals>
__global__ __launch_bounds__(kThreads) void k_radix_small(uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t n,
                                                         uint32_t begin_bit, uint32_t passes, int init_vals,
                                                         uint32_t* __restrict__ digit_totals_out) {
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
      uint32_t peers = __match_any_sync(0xffffffffu, d);
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
    s_tile_start[threadIdx.x] = block_excl_scan(run, s_warp, total);
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
    if (kVals) vals[i] = vbuf[cur][i];
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

}  // namespace

size_t radix_scratch_bytes(uint32_t n) {
  if (n <= (uint32_t)kTile) return 256;
  size_t tiles = (n + kTile - 1) / kTile;
  Carve c(nullptr, 0);
  c.take<uint32_t>(n);
  c.take<uint32_t>(n);
  c.take<uint32_t>(tiles * kRadix);
  c.take<uint32_t>(kRadix);
  return c.off + 256;
}

rt_status radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t begin_bit, uint32_t end_bit, int init_vals,
                           void* scratch, size_t scratch_bytes, cudaStream_t stream, uint32_t* digit_totals_out) {
  if (n == 0) return RT_OK;
  if (end_bit <= begin_bit || end_bit > 32) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t passes = (end_bit - begin_bit + 7) / 8;
  if (n <= (uint32_t)kTile) {
    if (!small_smem_ready()) return RT_ERR_CUDA;
    if (vals)
      k_radix_small<true><<<1, kThreads, kSmallSmem, stream>>>(keys, vals, n, begin_bit, passes, init_vals, digit_totals_out);
    else
      k_radix_small<false><<<1, kThreads, kSmallSmem, stream>>>(keys, nullptr, n, begin_bit, passes, 0, digit_totals_out);
    note_launch();
    RT_CHECK_LAUNCH();
    return RT_OK;
  }
  if (!scratch || scratch_bytes < radix_scratch_bytes(n)) return RT_ERR_SCRATCH_TOO_SMALL;
  const uint32_t tiles = (n + kTile - 1) / kTile;
  Carve c(scratch, scratch_bytes);
  uint32_t* kalt = c.take<uint32_t>(n);
  uint32_t* valt = c.take<uint32_t>(n);
  uint32_t* hist = c.take<uint32_t>((size_t)tiles * kRadix);
  uint32_t* totals = c.take<uint32_t>(kRadix);
  uint32_t *ks = keys, *vs = vals, *kd = kalt, *vd = valt;
  bool first = true;
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t shift = begin_bit + 8 * p;
    k_radix_hist<<<tiles, kThreads, 0, stream>>>(ks, n, shift, tiles, hist);
    k_radix_scan_digit<<<kRadix, kThreads, 0, stream>>>(hist, tiles, p + 1 == passes && digit_totals_out ? digit_totals_out : totals);
    const uint32_t* tot = p + 1 == passes && digit_totals_out ? digit_totals_out : totals;
    if (vals)
      k_radix_scatter<true><<<tiles, kThreads, 0, stream>>>(ks, (first && init_vals) ? nullptr : vs, kd, vd, n, shift, tiles, hist, tot);
    else
      k_radix_scatter<false><<<tiles, kThreads, 0, stream>>>(ks, nullptr, kd, nullptr, n, shift, tiles, hist, tot);
    note_launch(3);
    RT_CHECK_LAUNCH();
    first = false;
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
  if (n && (!keys || !values)) return RT_ERR_INVALID_ARGUMENT;
  if (n > (uint32_t)kTile && (!scratch || scratch_bytes < radix_scratch_bytes(n))) return RT_ERR_SCRATCH_TOO_SMALL;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (n == 1 && init_values) {
    k_iota<<<1, 32, 0, (cudaStream_t)stream>>>(values, 1);
    note_launch();
    RT_CHECK_LAUNCH();
    return RT_OK;
  }
  return radix_sort_pairs(keys, values, n, 0, bits_of(bit_depth), init_values, scratch, scratch_bytes, (cudaStream_t)stream, nullptr);
}

extern "C" rt_status rt_radix_sort_keys(uint32_t* keys, uint32_t n, uint32_t bit_depth, void* scratch, size_t scratch_bytes, rt_stream stream) {
  if (n && !keys) return RT_ERR_INVALID_ARGUMENT;
  if (n > (uint32_t)kTile && (!scratch || scratch_bytes < radix_scratch_bytes(n))) return RT_ERR_SCRATCH_TOO_SMALL;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  return radix_sort_pairs(keys, nullptr, n, 0, bits_of(bit_depth), 0, scratch, scratch_bytes, (cudaStream_t)stream, nullptr);
}
