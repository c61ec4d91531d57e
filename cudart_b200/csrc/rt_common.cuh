// rt_common.cuh -- shared device helpers for the LBVH build and traversal.
//
// Floating-point work that must match the reference bit for bit is compiled
// with -fmad=false (no FMA contraction), IEEE division and square root
// (nvcc's defaults -prec-div=true / -prec-sqrt=true), and min/max written as
// the selects of the reference's host helpers (types/_cuda_float.h:11-19).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <mutex>

#include "../../include/rt_core.h"

namespace rt {

constexpr float kHuge = 3.402823466e+38f;  // CUDART_NORM_HUGE_F
constexpr uint32_t kMinLeafDefault = 16;   // kernels/CUDA_buildMeshTreeLBVH.cu:39
constexpr uint32_t kMaxLeafDefault = 224;  // kernels/CUDA_buildMeshTreeLBVH.cu:40

__device__ __forceinline__ float fmin_sel(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmax_sel(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float4 f4min(float4 a, float4 b) {
  return make_float4(fmin_sel(a.x, b.x), fmin_sel(a.y, b.y), fmin_sel(a.z, b.z), fmin_sel(a.w, b.w));
}
__device__ __forceinline__ float4 f4max(float4 a, float4 b) {
  return make_float4(fmax_sel(a.x, b.x), fmax_sel(a.y, b.y), fmax_sel(a.z, b.z), fmax_sel(a.w, b.w));
}

// 128-bit read-only loads (ld.global.nc.v4) for data that no kernel writes
// while the reading kernel runs.
__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ uint4 ldg4(const uint4* p) { return __ldg(p); }
// Two consecutive float4 in one 32-byte read-only load (256-bit, sm_100); p must be 32-byte aligned.
__device__ __forceinline__ void ldg8(const float4* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// A named host range around an entry point, for profilers that read NVTX ranges (the header-only NVTX3 API does
// nothing unless a tool attaches).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
template <typename T>
inline T hmin(T a, T b) { return a < b ? a : b; }

// Bump allocator over a caller-provided scratch buffer.
struct Carve {
  char* base;
  size_t off = 0;
  size_t cap;
  Carve(void* p, size_t c) : base((char*)p), cap(c) {}
  template <typename T>
  T* take(size_t count) {
    off = align_up(off, 256);
    T* p = (T*)(base ? base + off : nullptr);
    off += count * sizeof(T);
    return p;
  }
  bool ok() const { return off <= cap; }
};

inline rt_status cuda_status(cudaError_t e) { return e == cudaSuccess ? RT_OK : RT_ERR_CUDA; }

#define RT_CHECK_LAUNCH()                                   \
  do {                                                      \
    cudaError_t _e = cudaGetLastError();                    \
    if (_e != cudaSuccess) return RT_ERR_CUDA;              \
  } while (0)

// A host-side set-up step (cudaFuncSetAttribute, a device query) that holds per device: `run` calls `fn` the
// first time it is reached with a given device current, remembers whether it succeeded, and answers from
// that record afterwards. Threads that race on the first call meet at the mutex; later calls only load an atomic.
struct PerDeviceOnce {
  static constexpr int kMaxDevices = 64;
  std::atomic<int> state[kMaxDevices];  // 0 not yet, 1 done, -1 failed (static storage: zero-initialized)
  std::mutex mu;
  template <typename F>
  bool run(F&& fn) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return false;
    int s = state[dev].load(std::memory_order_acquire);
    if (s == 0) {
      std::lock_guard<std::mutex> lock(mu);
      s = state[dev].load(std::memory_order_relaxed);
      if (s == 0) {
        s = fn() ? 1 : -1;
        state[dev].store(s, std::memory_order_release);
      }
    }
    return s == 1;
  }
};

// A side stream and two events for this host thread and the current device: a call forks an independent part of
// its work onto the side stream and joins it back (event record, stream wait: stream capture turns that into two
// parallel branches). Created on first use; nullptr when CUDA refuses (the caller then runs both parts in order).
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
SideStream* side_stream();

// Number of kernels this library has launched (process-wide); exported as
// rt_launch_count() so that a caller can count the kernels inside a timed region.
void note_launch(uint32_t kernels = 1);

// Exclusive scan of n words in place (rt_scan.cu); `sums` holds >= n / 1024 + 2
// words; `total` (device, optional) receives the sum of all n words.
void excl_scan(uint32_t* v, uint32_t n, uint32_t* sums, uint32_t* total, cudaStream_t st);

// Radix sort internals shared by the build (rt_sort.cu).
// Scratch bytes of an n-key sort (n > 4096 keys; n <= 4096 needs none): the other key and value buffers, and
// per digit pass (at most 4) one status word per (4096-key tile, digit), a tile counter and 256 digit counts;
// each region starts on a 256-byte boundary, plus 256 bytes of slack. radix_scratch_bytes() returns this.
constexpr size_t radix_scratch_bytes_of(uint32_t n) {
  const size_t tiles = ((size_t)n + 4095) / 4096;
  const size_t a = ((size_t)n * 4 + 255) / 256 * 256;
  return 2 * a + 4 * (4 * tiles * 256 + 4 * 64 + 4 * 256) + 256;
}
size_t radix_scratch_bytes(uint32_t n);
// Stable sort of (key, value) pairs by bits [begin_bit, end_bit) of the key; digit_totals_out (device, 256 words,
// optional) receives the digit counts of the last pass; err (device, optional) receives RT_DEVERR_WAIT_TIMEOUT
// if a bounded wait between tiles ran out. digit_counts_in (device, optional): the digit counts of every pass
// (pass p's 256 counts at p * 256, digit p = bits [begin_bit + 8p, begin_bit + 8p + 8)), counted by the keys'
// producer; the sort then reads the keys once less. seg_off / seg_count / seg_out (optional, with values):
// the last pass also writes seg_out[position] = the segment of the value placed there (the largest m < seg_count
// with seg_off[m] <= value).
rt_status radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t begin_bit, uint32_t end_bit, int init_vals,
                           void* scratch, size_t scratch_bytes, cudaStream_t stream, uint32_t* digit_totals_out,
                           uint32_t* err = nullptr, const uint32_t* digit_counts_in = nullptr, const uint32_t* seg_off = nullptr,
                           uint32_t seg_count = 0, uint32_t* seg_out = nullptr);

}  // namespace rt
