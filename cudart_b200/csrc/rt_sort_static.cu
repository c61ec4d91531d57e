// rt_sort_static.cu -- an allocation-free variant of rt_radix_sort_pairs.
//
// Some callers cannot allocate device memory at the point where they sort:
// plug-ins whose host application owns every device allocation (a renderer or
// game engine with a fixed memory budget hands them only the buffers they
// work on), and frame loops that cannot afford cudaMalloc/cudaFree, which may
// synchronize the whole device. rt_radix_sort_pairs needs a scratch buffer from
// its caller; this entry point instead uses a scratch array that lives in the
// library itself, as a file-scope __device__ array: every GPU that loads the
// library holds RT_STATIC_SORT_SCRATCH_BYTES of device memory for it until the
// process exits, and no call allocates anything.
//
// Set-up: the array's name, used in host code, is a host-side stand-in and not
// a device address, so the first call on each device (with that device
// current) asks the runtime for the address with cudaGetSymbolAddress and
// caches it per device. That first call should come before any stream capture.
//
// Sharing: all calls (all streams, all threads) use the same array, which keeps
// whatever the previous call left in it. Each sort first zeroes the part that
// must start at zero (the tiles' status words, the tile counters and the digit
// counts) and writes every other word before reading it (the ping-pong key and
// value buffers), so a call never sees the previous call's contents. Two calls that overlap
// on the GPU (different streams, or host threads without ordering) race on the
// array and corrupt each other's results; callers must serialize them.
#include <mutex>

#include "rt_common.cuh"

namespace {

constexpr uint32_t kMaxN = RT_STATIC_SORT_MAX_N;
constexpr size_t kScratchBytes = RT_STATIC_SORT_SCRATCH_BYTES;
static_assert(kScratchBytes >= rt::radix_scratch_bytes_of(kMaxN), "static scratch too small for RT_STATIC_SORT_MAX_N keys");

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

rt_status scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RT_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return RT_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return RT_ERR_CUDA;
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return RT_OK;
}

}  // namespace

extern "C" rt_status rt_radix_sort_pairs_static(uint32_t* keys, uint32_t* values, uint32_t n, uint32_t bit_depth, int init_values,
                                                rt_stream stream) {
  if (n && (!keys || !values)) return RT_ERR_INVALID_ARGUMENT;
  if (n > kMaxN) return RT_ERR_CAPACITY;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (n == 0) return RT_OK;
  void* scratch = nullptr;
  rt_status s = scratch_address(&scratch);
  if (s != RT_OK) return s;
  uint32_t bytes = bit_depth == 0 ? 1 : 1 + (bit_depth - 1) / 8;
  if (bytes > 4) bytes = 4;
  if (n == 1) {
    // one key: only the value may need setting
    if (init_values && cudaMemsetAsync(values, 0, 4, (cudaStream_t)stream) != cudaSuccess) return RT_ERR_CUDA;
    return RT_OK;
  }
  return rt::radix_sort_pairs(keys, values, n, 0, 8 * bytes, init_values, scratch, kScratchBytes, (cudaStream_t)stream, nullptr);
}
