// rt_scan.cu -- device-wide exclusive scan of 32-bit words, shared by the
// SAH build and the rasteriser: 1024-word blocks scanned in shared memory, the
// block sums scanned by one CTA, then added back.
#include "rt_device.cuh"

namespace rt {
namespace {
// Exclusive scan of n words in place; block sums in `sums` (>= ceil(n / 1024) + 1 words).
__global__ __launch_bounds__(256) void k_scan_blocks(uint32_t* v, uint32_t n, uint32_t* sums) {
  __shared__ uint32_t s_w[8];
  const uint32_t base = blockIdx.x * 1024u + threadIdx.x * 4u;
  uint32_t a[4], t = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) { a[k] = base + k < n ? v[base + k] : 0u; t += a[k]; }
  uint32_t total;
  uint32_t ex = block_excl_scan_nt<256>(t, s_w, total);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (base + k < n) v[base + k] = ex;
    ex += a[k];
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ __launch_bounds__(1024) void k_scan_sums(uint32_t* sums, uint32_t nb, uint32_t* total_out) {
  __shared__ uint32_t s_w[32];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < nb; b0 += 1024) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t x = i < nb ? sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_excl_scan_nt<1024>(x, s_w, total);
    const uint32_t carry = s_carry;
    if (i < nb) sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + total;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total_out) *total_out = s_carry;
}
__global__ __launch_bounds__(256) void k_scan_add(uint32_t* v, uint32_t n, const uint32_t* sums) {
  const uint32_t add = sums[blockIdx.x];
  const uint32_t base = blockIdx.x * 1024u + threadIdx.x * 4u;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (base + k < n) v[base + k] += add;
}
}  // namespace

void excl_scan(uint32_t* v, uint32_t n, uint32_t* sums, uint32_t* total, cudaStream_t st) {
  const uint32_t nb = (n + 1023) / 1024;
  k_scan_blocks<<<nb, 256, 0, st>>>(v, n, sums);
  k_scan_sums<<<1, 1024, 0, st>>>(sums, nb, total);
  k_scan_add<<<nb, 256, 0, st>>>(v, n, sums);
  note_launch(3);
}


}  // namespace rt
