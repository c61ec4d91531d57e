// rt_mlp.cu -- tensor-core kernels of the learned subtree proposal.
//
// The proposal network maps a ray (origin, direction) to one of 2^depth BVH
// subtrees: 6 inputs -> 12-frequency sin/cos encoding (144 features, padded
// with zeros to 192) -> 3 hidden layers of 128 (ReLU) -> 4096 logits. Weights
// are BF16 in [out][in] layout (K-major for the tensor cores), accumulation is
// FP32 in tensor memory, biases and the optimizer state are FP32.
//
// Kernels:
//   k_gemm_tc         C = alpha * A B^T (+ bias, ReLU, ReLU' mask) with FP32 /
//                     BF16 / transposed-BF16 outputs; one 128 x BN tile per CTA;
//                     TMA loads through a 4-stage ring, one thread issues
//                     tcgen05.mma, the accumulator lives in TMEM.
//   k_gemm_argmax_tc  one CTA owns 128 rows and sweeps all N columns in tiles
//                     of 256 with two TMEM accumulators (MMA of tile t+1
//                     overlaps the argmax epilogue of tile t); the logits never
//                     reach HBM.
//   k_ray_features, k_softmax_xent, k_transpose_bf16, k_colsum_bf16, k_adam.
// The reference has no learned component; none of this replaces reference code.
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "../../include/rt_propose.h"
#include "rt_tc.cuh"

namespace rt {
namespace {
using namespace tc;

constexpr uint32_t kBM = 128, kBK = 64, kStages = 4;
constexpr uint32_t kTileA = kBM * kBK * 2;  // 16 KB per A stage

// Four bf16 values as one 8-byte word, the first at the lowest address (an 8-byte store writes them in order).
__device__ __forceinline__ uint2 pack_bf16x4(__nv_bfloat16 a, __nv_bfloat16 b, __nv_bfloat16 c, __nv_bfloat16 d) {
  return make_uint2((uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16),
                    (uint32_t)__bfloat16_as_ushort(c) | ((uint32_t)__bfloat16_as_ushort(d) << 16));
}

int num_sms() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

struct GemmEpi {
  float alpha;
  const float* bias;
  uint32_t relu;
  const __nv_bfloat16* mask;
  uint32_t ldmask;
  float* c32;
  uint32_t ldc32;
  __nv_bfloat16* c16;
  uint32_t ldc16;
  __nv_bfloat16* ct16;
  uint32_t ldct;
  uint32_t gm, gn;  // rows and columns of one group's product
  uint32_t c32_v8, c16_v8;  // the output's 16-column pieces are 32-byte aligned: 256-bit stores
};

// One 32-byte store (256-bit, sm_100); p must be 32-byte aligned.
__device__ __forceinline__ void st_global_v8(void* p, const uint32_t (&w)[8]) {
  asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]),
               "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7])
               : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *(const uint32_t*)&h;
}

// row: stacked row of A / C; col: column inside group g's product.
__device__ __forceinline__ void epilogue16(const GemmEpi& E, uint32_t g, uint32_t row, uint32_t col, float (&v)[16]) {
  const float* bias = E.bias ? E.bias + (size_t)g * E.gn : nullptr;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    float x = v[i] * E.alpha;
    if (bias) x += __ldg(bias + col + i);
    if (E.relu) x = fmaxf(x, 0.0f);
    v[i] = x;
  }
  if (E.mask) {
    const uint4* mp = (const uint4*)(E.mask + (size_t)row * E.ldmask + col);
    const uint4 m0 = __ldg(mp), m1 = __ldg(mp + 1);
    const uint32_t w[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      // a BF16 value is > 0 when its sign bit is clear and it is not +0 (ReLU outputs hold no NaN)
      const uint32_t lo = w[i] & 0xFFFFu, hi = w[i] >> 16;
      if (!(lo != 0u && !(lo & 0x8000u))) v[2 * i] = 0.0f;
      if (!(hi != 0u && !(hi & 0x8000u))) v[2 * i + 1] = 0.0f;
    }
  }
  if (E.c32) {
    float* p = E.c32 + (size_t)row * E.ldc32 + col;
    if (E.c32_v8) {
      uint32_t a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) { a[i] = __float_as_uint(v[i]); b[i] = __float_as_uint(v[8 + i]); }
      st_global_v8(p, a);
      st_global_v8(p + 8, b);
    } else {
      float4* q = (float4*)p;
#pragma unroll
      for (int i = 0; i < 4; ++i) q[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
  }
  if (E.c16) {
    const uint32_t w[8] = {pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]),
                           pack_bf16(v[8], v[9]), pack_bf16(v[10], v[11]), pack_bf16(v[12], v[13]), pack_bf16(v[14], v[15])};
    __nv_bfloat16* p = E.c16 + (size_t)row * E.ldc16 + col;
    if (E.c16_v8) {
      st_global_v8(p, w);
    } else {
      uint4* q = (uint4*)p;
      q[0] = make_uint4(w[0], w[1], w[2], w[3]);
      q[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
  }
  if (E.ct16) {
    __nv_bfloat16* ct = E.ct16 + (size_t)g * E.gn * E.ldct + (row - g * E.gm);
#pragma unroll
    for (int i = 0; i < 16; ++i) ct[(size_t)(col + i) * E.ldct] = __float2bfloat16_rn(v[i]);
  }
}

// ----------------------------------------------------------------------------
// Generic GEMM: grid (n / bn, m / 128, groups), 128 threads. Warp 0 lane 0 loads
// (TMA) through a ring of `stages` stages (no more than the K chunks, so that a
// short-K GEMM leaves room for more CTAs per SM), warp 1 lane 0 issues the
// MMAs, then all four warps drain TMEM.
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 1)
    k_gemm_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmEpi E, uint32_t bn,
              uint32_t tmem_cols, uint32_t num_k, uint32_t stages, uint32_t* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t tile_b = bn * 128u;
  uint8_t* sA = smem;
  uint8_t* sB = smem + stages * kTileA;
  uint64_t* full = (uint64_t*)(sB + stages * tile_b);
  uint64_t* empty = full + stages;
  uint64_t* done = empty + stages;
  uint32_t* tmem_slot = (uint32_t*)(done + 1);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < stages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(done, 1);
    fence_mbar_init();
    prefetch_tmap(&ta);
    prefetch_tmap(&tb);
  }
  __syncwarp();
  if (warp == 0) {
    tmem_alloc(tmem_slot, tmem_cols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t g = blockIdx.z;
  const int32_t m0 = (int32_t)(g * E.gm + blockIdx.y * kBM), n0 = (int32_t)(blockIdx.x * bn);

  if (warp == 0 && lane == 0) {
    const int32_t b0 = (int32_t)(g * E.gn) + n0;
    uint32_t kc = 0;
    for (; kc < num_k; ++kc) {
      const uint32_t s = kc % stages;
      if (kc >= stages && !mbar_wait(empty + s, ((kc / stages) - 1u) & 1u, err)) break;
      mbar_arrive_expect_tx(full + s, kTileA + tile_b);
      tma_load_2d(sA + s * kTileA, &ta, (int32_t)(kc * kBK), m0, full + s);
      tma_load_2d(sB + s * tile_b, &tb, (int32_t)(kc * kBK), b0, full + s);
    }
    // the latest load of each stage has landed before the CTA may exit
    for (uint32_t j = kc > stages ? kc - stages : 0u; j < kc; ++j) mbar_wait(full + j % stages, (j / stages) & 1u, err);
  } else if (warp == 1 && lane == 0) {
    const uint32_t idesc = idesc_bf16_f32(kBM, bn);
    for (uint32_t kc = 0; kc < num_k; ++kc) {
      const uint32_t s = kc % stages;
      if (!mbar_wait(full + s, (kc / stages) & 1u, err)) break;
      tc_fence_after();
      const uint32_t a = smem_u32(sA + s * kTileA), b = smem_u32(sB + s * tile_b);
#pragma unroll
      for (uint32_t kk = 0; kk < kBK / 16; ++kk)
        mma_bf16(tmem, desc_sw128(a + kk * 32u), desc_sw128(b + kk * 32u), idesc, (kc | kk) != 0u);
      mma_commit(empty + s);
    }
    mma_commit(done);  // arrives once every MMA issued above has completed
  }
  __syncwarp();

  // warp-uniform, so that tcgen05.ld (.sync.aligned) runs on whole warps
  const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0, err));
  tc_fence_after();
  if (ok) {
    const uint32_t row = (uint32_t)m0 + warp * 32u + lane;
    const uint32_t tl = tmem + ((warp * 32u) << 16);
    for (uint32_t c = 0; c < bn; c += 16) {
      float v[16];
      tmem_ld16(tl + c, v);
      epilogue16(E, g, row, (uint32_t)n0 + c, v);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, tmem_cols);
}

// ----------------------------------------------------------------------------
// Row argmax of A B^T + bias: grid (m / 128, groups), 320 threads. Warps 0-7 drain TMEM
// (warp w reads lanes 32 (w % 4) .. + 31 and the column half w / 4 of each
// tile), warp 8 loads, warp 9 issues MMAs. A (128 rows x k, k <= 256) stays in
// shared memory; B tiles of 256 rows x 64 stream through the ring;
// accumulators alternate between TMEM columns [0, 256) and [256, 512). Each
// thread keeps four independent (max, index, runner-up) chains (columns
// i % 4) so that the compare chain does not serialize the epilogue.
// ----------------------------------------------------------------------------
constexpr uint32_t kArgBN = 256;
constexpr uint32_t kArgTileB = kArgBN * 128u;  // 32 KB
constexpr uint32_t kArgMaxN = 4096;
constexpr uint32_t kArgThreads = 320;

struct Top2 {
  float best, second;
  int32_t idx;
};
// Merge two partial results: the larger maximum wins (the lower index on equal
// maxima); the runner-up is the larger of the winner's runner-up and the
// loser's maximum.
__device__ __forceinline__ Top2 top2_merge(Top2 a, Top2 b) {
  const bool b_wins = b.best > a.best || (b.best == a.best && b.idx >= 0 && (a.idx < 0 || b.idx < a.idx));
  Top2 r;
  if (b_wins) {
    r.best = b.best; r.idx = b.idx; r.second = fmaxf(b.second, a.best);
  } else {
    r.best = a.best; r.idx = a.idx; r.second = fmaxf(a.second, b.best);
  }
  return r;
}

__global__ void __launch_bounds__(kArgThreads, 1)
    k_gemm_argmax_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const float* __restrict__ bias,
                     uint32_t n, uint32_t gm, uint32_t num_k, float min_margin, int32_t* __restrict__ out_idx,
                     float* __restrict__ out_val, float* __restrict__ out_margin, uint32_t* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = smem;                        // num_k x 16 KB
  uint8_t* sB = smem + num_k * kTileA;       // kStages x 32 KB
  float* s_bias = (float*)(sB + kStages * kArgTileB);  // n floats
  Top2* s_half = (Top2*)(s_bias + n);                  // 128 partial results of the upper column half
  uint64_t* full = (uint64_t*)(s_half + kBM);
  uint64_t* empty = full + kStages;
  uint64_t* a_full = empty + kStages;
  uint64_t* acc_full = a_full + 1;   // [2]
  uint64_t* acc_empty = acc_full + 2;  // [2]
  uint64_t* mdone = acc_empty + 2;
  uint32_t* tmem_slot = (uint32_t*)(mdone + 1);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t grp = blockIdx.y;
  for (uint32_t j = threadIdx.x; j < n; j += kArgThreads) s_bias[j] = bias ? bias[(size_t)grp * n + j] : 0.0f;
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < kStages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(a_full, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + b, 1);
      mbar_init(acc_empty + b, 256);
    }
    mbar_init(mdone, 1);
    fence_mbar_init();
    prefetch_tmap(&ta);
    prefetch_tmap(&tb);
  }
  __syncwarp();
  if (warp == 0) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int32_t m0 = (int32_t)(grp * gm + blockIdx.x * kBM);
  const uint32_t ntiles = n / kArgBN;
  Top2 res = {-INFINITY, -INFINITY, -1};
  bool ok = true;

  if (warp == 8) {
    if (lane == 0) {
      mbar_arrive_expect_tx(a_full, num_k * kTileA);
      for (uint32_t kc = 0; kc < num_k; ++kc) tma_load_2d(sA + kc * kTileA, &ta, (int32_t)(kc * kBK), m0, a_full);
      const uint32_t total = ntiles * num_k;
      uint32_t g = 0;
      for (; g < total; ++g) {
        const uint32_t s = g % kStages;
        if (g >= kStages && !mbar_wait(empty + s, ((g / kStages) - 1u) & 1u, err)) break;
        const uint32_t t = g / num_k, kc = g % num_k;
        mbar_arrive_expect_tx(full + s, kArgTileB);
        tma_load_2d(sB + s * kArgTileB, &tb, (int32_t)(kc * kBK), (int32_t)(grp * n + t * kArgBN), full + s);
      }
      // the A block and the latest load of each stage have landed before the CTA may exit
      mbar_wait(a_full, 0, err);
      for (uint32_t j = g > kStages ? g - kStages : 0u; j < g; ++j) mbar_wait(full + j % kStages, (j / kStages) & 1u, err);
    }
  } else if (warp == 9) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(kBM, kArgBN);
      bool mok = mbar_wait(a_full, 0, err);
      uint32_t g = 0;
      for (uint32_t t = 0; mok && t < ntiles; ++t) {
        const uint32_t buf = t & 1u;
        if (t >= 2 && !mbar_wait(acc_empty + buf, ((t >> 1) - 1u) & 1u, err)) break;
        tc_fence_after();
        const uint32_t d = tmem + buf * kArgBN;
        for (uint32_t kc = 0; kc < num_k; ++kc, ++g) {
          const uint32_t s = g % kStages;
          if (!mbar_wait(full + s, (g / kStages) & 1u, err)) { mok = false; break; }
          tc_fence_after();
          const uint32_t a = smem_u32(sA + kc * kTileA), b = smem_u32(sB + s * kArgTileB);
#pragma unroll
          for (uint32_t kk = 0; kk < kBK / 16; ++kk)
            mma_bf16(d, desc_sw128(a + kk * 32u), desc_sw128(b + kk * 32u), idesc, (kc | kk) != 0u);
          mma_commit(empty + s);
        }
        mma_commit(acc_full + buf);
      }
      mma_commit(mdone);  // every MMA issued above has completed before TMEM is released
      mbar_wait(mdone, 0, err);
    }
  } else {
    // epilogue warps 0-7: lane quarter warp % 4, column half warp / 4
    const uint32_t q = warp & 3u, half = warp >> 2;
    float bk[4], sk[4];
    int32_t ik[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) { bk[k] = -INFINITY; sk[k] = -INFINITY; ik[k] = -1; }
    for (uint32_t t = 0; t < ntiles; ++t) {
      const uint32_t buf = t & 1u;
      ok = __all_sync(0xffffffffu, ok && mbar_wait(acc_full + buf, (t >> 1) & 1u, err));
      tc_fence_after();
      if (ok) {
        const uint32_t c0 = half * (kArgBN / 2);
        const uint32_t tl = tmem + ((q * 32u) << 16) + buf * kArgBN + c0;
        for (uint32_t c = 0; c < kArgBN / 2; c += 16) {
          float v[16];
          tmem_ld16(tl + c, v);
          const uint32_t col = t * kArgBN + c0 + c;
          const float4* bp = (const float4*)(s_bias + col);
#pragma unroll
          for (int i4 = 0; i4 < 4; ++i4) {
            const float4 b4 = bp[i4];
            const float bb[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const float x = v[4 * i4 + k] + bb[k];
              sk[k] = fmaxf(sk[k], fminf(x, bk[k]));
              if (x > bk[k]) { bk[k] = x; ik[k] = (int32_t)(col + 4 * i4 + k); }
            }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(acc_empty + buf);
    }
    res = Top2{bk[0], sk[0], ik[0]};
#pragma unroll
    for (int k = 1; k < 4; ++k) res = top2_merge(res, Top2{bk[k], sk[k], ik[k]});
    if (half == 1) s_half[q * 32u + lane] = res;
  }
  __syncthreads();
  if (warp < 4) {
    const uint32_t r = warp * 32u + lane;
    res = top2_merge(res, s_half[r]);
    const uint32_t row = (uint32_t)m0 + r;
    const float margin = res.best - res.second;
    out_idx[row] = (ok && margin >= min_margin) ? res.idx : -1;
    if (out_val) out_val[row] = res.best;
    if (out_margin) out_margin[row] = margin;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ----------------------------------------------------------------------------
// Logits + softmax cross-entropy gradient: grid (m / 128, groups), 576 threads:
// warps 0-15 drain TMEM (warp w: lane quarter w % 4, column quarter w / 4 of
// each 256-wide logit tile), warp 16 loads, warp 17 issues the MMAs. The
// logits of a 128-row block are computed twice, never stored: pass 1 keeps
// each row's running max and sum of exponentials (per column quarter, merged
// in a fixed order through shared memory); pass 2 writes g = (softmax -
// onehot(label)) * scale in BF16, row-major and transposed, and adds the row's
// loss scale * (log sum - logit[label]). Rows whose label is outside [0, n)
// get g = 0 and no loss.
constexpr uint32_t kXentThreads = 576;
// ----------------------------------------------------------------------------
struct XentArgs {
  const float* bias;
  const int32_t* labels;
  uint32_t n, gm;
  float scale;
  __nv_bfloat16* g;
  uint32_t ldg;
  __nv_bfloat16* gt;
  uint32_t ldgt;
  float* loss_sum;
  uint32_t* err;
  uint32_t g32;  // g and ldg keep every 16-column piece of a row 32-byte aligned: one 256-bit store per piece
};

size_t xent_smem(uint32_t num_k, uint32_t n) {
  return 1024 + num_k * (size_t)kTileA + kStages * (size_t)kArgTileB + (size_t)n * 4 + 3 * kBM * 16 + 16 * 8 + 64;
}

__global__ void __launch_bounds__(kXentThreads, 1)
    k_gemm_xent_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, XentArgs X, uint32_t num_k) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = smem;
  uint8_t* sB = smem + num_k * kTileA;
  float* s_bias = (float*)(sB + kStages * kArgTileB);
  float4* s_x = (float4*)(s_bias + X.n);  // [3][128]: (max, sum, logit[label], -) of column quarters 1..3
  uint64_t* full = (uint64_t*)(s_x + 3 * kBM);
  uint64_t* empty = full + kStages;
  uint64_t* a_full = empty + kStages;
  uint64_t* acc_full = a_full + 1;     // [2]
  uint64_t* acc_empty = acc_full + 2;  // [2]
  uint64_t* xch_a = acc_empty + 2;
  uint64_t* xch_b = xch_a + 1;
  uint64_t* mdone = xch_b + 1;
  uint32_t* tmem_slot = (uint32_t*)(mdone + 1);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t grp = blockIdx.y, n = X.n;
  for (uint32_t j = threadIdx.x; j < n; j += kXentThreads) s_bias[j] = X.bias ? X.bias[(size_t)grp * n + j] : 0.0f;
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < kStages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(a_full, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + b, 1);
      mbar_init(acc_empty + b, 512);
    }
    mbar_init(xch_a, 3 * 128);
    mbar_init(xch_b, 128);
    mbar_init(mdone, 1);
    fence_mbar_init();
    prefetch_tmap(&ta);
    prefetch_tmap(&tb);
  }
  __syncwarp();
  if (warp == 0) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int32_t m0 = (int32_t)(grp * X.gm + blockIdx.x * kBM);
  const uint32_t ntiles = n / kArgBN, total_tiles = 2 * ntiles;

  if (warp == 16) {
    if (lane == 0) {
      mbar_arrive_expect_tx(a_full, num_k * kTileA);
      for (uint32_t kc = 0; kc < num_k; ++kc) tma_load_2d(sA + kc * kTileA, &ta, (int32_t)(kc * kBK), m0, a_full);
      const uint32_t total = total_tiles * num_k;
      uint32_t q = 0;
      for (; q < total; ++q) {
        const uint32_t s = q % kStages;
        if (q >= kStages && !mbar_wait(empty + s, ((q / kStages) - 1u) & 1u, X.err)) break;
        const uint32_t t = (q / num_k) % ntiles, kc = q % num_k;
        mbar_arrive_expect_tx(full + s, kArgTileB);
        tma_load_2d(sB + s * kArgTileB, &tb, (int32_t)(kc * kBK), (int32_t)(grp * n + t * kArgBN), full + s);
      }
      // the latest load of each stage (and A) has landed before the CTA may exit
      mbar_wait(a_full, 0, X.err);
      for (uint32_t j = q > kStages ? q - kStages : 0u; j < q; ++j) mbar_wait(full + j % kStages, (j / kStages) & 1u, X.err);
    }
  } else if (warp == 17) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(kBM, kArgBN);
      bool mok = mbar_wait(a_full, 0, X.err);
      uint32_t q = 0;
      for (uint32_t t = 0; mok && t < total_tiles; ++t) {
        const uint32_t buf = t & 1u;
        if (t >= 2 && !mbar_wait(acc_empty + buf, ((t >> 1) - 1u) & 1u, X.err)) break;
        tc_fence_after();
        const uint32_t d = tmem + buf * kArgBN;
        for (uint32_t kc = 0; kc < num_k; ++kc, ++q) {
          const uint32_t s = q % kStages;
          if (!mbar_wait(full + s, (q / kStages) & 1u, X.err)) { mok = false; break; }
          tc_fence_after();
          const uint32_t a = smem_u32(sA + kc * kTileA), b = smem_u32(sB + s * kArgTileB);
#pragma unroll
          for (uint32_t kk = 0; kk < kBK / 16; ++kk)
            mma_bf16(d, desc_sw128(a + kk * 32u), desc_sw128(b + kk * 32u), idesc, (kc | kk) != 0u);
          mma_commit(empty + s);
        }
        if (mok) mma_commit(acc_full + buf);
      }
      mma_commit(mdone);  // every MMA issued above has completed before TMEM is released
      mbar_wait(mdone, 0, X.err);
    }
  } else {
    const uint32_t qw = warp & 3u, cq = warp >> 2;
    const uint32_t trow = qw * 32u + lane, row = (uint32_t)m0 + trow, rowl = blockIdx.x * kBM + trow;
    const int32_t lab = X.labels[row];
    const bool valid = lab >= 0 && lab < (int32_t)n;
    const uint32_t c0 = cq * (kArgBN / 4);
    float mx = -INFINITY, sum = 0.0f, xl = 0.0f, inv = 0.0f;
    bool ok = true;
    for (uint32_t t2 = 0; t2 < total_tiles; ++t2) {
      const uint32_t buf = t2 & 1u, pass = t2 / ntiles, t = t2 - pass * ntiles;
      if (t2 == ntiles && ok) {
        // merge the four column quarters of each row (quarter 0 merges 1, 2, 3 in that order) and share the result
        if (cq > 0) {
          s_x[(cq - 1u) * kBM + trow] = make_float4(mx, sum, xl, 0.0f);
          mbar_arrive(xch_a);
          ok = __all_sync(0xffffffffu, mbar_wait(xch_b, 0, X.err));
          const float4 w = s_x[trow];
          mx = w.x; sum = w.y;
        } else {
          ok = __all_sync(0xffffffffu, mbar_wait(xch_a, 0, X.err));
#pragma unroll
          for (uint32_t j = 0; j < 3; ++j) {
            const float4 w = s_x[j * kBM + trow];
            const float m2 = fmaxf(mx, w.x);
            sum = sum * __expf(mx - m2) + w.y * __expf(w.x - m2);
            mx = m2;
            xl += w.z;  // exactly one quarter saw the label's column; the others hold 0
          }
          // every partial has been read above: slot 0 now carries the merged row
          s_x[trow] = make_float4(mx, sum, 0.0f, 0.0f);
          mbar_arrive(xch_b);
          if (valid && X.loss_sum) atomicAdd(X.loss_sum, (logf(sum) + mx - xl) * X.scale);
        }
        inv = 1.0f / sum;
      }
      ok = ok && __all_sync(0xffffffffu, mbar_wait(acc_full + buf, (t2 >> 1) & 1u, X.err));
      tc_fence_after();
      if (ok) {
        const uint32_t tl = tmem + ((qw * 32u) << 16) + buf * kArgBN + c0;
        for (uint32_t c = 0; c < kArgBN / 4; c += 16) {
          float v[16];
          tmem_ld16(tl + c, v);
          const uint32_t col = t * kArgBN + c0 + c;
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] += s_bias[col + i];
          if (pass == 0) {
            float cm = v[0];
#pragma unroll
            for (int i = 1; i < 16; ++i) cm = fmaxf(cm, v[i]);
            if (cm > mx) {
              sum *= __expf(mx - cm);
              mx = cm;
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              sum += __expf(v[i] - mx);
              if ((int32_t)(col + i) == lab) xl = v[i];
            }
          } else {
            uint32_t w[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              float p0 = __expf(v[2 * i] - mx) * inv, p1 = __expf(v[2 * i + 1] - mx) * inv;
              if ((int32_t)(col + 2 * i) == lab) p0 -= 1.0f;
              if ((int32_t)(col + 2 * i + 1) == lab) p1 -= 1.0f;
              w[i] = valid ? pack_bf16(p0 * X.scale, p1 * X.scale) : 0u;
            }
            __nv_bfloat16* gr = X.g + (size_t)row * X.ldg + col;
            if (X.g32) {
              st_global_v8(gr, w);
            } else {
              uint4* gp = (uint4*)gr;
              gp[0] = make_uint4(w[0], w[1], w[2], w[3]);
              gp[1] = make_uint4(w[4], w[5], w[6], w[7]);
            }
            __nv_bfloat16* gt = X.gt + ((size_t)grp * n + col) * X.ldgt + rowl;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              gt[(size_t)(2 * i) * X.ldgt] = __ushort_as_bfloat16((unsigned short)(w[i] & 0xFFFFu));
              gt[(size_t)(2 * i + 1) * X.ldgt] = __ushort_as_bfloat16((unsigned short)(w[i] >> 16));
            }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(acc_empty + buf);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ----------------------------------------------------------------------------
// Small kernels
// ----------------------------------------------------------------------------
// The six network inputs of a ray: the origin scaled to [-1, 1] over the box
// (component i < 3), the unit direction (component i < 3 of dir_input).
__device__ __forceinline__ float origin_input(const float4& o, float3 c, float3 s, uint32_t i) {
  return i == 0 ? (o.x - c.x) * s.x : (i == 1 ? (o.y - c.y) * s.y : (o.z - c.z) * s.z);
}
__device__ __forceinline__ float dir_input(const float4& d, uint32_t i) {
  const float len = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  const float inv = len > 0.0f ? 1.0f / len : 0.0f;
  return (i == 0 ? d.x : (i == 1 ? d.y : d.z)) * inv;
}
// w[j] = BF16 pair (sin(pi 2^j x), cos(pi 2^j x)), j < 12.
__device__ __forceinline__ void encode12(float x, uint32_t (&w)[12]) {
#pragma unroll
  for (int j = 0; j < 12; ++j) {
    float sv, cv;
    sincospif(x, &sv, &cv);
    w[j] = pack_bf16(sv, cv);
    x *= 2.0f;
  }
}

// Features of one ray: u = ((o - c) * s, d / |d|); f[24 i + 2 j] = sin(pi 2^j u_i),
// f[24 i + 2 j + 1] = cos(pi 2^j u_i) for j < 12; columns 144..191 are zero
// (rows hold ld >= 192 elements). Eight threads per ray: thread i < 6 encodes input i (48 bytes), threads 6
// and 7 write the zero padding, so a warp stores 4 whole 384-byte rows.
// out_t: one [192][group_rows] transpose per group of group_rows rays.
__global__ __launch_bounds__(256) void k_ray_features(const float4* __restrict__ orig, const float4* __restrict__ dir, uint32_t count,
                                                      float3 c, float3 s, __nv_bfloat16* __restrict__ out, uint32_t ld,
                                                      __nv_bfloat16* __restrict__ out_t, uint32_t ld_t, uint32_t group_rows) {
  const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t r = gid >> 3, i = gid & 7u;
  if (r >= count) return;
  uint32_t w[12];
  if (i < 6) {
    encode12(i < 3 ? origin_input(__ldg(orig + r), c, s, i) : dir_input(__ldg(dir + r), i - 3), w);
  } else {
#pragma unroll
    for (int j = 0; j < 12; ++j) w[j] = 0u;
  }
  if (out) {
    uint4* p = (uint4*)(out + (size_t)r * ld + 24u * i);
    p[0] = make_uint4(w[0], w[1], w[2], w[3]);
    p[1] = make_uint4(w[4], w[5], w[6], w[7]);
    p[2] = make_uint4(w[8], w[9], w[10], w[11]);
  }
  if (out_t) {
    const uint32_t g = r / group_rows;
    __nv_bfloat16* ot = out_t + (size_t)g * 192u * ld_t + (r - g * group_rows);
#pragma unroll
    for (int j = 0; j < 12; ++j) {
      const uint32_t f = 24u * i + 2u * j;
      ot[(size_t)f * ld_t] = __ushort_as_bfloat16((unsigned short)(w[j] & 0xFFFFu));
      ot[(size_t)(f + 1) * ld_t] = __ushort_as_bfloat16((unsigned short)(w[j] >> 16));
    }
  }
}

// One warp per row: grad = (softmax(logits) - onehot(label)) * scale (BF16),
// loss_sum += logsumexp - logit[label]. Rows with label < 0 get zero gradient.
__global__ __launch_bounds__(256) void k_softmax_xent(const float* __restrict__ logits, uint32_t rows, uint32_t cols,
                                                      const int32_t* __restrict__ labels, float scale,
                                                      __nv_bfloat16* __restrict__ grad, float* __restrict__ loss_sum) {
  const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t lane = threadIdx.x & 31u;
  if (row >= rows) return;
  const float* x = logits + (size_t)row * cols;
  __nv_bfloat16* g = grad + (size_t)row * cols;
  const int32_t lab = labels[row];
  if (lab < 0 || lab >= (int32_t)cols) {
    for (uint32_t j = lane * 2; j < cols; j += 64) *(uint32_t*)(g + j) = 0u;
    return;
  }
  float mx = -INFINITY;
  for (uint32_t j = lane * 4; j < cols; j += 128) {
    const float4 v = *(const float4*)(x + j);
    mx = fmaxf(mx, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
  }
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  float sum = 0.0f;
  for (uint32_t j = lane * 4; j < cols; j += 128) {
    const float4 v = *(const float4*)(x + j);
    sum += __expf(v.x - mx) + __expf(v.y - mx) + __expf(v.z - mx) + __expf(v.w - mx);
  }
  for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  const float inv = 1.0f / sum;
  for (uint32_t j = lane * 4; j < cols; j += 128) {
    const float4 v = *(const float4*)(x + j);
    float p0 = __expf(v.x - mx) * inv, p1 = __expf(v.y - mx) * inv, p2 = __expf(v.z - mx) * inv, p3 = __expf(v.w - mx) * inv;
    if ((int32_t)j == lab) p0 -= 1.0f;
    if ((int32_t)j + 1 == lab) p1 -= 1.0f;
    if ((int32_t)j + 2 == lab) p2 -= 1.0f;
    if ((int32_t)j + 3 == lab) p3 -= 1.0f;
    *(uint2*)(g + j) = make_uint2(pack_bf16(p0 * scale, p1 * scale), pack_bf16(p2 * scale, p3 * scale));
  }
  if (lane == 0 && loss_sum) atomicAdd(loss_sum, (logf(sum) + mx - x[lab]) * scale);
}

// out[c][r] = in[r][c], 32 x 32 tiles through shared memory; blockIdx.z = group.
__global__ __launch_bounds__(256) void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, uint32_t rows, uint32_t cols, uint32_t ld_in,
                                                        __nv_bfloat16* __restrict__ out, uint32_t ld_out) {
  __shared__ __nv_bfloat16 tile[32][33];
  const uint32_t c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  in += (size_t)blockIdx.z * rows * ld_in;
  out += (size_t)blockIdx.z * cols * ld_out;
  for (uint32_t y = threadIdx.y; y < 32; y += blockDim.y) {
    const uint32_t r = r0 + y, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[y][threadIdx.x] = in[(size_t)r * ld_in + c];
  }
  __syncthreads();
  for (uint32_t y = threadIdx.y; y < 32; y += blockDim.y) {
    const uint32_t c = c0 + y, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * ld_out + r] = tile[threadIdx.x][y];
  }
}

// out[g cols + c] = sum of in[g rows + r][c] over r < rows, FP32, in a fixed
// order: block (32, 8) per 32 columns of one group (blockIdx.y); thread y sums
// rows y, y + 8, ... and the eight partial sums are added in order y = 0..7.
// The same sums with two columns per thread (4-byte loads, whole 128-byte
// rows per warp) and four rows in flight; each column's summation order is
// unchanged (row y, y + 8, ... per thread, then the eight partials in order),
// so the results are the same bits. Needs even cols and ld.
__global__ __launch_bounds__(256) void k_colsum2_bf16(const __nv_bfloat16* __restrict__ in, uint32_t rows, uint32_t cols, uint32_t ld,
                                                      float* __restrict__ out) {
  __shared__ float2 part[8][33];
  const uint32_t c = (blockIdx.x * 32 + threadIdx.x) * 2, g = blockIdx.y;
  const __nv_bfloat162* p = (const __nv_bfloat162*)(in + (size_t)g * rows * ld + c);
  const uint32_t ld2 = ld / 2;
  float s0 = 0.0f, s1 = 0.0f;
  if (c < cols) {
    uint32_t r = threadIdx.y;
    for (; r + 24 < rows; r += 32) {
      __nv_bfloat162 h[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) h[k] = p[(size_t)(r + 8 * k) * ld2];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        s0 += __low2float(h[k]);
        s1 += __high2float(h[k]);
      }
    }
    for (; r < rows; r += 8) {
      const __nv_bfloat162 h = p[(size_t)r * ld2];
      s0 += __low2float(h);
      s1 += __high2float(h);
    }
  }
  part[threadIdx.y][threadIdx.x] = make_float2(s0, s1);
  __syncthreads();
  if (threadIdx.y == 0 && c < cols) {
    float2 t = part[0][threadIdx.x];
#pragma unroll
    for (int y = 1; y < 8; ++y) {
      t.x += part[y][threadIdx.x].x;
      t.y += part[y][threadIdx.x].y;
    }
    *(float2*)(out + (size_t)g * cols + c) = t;
  }
}

__global__ __launch_bounds__(256) void k_colsum_bf16(const __nv_bfloat16* __restrict__ in, uint32_t rows, uint32_t cols, uint32_t ld,
                                                     float* __restrict__ out) {
  __shared__ float part[8][33];
  const uint32_t c = blockIdx.x * 32 + threadIdx.x, g = blockIdx.y;
  const __nv_bfloat16* p = in + (size_t)g * rows * ld + c;
  float s = 0.0f;
  if (c < cols)
    for (uint32_t r = threadIdx.y; r < rows; r += 8) s += __bfloat162float(p[(size_t)r * ld]);
  part[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && c < cols) {
    float t = part[0][threadIdx.x];
#pragma unroll
    for (int y = 1; y < 8; ++y) t += part[y][threadIdx.x];
    out[(size_t)g * cols + c] = t;
  }
}

// Row g batch + b <- row g stride + q, q from a strided walk of the group's
// rows (or of its index list).
__global__ __launch_bounds__(256) void k_gather_batch(const float4* __restrict__ orig, const float4* __restrict__ dir,
                                                      const int32_t* __restrict__ labels, uint32_t groups, uint32_t stride,
                                                      uint32_t offset, uint32_t batch, uint32_t hop, const uint32_t* __restrict__ index,
                                                      const uint32_t* __restrict__ index_count, float4* __restrict__ oo,
                                                      float4* __restrict__ od, int32_t* __restrict__ ol) {
  const size_t total = (size_t)groups * batch;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t g = (uint32_t)(i / batch), b = (uint32_t)(i - (size_t)g * batch);
    const uint32_t n = index ? __ldg(index_count + g) : stride;
    if (n == 0) {
      oo[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      od[i] = make_float4(0.f, 0.f, 1.f, 0.f);
      if (ol) ol[i] = -1;
      continue;
    }
    const uint32_t k = (uint32_t)((((uint64_t)offset + b) * hop) % n);
    const size_t src = (size_t)g * stride + (index ? __ldg(index + (size_t)g * stride + k) : k);
    oo[i] = __ldg(orig + src);
    od[i] = __ldg(dir + src);
    if (labels) ol[i] = __ldg(labels + src);
  }
}

// One CTA per group: stable compaction of the rows with a label >= 0.
__global__ __launch_bounds__(1024) void k_group_select(const int32_t* __restrict__ labels, uint32_t stride, uint32_t* __restrict__ index,
                                                       uint32_t* __restrict__ count) {
  __shared__ uint32_t s_w[32];
  const uint32_t g = blockIdx.x;
  const int32_t* lab = labels + (size_t)g * stride;
  uint32_t* idx = index + (size_t)g * stride;
  uint32_t base = 0;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  for (uint32_t c = 0; c < stride; c += 1024) {
    const uint32_t r = c + threadIdx.x;
    const bool keep = r < stride && __ldg(lab + r) >= 0;
    const uint32_t bal = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) s_w[warp] = __popc(bal);
    __syncthreads();
    uint32_t before = 0, tot = 0;
    for (uint32_t w = 0; w < 32; ++w) {
      const uint32_t x = s_w[w];
      before += w < warp ? x : 0u;
      tot += x;
    }
    if (keep) idx[base + before + __popc(bal & ((1u << lane) - 1u))] = r;
    base += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) count[g] = base;
}

__device__ __forceinline__ float adam_update(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                             float* __restrict__ v, size_t i, float lr, float b1, float b2, float eps, float c1, float c2) {
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  p[i] = pi;
  return pi;
}

// Adam (bias-corrected) on FP32 parameters [rows][cols]; refreshes the BF16
// copies [rows][ld16] and transposed [cols][ld16t] when given (with groups of
// group_rows rows: one transpose per group, group q in rows q cols ..).
__global__ __launch_bounds__(256) void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                              float* __restrict__ v, uint32_t rows, uint32_t cols, float lr, float b1, float b2,
                                              float eps, float c1, float c2, __nv_bfloat16* __restrict__ out16, uint32_t ld16,
                                              __nv_bfloat16* __restrict__ out16t, uint32_t ld16t, uint32_t group_rows) {
  const size_t total = (size_t)rows * cols;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const float pi = adam_update(p, g, m, v, i, lr, b1, b2, eps, c1, c2);
    const uint32_t r = (uint32_t)(i / cols), c = (uint32_t)(i % cols);
    if (out16) out16[(size_t)r * ld16 + c] = __float2bfloat16_rn(pi);
    if (out16t) {
      const uint32_t q = r / group_rows;
      out16t[((size_t)q * cols + c) * ld16t + (r - q * group_rows)] = __float2bfloat16_rn(pi);
    }
  }
}

// The same update over 32 x 32 tiles (block 32 x 8), with the BF16 transpose
// staged through shared memory so that both copies are written coalesced.
// The same update with four consecutive columns per thread (16-byte loads
// and stores; rows, cols, the BF16 leading dimensions and the group rows are
// multiples of 4 and the FP32 arrays 16-byte aligned): 256 threads per 32 x 32
// tile, the transposed BF16 copy through shared memory, 4 rows per 8-byte store.
__global__ __launch_bounds__(256) void k_adam_t4(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                                 float* __restrict__ v, uint32_t rows, uint32_t cols, float lr, float b1, float b2,
                                                 float eps, float c1, float c2, __nv_bfloat16* __restrict__ out16, uint32_t ld16,
                                                 __nv_bfloat16* __restrict__ out16t, uint32_t ld16t, uint32_t group_rows) {
  __shared__ __nv_bfloat16 tile[32][40];
  const uint32_t c0 = blockIdx.x * 32, r0 = blockIdx.y * 32, t = threadIdx.x;
  {
    const uint32_t lr_ = t >> 3, lc = (t & 7u) * 4u, r = r0 + lr_, c = c0 + lc;
    if (r < rows && c < cols) {
      const size_t i = (size_t)r * cols + c;
      const float4 gi = *(const float4*)(g + i);
      float4 mi = *(const float4*)(m + i), vi = *(const float4*)(v + i), pi = *(const float4*)(p + i);
      const float gv[4] = {gi.x, gi.y, gi.z, gi.w};
      float mv[4] = {mi.x, mi.y, mi.z, mi.w}, vv[4] = {vi.x, vi.y, vi.z, vi.w}, pv[4] = {pi.x, pi.y, pi.z, pi.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        // adam_update's arithmetic, element by element
        mv[k] = b1 * mv[k] + (1.0f - b1) * gv[k];
        vv[k] = b2 * vv[k] + (1.0f - b2) * gv[k] * gv[k];
        pv[k] = pv[k] - lr * (mv[k] * c1) / (sqrtf(vv[k] * c2) + eps);
      }
      *(float4*)(m + i) = make_float4(mv[0], mv[1], mv[2], mv[3]);
      *(float4*)(v + i) = make_float4(vv[0], vv[1], vv[2], vv[3]);
      *(float4*)(p + i) = make_float4(pv[0], pv[1], pv[2], pv[3]);
      __nv_bfloat16 h[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        h[k] = __float2bfloat16_rn(pv[k]);
        tile[lr_][lc + k] = h[k];
      }
      if (out16) *(uint2*)(out16 + (size_t)r * ld16 + c) = pack_bf16x4(h[0], h[1], h[2], h[3]);
    }
  }
  __syncthreads();
  {
    const uint32_t lc = t >> 3, lr_ = (t & 7u) * 4u, c = c0 + lc, r = r0 + lr_;
    if (r < rows && c < cols) {
      __nv_bfloat16 h[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) h[k] = tile[lr_ + k][lc];
      const uint32_t q = r / group_rows;
      *(uint2*)(out16t + ((size_t)q * cols + c) * ld16t + (r - q * group_rows)) = pack_bf16x4(h[0], h[1], h[2], h[3]);
    }
  }
}

__global__ __launch_bounds__(256) void k_adam_t(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                                float* __restrict__ v, uint32_t rows, uint32_t cols, float lr, float b1, float b2,
                                                float eps, float c1, float c2, __nv_bfloat16* __restrict__ out16, uint32_t ld16,
                                                __nv_bfloat16* __restrict__ out16t, uint32_t ld16t, uint32_t group_rows) {
  __shared__ __nv_bfloat16 tile[32][34];
  const uint32_t c0 = blockIdx.x * 32, r0 = blockIdx.y * 32, tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k) {
    const uint32_t r = r0 + ty + 8 * k, c = c0 + tx;
    if (r < rows && c < cols) {
      const float pi = adam_update(p, g, m, v, (size_t)r * cols + c, lr, b1, b2, eps, c1, c2);
      const __nv_bfloat16 h = __float2bfloat16_rn(pi);
      if (out16) out16[(size_t)r * ld16 + c] = h;
      tile[ty + 8 * k][tx] = h;
    }
  }
  __syncthreads();
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k) {
    const uint32_t c = c0 + ty + 8 * k, r = r0 + tx;
    if (r < rows && c < cols) {
      const uint32_t q = r / group_rows;
      out16t[((size_t)q * cols + c) * ld16t + (r - q * group_rows)] = tile[tx][ty + 8 * k];
    }
  }
}

// ----------------------------------------------------------------------------
// Fused proposal: features -> 3 x (128, ReLU) -> argmax over n logits for a
// tile of 128 rays per step, persistent over tiles (grid <= SM count).
// Warps 0-15 compute: warp w serves TMEM lane quarter w % 4 and column quarter
// w / 4 (features into shared memory; the hidden layers' bias + ReLU from TMEM
// back into shared memory as the next layer's A operand; a running top-2 over
// its quarter of the logits, merged per row through shared memory). Warp 16
// streams the weight tiles through a 3-stage TMA ring (W1..W3 as 128 x 64, W4
// as 256 x 64) and the tile's biases into one of two shared buffers with bulk
// copies; warp 17 issues the MMAs. Activations never leave the SM. Shared
// memory: A (48 KB: X, then H2), B (32 KB: H1, then H3), ring 3 x 32 KB, bias
// 2 x (n + 384) floats. TMEM: the hidden layers use columns [0, 128); the
// logits alternate [0, 256) / [256, 512). Every wait is bounded; one that runs
// out raises the shared abort flag, and every role leaves its tile loop at its
// next wait.
// ----------------------------------------------------------------------------
constexpr uint32_t kFuseCompute = 512;
constexpr uint32_t kFuseThreads = kFuseCompute + 64;
constexpr uint32_t kFuseStages = 3;
constexpr uint32_t kFuseStage = 32768;
constexpr uint32_t kFuseBias = kArgMaxN + 384;  // floats per bias buffer: b4 [n], b1, b2, b3 [128] at kArgMaxN

struct FuseArgs {
  const float4* orig;
  const float4* dir;
  uint32_t count;
  float3 c, s;
  const float* b1;
  const float* b2;
  const float* b3;
  const float* b4;
  uint32_t n, group_rows, tiles;
  float min_margin;
  int32_t* out_idx;
  float* out_val;
  float* out_margin;
  uint32_t* err;
  const float* tmax;  // optional: rays with tmax <= 0 get -1; all-inactive tiles are skipped
};

// Whether any ray of the tile starting at row0 is active (tmax > 0), computed
// by a whole warp; every role of the CTA reaches the same answer.
__device__ __forceinline__ bool tile_active(const FuseArgs& P, uint32_t row0) {
  if (!P.tmax) return true;
  bool any = false;
  for (uint32_t i = lane_id(); i < kBM; i += 32) {
    const uint32_t row = row0 + i;
    any |= row < P.count && __ldg(P.tmax + row) > 0.0f;
  }
  return __any_sync(0xffffffffu, any);
}

size_t fuse_smem() {
  return 1024 + 5 * (size_t)kTileA + kFuseStages * (size_t)kFuseStage + 2 * (size_t)kFuseBias * 4 + 3 * kBM * sizeof(Top2) + 24 * 8 +
         64;
}

// Two IEEE single additions in one packed instruction (add.rn.f32x2, sm_100):
// each lane rounds exactly as a scalar add.
__device__ __forceinline__ void add2(float a0, float a1, float b0, float b1, float& d0, float& d1) {
  asm("{\n\t.reg .b64 pa, pb, pd;\n\t"
      "mov.b64 pa, {%2, %3};\n\t"
      "mov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pd, pa, pb;\n\t"
      "mov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(d0), "=f"(d1)
      : "f"(a0), "f"(a1), "f"(b0), "f"(b1));
}

// Top-1 sweep of 16 logits (TMEM columns col .. col + 15 of this row) plus
// their biases into the four interleaved chains (chain j: columns = j mod 4).
__device__ __forceinline__ void sweep16_top1(const uint32_t (&r)[16], const float* sb, uint32_t col, float (&bk)[4], int32_t (&ik)[4]) {
  const float4* bp = (const float4*)(sb + col);
#pragma unroll
  for (int i4 = 0; i4 < 4; ++i4) {
    const float4 b = bp[i4];
    float x[4];
    add2(__uint_as_float(r[4 * i4]), __uint_as_float(r[4 * i4 + 1]), b.x, b.y, x[0], x[1]);
    add2(__uint_as_float(r[4 * i4 + 2]), __uint_as_float(r[4 * i4 + 3]), b.z, b.w, x[2], x[3]);
    const int32_t base = (int32_t)(col + 4 * i4);
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (x[j] > bk[j]) { bk[j] = x[j]; ik[j] = base; }
  }
}

// kTop2: also track each row's runner-up (for a margin); without it the logit
// sweep keeps only the maximum and its index (the same index either way).
template <bool kTop2>
__global__ void __launch_bounds__(kFuseThreads, 1)
    k_mlp_propose_tc(const __grid_constant__ CUtensorMap t1, const __grid_constant__ CUtensorMap t2,
                     const __grid_constant__ CUtensorMap t3, const __grid_constant__ CUtensorMap t4, FuseArgs P) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = smem;                   // 3 atoms of 128 x 64 BF16
  uint8_t* sB = sA + 3 * kTileA;        // 2 atoms
  uint8_t* sR = sB + 2 * kTileA;        // ring
  float* s_bias = (float*)(sR + kFuseStages * kFuseStage);  // [2][kFuseBias]
  Top2* s_part = (Top2*)(s_bias + 2 * kFuseBias);           // [3][128]: column quarters 1..3
  uint64_t* full = (uint64_t*)(s_part + 3 * kBM);
  uint64_t* empty = full + kFuseStages;
  uint64_t* x_ready = empty + kFuseStages;
  uint64_t* h_ready = x_ready + 1;
  uint64_t* lay_done = h_ready + 1;
  uint64_t* acc_full = lay_done + 1;   // [2]
  uint64_t* acc_empty = acc_full + 2;  // [2]
  uint64_t* part_ready = acc_empty + 2;
  uint64_t* part_free = part_ready + 1;
  uint64_t* bias_full = part_free + 1;    // [2]
  uint64_t* bias_empty = bias_full + 2;   // [2]
  uint64_t* done = bias_empty + 2;
  uint32_t* tmem_slot = (uint32_t*)(done + 1);
  volatile uint32_t* s_abort = tmem_slot + 1;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  if (threadIdx.x == 0) {
    for (uint32_t q = 0; q < kFuseStages; ++q) {
      mbar_init(full + q, 1);
      mbar_init(empty + q, 1);
    }
    mbar_init(x_ready, kFuseCompute);
    mbar_init(h_ready, kFuseCompute);
    mbar_init(lay_done, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + b, 1);
      mbar_init(acc_empty + b, kFuseCompute);
      mbar_init(bias_full + b, 1);
      mbar_init(bias_empty + b, kFuseCompute);
    }
    mbar_init(part_ready, 3 * kBM);
    mbar_init(part_free, kBM);
    mbar_init(done, 1);
    *s_abort = 0u;
    fence_mbar_init();
    prefetch_tmap(&t1);
    prefetch_tmap(&t2);
    prefetch_tmap(&t3);
    prefetch_tmap(&t4);
  }
  // features 144 .. 191 (atom 2, columns 16 .. 63) stay zero: no tile writes them
  for (uint32_t i = threadIdx.x; i < kTileA / 16; i += kFuseThreads) ((uint4*)(sA + 2 * kTileA))[i] = make_uint4(0u, 0u, 0u, 0u);
  fence_proxy_async();
  __syncwarp();
  if (warp == 0) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t ntiles = P.n / kArgBN;
  // bounded wait that also honours (and raises) the abort flag
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    if (*s_abort) return false;
    if (mbar_wait(bar, parity, P.err)) return true;
    *s_abort = 1u;
    return false;
  };

  if (warp == 16) {
    {
      uint32_t q = 0, k = 0;
      bool ok = true;
      auto load = [&](const CUtensorMap* m, int32_t x, int32_t y, uint32_t bytes) -> bool {
        const uint32_t st = q % kFuseStages;
        if (q >= kFuseStages && !wait(empty + st, ((q / kFuseStages) - 1u) & 1u)) return false;
        mbar_arrive_expect_tx(full + st, bytes);
        tma_load_2d(sR + st * kFuseStage, m, x, y, full + st);
        ++q;
        return true;
      };
      // lane 0 issues the copies; the whole warp only decides which tiles are active
      for (uint32_t tile = blockIdx.x; ok && tile < P.tiles; tile += gridDim.x) {
        if (!tile_active(P, tile * kBM)) continue;
        bool issued = false;  // the tile's bias copy went out (k counts those)
        if (lane == 0 && k >= 2) ok = wait(bias_empty + (k & 1u), ((k >> 1) - 1u) & 1u);
        if (lane == 0 && ok) {
          const uint32_t g = tile * kBM / P.group_rows, bb = k & 1u;
          float* sb = s_bias + bb * kFuseBias;
          issued = true;
          mbar_arrive_expect_tx(bias_full + bb, P.n * 4u + 3u * 512u);
          bulk_load(sb, P.b4 + (size_t)g * P.n, P.n * 4u, bias_full + bb);
          bulk_load(sb + kArgMaxN, P.b1 + (size_t)g * 128u, 512u, bias_full + bb);
          bulk_load(sb + kArgMaxN + 128, P.b2 + (size_t)g * 128u, 512u, bias_full + bb);
          bulk_load(sb + kArgMaxN + 256, P.b3 + (size_t)g * 128u, 512u, bias_full + bb);
          for (uint32_t kc = 0; ok && kc < 3; ++kc) ok = load(&t1, (int32_t)(kc * kBK), (int32_t)(g * kBM), kTileA);
          for (uint32_t kc = 0; ok && kc < 2; ++kc) ok = load(&t2, (int32_t)(kc * kBK), (int32_t)(g * kBM), kTileA);
          for (uint32_t kc = 0; ok && kc < 2; ++kc) ok = load(&t3, (int32_t)(kc * kBK), (int32_t)(g * kBM), kTileA);
          for (uint32_t t = 0; ok && t < ntiles; ++t)
            for (uint32_t kc = 0; ok && kc < 2; ++kc) ok = load(&t4, (int32_t)(kc * kBK), (int32_t)(g * P.n + t * kArgBN), kArgTileB);
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (__shfl_sync(0xffffffffu, issued, 0)) ++k;
      }
      // the last copy into each stage / bias buffer has landed before the CTA may exit
      if (lane == 0) {
        for (uint32_t j = q > kFuseStages ? q - kFuseStages : 0u; j < q; ++j)
          mbar_wait(full + j % kFuseStages, (j / kFuseStages) & 1u, P.err);
        for (uint32_t j = k > 2 ? k - 2 : 0u; j < k; ++j) mbar_wait(bias_full + (j & 1u), (j >> 1) & 1u, P.err);
      }
    }
  } else if (warp == 17) {
    // lane 0 issues the MMAs of this CTA's active tiles (every tile takes the same MMA sequence)
    uint32_t nact = 0;
    for (uint32_t tile = blockIdx.x; tile < P.tiles; tile += gridDim.x) nact += tile_active(P, tile * kBM) ? 1u : 0u;
    if (lane == 0) {
      const uint32_t id_h = idesc_bf16_f32(kBM, 128), id_l = idesc_bf16_f32(kBM, kArgBN);
      uint32_t q = 0, xr = 0, hr = 0, n4 = 0;
      bool ok = true;
      // one 64-wide K chunk: A atom at a_atom, B from the next ring stage
      auto chunk = [&](uint32_t d, const uint8_t* a_atom, uint32_t idesc, bool first) -> bool {
        const uint32_t st = q % kFuseStages;
        if (!wait(full + st, (q / kFuseStages) & 1u)) return false;
        tc_fence_after();
        const uint32_t a = smem_u32(a_atom), b = smem_u32(sR + st * kFuseStage);
#pragma unroll
        for (uint32_t kk = 0; kk < kBK / 16; ++kk) mma_bf16(d, desc_sw128(a + kk * 32u), desc_sw128(b + kk * 32u), idesc, (!first || kk) ? 1u : 0u);
        mma_commit(empty + st);
        ++q;
        return true;
      };
      for (uint32_t it = 0; ok && it < nact; ++it) {
        ok = wait(x_ready, xr++ & 1u);
        tc_fence_after();
        for (uint32_t kc = 0; ok && kc < 3; ++kc) ok = chunk(tmem, sA + kc * kTileA, id_h, kc == 0);
        if (!ok) break;
        mma_commit(lay_done);
        ok = wait(h_ready, hr++ & 1u);
        tc_fence_after();
        for (uint32_t kc = 0; ok && kc < 2; ++kc) ok = chunk(tmem, sB + kc * kTileA, id_h, kc == 0);
        if (!ok) break;
        mma_commit(lay_done);
        ok = wait(h_ready, hr++ & 1u);
        tc_fence_after();
        for (uint32_t kc = 0; ok && kc < 2; ++kc) ok = chunk(tmem, sA + kc * kTileA, id_h, kc == 0);
        if (!ok) break;
        mma_commit(lay_done);
        ok = wait(h_ready, hr++ & 1u);
        tc_fence_after();
        for (uint32_t t = 0; ok && t < ntiles; ++t, ++n4) {
          const uint32_t buf = n4 & 1u;
          if (n4 >= 2 && !(ok = wait(acc_empty + buf, ((n4 >> 1) - 1u) & 1u))) break;
          tc_fence_after();
          for (uint32_t kc = 0; ok && kc < 2; ++kc) ok = chunk(tmem + buf * kArgBN, sB + kc * kTileA, id_l, kc == 0);
          if (ok) mma_commit(acc_full + buf);
        }
      }
      mma_commit(done);  // arrives when every MMA issued above has completed
      mbar_wait(done, 0, P.err);
    }
  } else {
    // compute warps 0-15: TMEM lane quarter warp % 4, column quarter warp / 4
    const uint32_t qw = warp & 3u, cq = warp >> 2, tid = threadIdx.x;
    const uint32_t trow = qw * 32u + lane;  // TMEM lane = tile row of this thread
    uint32_t ld = 0, n4 = 0, k = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; ok && tile < P.tiles; tile += gridDim.x) {
      const uint32_t row0 = tile * kBM, bb = k & 1u;
      if (!tile_active(P, row0)) {  // no ray of the tile is active: no proposal
        if (cq == 0 && row0 + trow < P.count) {
          P.out_idx[row0 + trow] = -1;
          if (P.out_val) P.out_val[row0 + trow] = -INFINITY;
          if (P.out_margin) P.out_margin[row0 + trow] = 0.0f;
        }
        continue;
      }
      // features: (ray r, input i) pairs p = 128 i + r, i < 6
      for (uint32_t p = tid; p < 6u * kBM; p += kFuseCompute) {
        const uint32_t r = p & 127u, i = p >> 7, row = row0 + r;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (row < P.count) v = __ldg((i < 3 ? P.orig : P.dir) + row);
        uint32_t w[12];
        encode12(i < 3 ? origin_input(v, P.c, P.s, i) : dir_input(v, i - 3), w);
        const uint32_t f0 = 24u * i;
#pragma unroll
        for (uint32_t j = 0; j < 12; ++j) {
          const uint32_t f = f0 + 2u * j;
          *(uint32_t*)(sA + (f >> 6) * kTileA + sw128_offset(r, f & 63u)) = w[j];
        }
      }
      fence_proxy_async();
      mbar_arrive(x_ready);
      ok = __all_sync(0xffffffffu, wait(bias_full + bb, (k >> 1) & 1u));
      if (!ok) break;
      const float* sb = s_bias + bb * kFuseBias;
      // hidden layers: bias + ReLU of TMEM columns [32 cq, 32 cq + 32) into the next A operand
      for (uint32_t L = 0; L < 3; ++L) {
        ok = __all_sync(0xffffffffu, wait(lay_done, ld++ & 1u));
        tc_fence_after();
        if (!ok) break;
        uint8_t* atom = (L == 1 ? sA : sB) + (cq >> 1) * kTileA;
        const float* bias = sb + kArgMaxN + L * 128u;
        const uint32_t tl = tmem + ((qw * 32u) << 16) + cq * 32u;
#pragma unroll
        for (uint32_t c = 0; c < 32; c += 16) {
          float v[16];
          tmem_ld16(tl + c, v);
          const uint32_t col = cq * 32u + c, kin = col & 63u;
          uint32_t w[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float a = fmaxf(v[2 * i] + bias[col + 2 * i], 0.0f);
            const float b = fmaxf(v[2 * i + 1] + bias[col + 2 * i + 1], 0.0f);
            w[i] = pack_bf16(a, b);
          }
          *(uint4*)(atom + sw128_offset(trow, kin)) = make_uint4(w[0], w[1], w[2], w[3]);
          *(uint4*)(atom + sw128_offset(trow, kin + 8u)) = make_uint4(w[4], w[5], w[6], w[7]);
        }
        fence_proxy_async();
        tc_fence_before();
        mbar_arrive(h_ready);
      }
      if (!ok) break;
      // logits: running maximum (and runner-up) over four interleaved column
      // chains of this quarter; chain j holds columns = j (mod 4), and ik[j]
      // keeps the winner's column minus j
      float bk[4], sk[4];
      int32_t ik[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) { bk[j] = -INFINITY; sk[j] = -INFINITY; ik[j] = -1 - j; }
      for (uint32_t t = 0; t < ntiles; ++t, ++n4) {
        const uint32_t buf = n4 & 1u;
        ok = ok && __all_sync(0xffffffffu, wait(acc_full + buf, (n4 >> 1) & 1u));
        tc_fence_after();
        if (ok && !kTop2) {
          // four 16-column loads, each started before the previous one is swept
          const uint32_t c0 = cq * (kArgBN / 4);
          const uint32_t tl = tmem + ((qw * 32u) << 16) + buf * kArgBN + c0;
          const uint32_t col0 = t * kArgBN + c0;
          uint32_t ra[16], rb[16];
          tmem_ld16_issue(tl, ra);
          tmem_ld_wait(ra);
#pragma unroll
          for (uint32_t c = 0; c < kArgBN / 4; c += 32) {
            tmem_ld16_issue(tl + c + 16, rb);
            sweep16_top1(ra, sb, col0 + c, bk, ik);
            tmem_ld_wait(rb);
            if (c + 32 < kArgBN / 4) tmem_ld16_issue(tl + c + 32, ra);
            sweep16_top1(rb, sb, col0 + c + 16, bk, ik);
            if (c + 32 < kArgBN / 4) tmem_ld_wait(ra);
          }
        } else if (ok) {
          const uint32_t c0 = cq * (kArgBN / 4);
          const uint32_t tl = tmem + ((qw * 32u) << 16) + buf * kArgBN + c0;
#pragma unroll
          for (uint32_t c = 0; c < kArgBN / 4; c += 16) {
            float v[16];
            tmem_ld16(tl + c, v);
            const uint32_t col = t * kArgBN + c0 + c;
            const float4* bp = (const float4*)(sb + col);
#pragma unroll
            for (int i4 = 0; i4 < 4; ++i4) {
              const float4 b = bp[i4];
              const float bv[4] = {b.x, b.y, b.z, b.w};
              const int32_t base = (int32_t)(col + 4 * i4);
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                const float x = v[4 * i4 + j] + bv[j];
                if (kTop2) sk[j] = fmaxf(sk[j], fminf(x, bk[j]));
                if (x > bk[j]) { bk[j] = x; ik[j] = base; }
              }
            }
          }
        }
        tc_fence_before();
        mbar_arrive(acc_empty + buf);
      }
      mbar_arrive(bias_empty + bb);
      if (!ok) break;
      Top2 res = Top2{bk[0], sk[0], ik[0]};
#pragma unroll
      for (int j = 1; j < 4; ++j) res = top2_merge(res, Top2{bk[j], sk[j], ik[j] + j});
      if (cq > 0) {
        if (k > 0) ok = __all_sync(0xffffffffu, wait(part_free, (k - 1u) & 1u));
        if (!ok) break;
        s_part[(cq - 1u) * kBM + trow] = res;
        mbar_arrive(part_ready);
      } else {
        ok = __all_sync(0xffffffffu, wait(part_ready, k & 1u));
        if (!ok) break;
#pragma unroll
        for (uint32_t j = 0; j < 3; ++j) res = top2_merge(res, s_part[j * kBM + trow]);
        mbar_arrive(part_free);
        const uint32_t row = row0 + trow;
        if (row < P.count) {
          const float margin = res.best - res.second;
          const bool active = !P.tmax || __ldg(P.tmax + row) > 0.0f;
          P.out_idx[row] = (active && margin >= P.min_margin) ? res.idx : -1;
          if (P.out_val) P.out_val[row] = res.best;
          if (P.out_margin) P.out_margin[row] = margin;
        }
      }
      ++k;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ----------------------------------------------------------------------------
// Host side
// ----------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    else
      cudaGetLastError();
  });
  return fn;
}

// BF16 matrix [rows][ld] (K-major, k valid columns) as boxes of 64 x box_rows
// with the 128-byte swizzle.
bool make_map(CUtensorMap* map, const void* base, uint32_t k, uint32_t rows, uint32_t ld, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {k, rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2u};
  cuuint32_t box[2] = {kBK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

uint32_t pick_bn(uint32_t n) {
  for (uint32_t bn = 256; bn >= 16; bn -= 16)
    if (n % bn == 0) return bn;
  return 0;
}

uint32_t pow2_cols(uint32_t n) {
  uint32_t c = 32;
  while (c < n) c <<= 1;
  return c;
}

size_t gemm_smem(uint32_t bn, uint32_t stages = kStages) { return 1024 + stages * (kTileA + (size_t)bn * 128u) + 256; }
size_t argmax_smem(uint32_t num_k, uint32_t n) {
  return 1024 + num_k * (size_t)kTileA + kStages * (size_t)kArgTileB + (size_t)n * 4 + kBM * sizeof(Top2) + 256;
}

// Self-test of the bounded-wait path that every tensor-core kernel above takes when a copy or an MMA never
// completes: one warp allocates 32 TMEM columns, waits on a barrier that nothing arrives at for limit_ns,
// records the outcome, releases the TMEM and returns. Nothing is in flight while it waits.
__global__ void __launch_bounds__(32, 1) k_wait_selftest(unsigned long long limit_ns, uint32_t* err, uint32_t* result) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t slot;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncwarp();
  tmem_alloc(&slot, 32);
  tmem_relinquish();
  tc_fence_before();
  __syncwarp();
  tc_fence_after();
  const uint32_t tmem = slot;
  const unsigned long long t0 = global_ns();
  const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar, 0, err, limit_ns));
  const unsigned long long t1 = global_ns();
  if (threadIdx.x == 0) {
    result[0] = ok ? 1u : 0u;
    result[1] = (uint32_t)((t1 - t0) / 1000ull);
  }
  tc_fence_before();
  __syncwarp();
  tmem_dealloc(tmem, 32);
}

}  // namespace
}  // namespace rt

using namespace rt;

extern "C" rt_status rt_tc_wait_selftest(uint32_t limit_us, uint32_t* error_word, uint32_t* result, rt_stream stream) {
  if (!error_word || !result || limit_us == 0 || limit_us > 2000000u) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  k_wait_selftest<<<1, 32, 0, (cudaStream_t)stream>>>(1000ull * limit_us, error_word, result);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" uint32_t rt_propose_abi_version(void) { return RT_PROPOSE_ABI_VERSION; }

extern "C" rt_status rt_gemm_bf16(const rt_gemm_desc* d, rt_stream stream) {
  if (!d || !d->a || !d->b) return RT_ERR_INVALID_ARGUMENT;
  if (d->m == 0 || d->n == 0 || d->k == 0) return RT_ERR_INVALID_ARGUMENT;
  if (d->m % kBM || d->k % kBK || d->n % 16) return RT_ERR_INVALID_ARGUMENT;
  if (d->lda < d->k || d->ldb < d->k || d->lda % 8 || d->ldb % 8) return RT_ERR_INVALID_ARGUMENT;
  if (!aligned16(d->a) || !aligned16(d->b)) return RT_ERR_INVALID_ARGUMENT;
  if (d->c_f32 && (d->ldc_f32 < d->n || d->ldc_f32 % 4 || !aligned16(d->c_f32))) return RT_ERR_INVALID_ARGUMENT;
  if (d->c_bf16 && (d->ldc_bf16 < d->n || d->ldc_bf16 % 8 || !aligned16(d->c_bf16))) return RT_ERR_INVALID_ARGUMENT;
  if (d->mask && (d->ldmask < d->n || d->ldmask % 8 || !aligned16(d->mask))) return RT_ERR_INVALID_ARGUMENT;
  if (d->ct_bf16 && d->ldct < d->m) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t G = d->groups ? d->groups : 1u;
  if (G > 65535u || (uint64_t)G * d->m > 0x7FFFFFFFull || (uint64_t)G * d->n > 0x7FFFFFFFull) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  const uint32_t bn = pick_bn(d->n);
  CUtensorMap ta, tb;
  if (!make_map(&ta, d->a, d->k, G * d->m, d->lda, kBM) || !make_map(&tb, d->b, d->k, G * d->n, d->ldb, bn)) return RT_ERR_UNSUPPORTED;
  GemmEpi E;
  E.alpha = d->alpha; E.bias = d->bias; E.relu = d->relu; E.mask = (const __nv_bfloat16*)d->mask; E.ldmask = d->ldmask;
  E.c32 = d->c_f32; E.ldc32 = d->ldc_f32; E.c16 = (__nv_bfloat16*)d->c_bf16; E.ldc16 = d->ldc_bf16;
  E.ct16 = (__nv_bfloat16*)d->ct_bf16; E.ldct = d->ldct;
  E.gm = d->m; E.gn = d->n;
  E.c32_v8 = (d->c_f32 && d->ldc_f32 % 8 == 0 && ((uintptr_t)d->c_f32 & 31u) == 0) ? 1u : 0u;
  E.c16_v8 = (d->c_bf16 && d->ldc_bf16 % 16 == 0 && ((uintptr_t)d->c_bf16 & 31u) == 0) ? 1u : 0u;
  const uint32_t num_k = d->k / kBK, stages = num_k < kStages ? num_k : kStages;
  const size_t smem = gemm_smem(bn, stages);
  static PerDeviceOnce once;
  if (!once.run([] { return cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem(256)) == cudaSuccess; }))
    return RT_ERR_CUDA;
  dim3 grid(d->n / bn, d->m / kBM, G);
  k_gemm_tc<<<grid, 128, smem, (cudaStream_t)stream>>>(ta, tb, E, bn, pow2_cols(bn), num_k, stages, d->error_word);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_gemm_argmax_bf16(const rt_gemm_argmax_desc* d, rt_stream stream) {
  if (!d || !d->a || !d->b || !d->out_index) return RT_ERR_INVALID_ARGUMENT;
  if (d->m == 0 || d->m % kBM || d->n == 0 || d->n % kArgBN || d->n > kArgMaxN || d->k == 0 || d->k % kBK || d->k > 256)
    return RT_ERR_INVALID_ARGUMENT;
  if (d->lda < d->k || d->ldb < d->k || d->lda % 8 || d->ldb % 8 || !aligned16(d->a) || !aligned16(d->b))
    return RT_ERR_INVALID_ARGUMENT;
  const uint32_t G = d->groups ? d->groups : 1u;
  if (G > 65535u || (uint64_t)G * d->m > 0x7FFFFFFFull || (uint64_t)G * d->n > 0x7FFFFFFFull) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  CUtensorMap ta, tb;
  if (!make_map(&ta, d->a, d->k, G * d->m, d->lda, kBM) || !make_map(&tb, d->b, d->k, G * d->n, d->ldb, kArgBN)) return RT_ERR_UNSUPPORTED;
  const uint32_t num_k = d->k / kBK;
  static PerDeviceOnce once;
  if (!once.run([] {
        return cudaFuncSetAttribute(k_gemm_argmax_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)argmax_smem(4, kArgMaxN)) ==
               cudaSuccess;
      }))
    return RT_ERR_CUDA;
  k_gemm_argmax_tc<<<dim3(d->m / kBM, G), kArgThreads, argmax_smem(num_k, d->n), (cudaStream_t)stream>>>(
      ta, tb, d->bias, d->n, d->m, num_k, d->min_margin, d->out_index, d->out_value, d->out_margin, d->error_word);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_gemm_xent_bf16(const rt_gemm_xent_desc* d, rt_stream stream) {
  if (!d || !d->a || !d->b || !d->labels || !d->g || !d->gt) return RT_ERR_INVALID_ARGUMENT;
  if (d->m == 0 || d->m % kBM || d->n == 0 || d->n % kArgBN || d->n > kArgMaxN || d->k == 0 || d->k % kBK || d->k > 256)
    return RT_ERR_INVALID_ARGUMENT;
  if (d->lda < d->k || d->ldb < d->k || d->lda % 8 || d->ldb % 8 || !aligned16(d->a) || !aligned16(d->b))
    return RT_ERR_INVALID_ARGUMENT;
  if (d->ldg < d->n || d->ldg % 8 || !aligned16(d->g) || d->ldgt < d->m) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t G = d->groups ? d->groups : 1u;
  if (G > 65535u || (uint64_t)G * d->m > 0x7FFFFFFFull || (uint64_t)G * d->n > 0x7FFFFFFFull) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  CUtensorMap ta, tb;
  if (!make_map(&ta, d->a, d->k, G * d->m, d->lda, kBM) || !make_map(&tb, d->b, d->k, G * d->n, d->ldb, kArgBN)) return RT_ERR_UNSUPPORTED;
  XentArgs X;
  X.bias = d->bias; X.labels = d->labels; X.n = d->n; X.gm = d->m; X.scale = d->scale;
  X.g = (__nv_bfloat16*)d->g; X.ldg = d->ldg; X.gt = (__nv_bfloat16*)d->gt; X.ldgt = d->ldgt; X.loss_sum = d->loss_sum;
  X.err = d->error_word;
  X.g32 = (d->ldg % 16 == 0 && ((uintptr_t)d->g & 31u) == 0) ? 1u : 0u;
  const uint32_t num_k = d->k / kBK;
  static PerDeviceOnce once;
  if (!once.run([] {
        return cudaFuncSetAttribute(k_gemm_xent_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xent_smem(4, kArgMaxN)) ==
               cudaSuccess;
      }))
    return RT_ERR_CUDA;
  k_gemm_xent_tc<<<dim3(d->m / kBM, G), kXentThreads, xent_smem(num_k, d->n), (cudaStream_t)stream>>>(ta, tb, X, num_k);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_mlp_propose(const rt_mlp_propose_desc* d, rt_stream stream) {
  if (!d || !d->orig || !d->dir || !d->w1 || !d->w2 || !d->w3 || !d->w4 || !d->b1 || !d->b2 || !d->b3 || !d->b4 || !d->out_index)
    return RT_ERR_INVALID_ARGUMENT;
  if (d->n == 0 || d->n % kArgBN || d->n > kArgMaxN) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t G = d->groups ? d->groups : 1u;
  if (G > 1 && (d->group_rows == 0 || d->group_rows % kBM || (uint64_t)G * d->group_rows != d->count)) return RT_ERR_INVALID_ARGUMENT;
  if ((uint64_t)G * d->n > 0x7FFFFFFFull || !aligned16(d->w1) || !aligned16(d->w2) || !aligned16(d->w3) || !aligned16(d->w4) ||
      !aligned16(d->b1) || !aligned16(d->b2) || !aligned16(d->b3) || !aligned16(d->b4))
    return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (d->count == 0) return RT_OK;
  CUtensorMap t1, t2, t3, t4;
  if (!make_map(&t1, d->w1, 192, G * kBM, 192, kBM) || !make_map(&t2, d->w2, 128, G * kBM, 128, kBM) ||
      !make_map(&t3, d->w3, 128, G * kBM, 128, kBM) || !make_map(&t4, d->w4, 128, G * d->n, 128, kArgBN))
    return RT_ERR_UNSUPPORTED;
  FuseArgs P;
  P.orig = (const float4*)d->orig; P.dir = (const float4*)d->dir; P.count = d->count;
  P.c = make_float3(0.5f * (d->box_lo[0] + d->box_hi[0]), 0.5f * (d->box_lo[1] + d->box_hi[1]), 0.5f * (d->box_lo[2] + d->box_hi[2]));
  P.s = make_float3(2.0f / (d->box_hi[0] - d->box_lo[0]), 2.0f / (d->box_hi[1] - d->box_lo[1]), 2.0f / (d->box_hi[2] - d->box_lo[2]));
  P.b1 = d->b1; P.b2 = d->b2; P.b3 = d->b3; P.b4 = d->b4; P.n = d->n;
  P.tiles = (d->count + kBM - 1) / kBM;
  P.group_rows = G > 1 ? d->group_rows : P.tiles * kBM;
  P.min_margin = d->min_margin; P.out_idx = d->out_index; P.out_val = d->out_value; P.out_margin = d->out_margin; P.err = d->error_word;
  P.tmax = d->tmax;
  static PerDeviceOnce once;
  if (!once.run([] {
        return cudaFuncSetAttribute(k_mlp_propose_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fuse_smem()) ==
                   cudaSuccess &&
               cudaFuncSetAttribute(k_mlp_propose_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fuse_smem()) ==
                   cudaSuccess;
      }))
    return RT_ERR_CUDA;
  const uint32_t grid = (uint32_t)hmin<uint32_t>(P.tiles, (uint32_t)num_sms());
  if (d->out_margin || d->min_margin > 0.0f)
    k_mlp_propose_tc<true><<<grid, kFuseThreads, fuse_smem(), (cudaStream_t)stream>>>(t1, t2, t3, t4, P);
  else
    k_mlp_propose_tc<false><<<grid, kFuseThreads, fuse_smem(), (cudaStream_t)stream>>>(t1, t2, t3, t4, P);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_ray_features(const rt_feature_desc* d, rt_stream stream) {
  if (!d || !d->orig || !d->dir || (!d->out && !d->out_t)) return RT_ERR_INVALID_ARGUMENT;
  if (d->out && (d->ld_out < 192 || d->ld_out % 8 || !aligned16(d->out))) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t gr = d->group_rows ? d->group_rows : d->count;
  if (d->group_rows && d->count % d->group_rows) return RT_ERR_INVALID_ARGUMENT;
  if (d->out_t && d->ld_out_t < gr) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (d->count == 0) return RT_OK;
  const float3 c = make_float3(0.5f * (d->box_lo[0] + d->box_hi[0]), 0.5f * (d->box_lo[1] + d->box_hi[1]), 0.5f * (d->box_lo[2] + d->box_hi[2]));
  const float3 s = make_float3(2.0f / (d->box_hi[0] - d->box_lo[0]), 2.0f / (d->box_hi[1] - d->box_lo[1]), 2.0f / (d->box_hi[2] - d->box_lo[2]));
  k_ray_features<<<(uint32_t)(((size_t)d->count * 8 + 255) / 256), 256, 0, (cudaStream_t)stream>>>((const float4*)d->orig, (const float4*)d->dir, d->count, c, s,
                                                                           (__nv_bfloat16*)d->out, d->ld_out, (__nv_bfloat16*)d->out_t,
                                                                           d->ld_out_t, gr);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_softmax_xent(const float* logits, uint32_t rows, uint32_t cols, const int32_t* labels, float scale, void* grad_bf16,
                                     float* loss_sum, rt_stream stream) {
  if (!logits || !labels || !grad_bf16 || cols == 0 || cols % 128) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (rows == 0) return RT_OK;
  k_softmax_xent<<<(rows + 7) / 8, 256, 0, (cudaStream_t)stream>>>(logits, rows, cols, labels, scale, (__nv_bfloat16*)grad_bf16, loss_sum);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_transpose_bf16_grouped(const void* in, uint32_t groups, uint32_t rows, uint32_t cols, uint32_t ld_in, void* out,
                                               uint32_t ld_out, rt_stream stream) {
  if (!in || !out || ld_in < cols || ld_out < rows || groups == 0 || groups > 65535u) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (rows == 0 || cols == 0) return RT_OK;
  dim3 grid((cols + 31) / 32, (rows + 31) / 32, groups);
  k_transpose_bf16<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, rows, cols, ld_in, (__nv_bfloat16*)out, ld_out);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_transpose_bf16(const void* in, uint32_t rows, uint32_t cols, uint32_t ld_in, void* out, uint32_t ld_out,
                                       rt_stream stream) {
  return rt_transpose_bf16_grouped(in, 1, rows, cols, ld_in, out, ld_out, stream);
}

extern "C" rt_status rt_colsum_bf16_grouped(const void* in, uint32_t groups, uint32_t rows, uint32_t cols, uint32_t ld, float* out,
                                            rt_stream stream) {
  if (!in || !out || ld < cols || groups == 0 || groups > 65535u) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (cols == 0) return RT_OK;
  if (cols % 2 == 0 && ld % 2 == 0 && ((uintptr_t)in & 3u) == 0 && ((uintptr_t)out & 7u) == 0)
    k_colsum2_bf16<<<dim3((cols + 63) / 64, groups), dim3(32, 8), 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, rows, cols, ld, out);
  else
    k_colsum_bf16<<<dim3((cols + 31) / 32, groups), dim3(32, 8), 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, rows, cols, ld, out);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_colsum_bf16(const void* in, uint32_t rows, uint32_t cols, uint32_t ld, float* out, rt_stream stream) {
  return rt_colsum_bf16_grouped(in, 1, rows, cols, ld, out, stream);
}

extern "C" rt_status rt_gather_batch(const rt_batch_gather_desc* d, rt_stream stream) {
  if (!d || !d->orig || !d->dir || !d->out_orig || !d->out_dir || (d->labels && !d->out_labels) || d->group_stride == 0 ||
      (d->index && !d->index_count))
    return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  const size_t total = (size_t)d->groups * d->batch;
  if (total == 0) return RT_OK;
  const uint32_t blocks = (uint32_t)hmin<size_t>((total + 255) / 256, (size_t)num_sms() * 8);
  k_gather_batch<<<blocks, 256, 0, (cudaStream_t)stream>>>((const float4*)d->orig, (const float4*)d->dir, d->labels, d->groups,
                                                           d->group_stride, d->offset, d->batch, d->hop ? d->hop : 1u, d->index,
                                                           d->index_count, (float4*)d->out_orig, (float4*)d->out_dir, d->out_labels);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_group_select(const int32_t* labels, uint32_t groups, uint32_t group_stride, uint32_t* index, uint32_t* count,
                                     rt_stream stream) {
  if (!labels || !index || !count || groups == 0 || groups > 0x7FFFFFFFu) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  k_group_select<<<groups, 1024, 0, (cudaStream_t)stream>>>(labels, group_stride, index, count);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_adam_step(const rt_adam_desc* d, rt_stream stream) {
  if (!d || !d->param || !d->grad || !d->m || !d->v || d->step == 0) return RT_ERR_INVALID_ARGUMENT;
  const uint32_t G = d->groups ? d->groups : 1u;
  if (d->rows % G) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  const size_t total = (size_t)d->rows * d->cols;
  if (total == 0) return RT_OK;
  const float c1 = 1.0f / (1.0f - powf(d->beta1, (float)d->step));
  const float c2 = 1.0f / (1.0f - powf(d->beta2, (float)d->step));
  const uint32_t gr = G > 1 ? d->rows / G : (d->rows ? d->rows : 1u);
  const bool by4 = d->rows % 4 == 0 && d->cols % 4 == 0 && gr % 4 == 0 && d->ld_bf16_t % 4 == 0 && (!d->out_bf16 || d->ld_bf16 % 4 == 0) &&
                   aligned16(d->param) && aligned16(d->grad) && aligned16(d->m) && aligned16(d->v) &&
                   ((uintptr_t)d->out_bf16 & 7u) == 0 && ((uintptr_t)d->out_bf16_t & 7u) == 0;
  if (d->out_bf16_t && by4) {
    k_adam_t4<<<dim3((d->cols + 31) / 32, (d->rows + 31) / 32), 256, 0, (cudaStream_t)stream>>>(
        d->param, d->grad, d->m, d->v, d->rows, d->cols, d->lr, d->beta1, d->beta2, d->eps, c1, c2, (__nv_bfloat16*)d->out_bf16,
        d->ld_bf16, (__nv_bfloat16*)d->out_bf16_t, d->ld_bf16_t, gr);
  } else if (d->out_bf16_t) {
    k_adam_t<<<dim3((d->cols + 31) / 32, (d->rows + 31) / 32), dim3(32, 8), 0, (cudaStream_t)stream>>>(
        d->param, d->grad, d->m, d->v, d->rows, d->cols, d->lr, d->beta1, d->beta2, d->eps, c1, c2, (__nv_bfloat16*)d->out_bf16,
        d->ld_bf16, (__nv_bfloat16*)d->out_bf16_t, d->ld_bf16_t, gr);
  } else {
    const uint32_t blocks = (uint32_t)hmin<size_t>((total + 255) / 256, (size_t)num_sms() * 8);
    k_adam<<<blocks, 256, 0, (cudaStream_t)stream>>>(d->param, d->grad, d->m, d->v, d->rows, d->cols, d->lr, d->beta1, d->beta2, d->eps,
                                                      c1, c2, (__nv_bfloat16*)d->out_bf16, d->ld_bf16, nullptr, 0, gr);
  }
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}
