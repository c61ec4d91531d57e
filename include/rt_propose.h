/* rt_propose.h -- C ABI of the learned subtree proposal (sm_100a).
 *
 * No reference counterpart: gatouillatpy/cudart has no learned component.
 * These entry points add a proposal in front of rt_trace_closest: a small MLP
 * maps each ray to one BVH subtree (a "slot" of the tree cut at a fixed depth),
 * the traversal tests that subtree first and starts the full traversal with the
 * hit it found as its best so far. The full traversal still runs, so the hit
 * (id, t, u, v) is bit-identical to rt_trace_closest's; only the work changes.
 *
 * Network: 6 inputs (origin scaled to [-1, 1] over a box, unit direction) ->
 * sin/cos(pi 2^j u), j < 12 (144 features, zero-padded to 192) -> 3 x 128 ReLU
 * -> 2^depth logits. BF16 weights [out][in], FP32 biases, FP32 accumulation on
 * the tensor cores (tcgen05, TMA, tensor memory).
 *
 * Groups: several independent networks (one per mesh of a batched build) run
 * in the same launches. A grouped operand stacks the groups' matrices along
 * its rows (group g's rows follow group g - 1's); every group has the same
 * shape. Group g's results equal, bit for bit, an ungrouped call on group g's
 * rows alone.
 */
#ifndef RT_PROPOSE_H
#define RT_PROPOSE_H

#include "rt_core.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RT_PROPOSE_ABI_VERSION 2u
uint32_t rt_propose_abi_version(void);

/* C = alpha * A * B^T (+ bias[n]) (ReLU) (* (mask > 0)), on the tensor cores.
 * A: BF16 [m][lda], B: BF16 [n][ldb], both K-major. m % 128 == 0, k % 64 == 0,
 * n % 16 == 0; lda, ldb multiples of 8; pointers 16-byte aligned. Outputs (any
 * subset): FP32 [m][ldc_f32], BF16 [m][ldc_bf16], BF16 transposed [n][ldct].
 * groups > 1: C_g = A_g B_g^T for g < groups with A [groups m][lda],
 * B [groups n][ldb], bias [groups n], mask and C [groups m][.], and C^T
 * [groups n][ldct] (group g's transpose in rows g n .. g n + n - 1, columns
 * 0 .. m - 1). */
typedef struct rt_gemm_desc {
  const void* a;
  uint32_t lda;
  const void* b;
  uint32_t ldb;
  uint32_t m, n, k;
  float alpha;
  const float* bias;
  uint32_t relu;
  const void* mask; /* BF16 [m][ldmask] or NULL: outputs where mask <= 0 are zeroed (ReLU backward) */
  uint32_t ldmask;
  float* c_f32;
  uint32_t ldc_f32;
  void* c_bf16;
  uint32_t ldc_bf16;
  void* ct_bf16;
  uint32_t ldct;
  uint32_t* error_word; /* optional: RT_DEVERR_WAIT_TIMEOUT */
  uint32_t groups;      /* 0 or 1: one product */
} rt_gemm_desc;
rt_status rt_gemm_bf16(const rt_gemm_desc* d, rt_stream stream);

/* out_index[i] = argmax_j (A B^T + bias)[i][j] (lowest j among equal maxima),
 * out_value[i] = that maximum, out_margin[i] = maximum - second largest value;
 * out_index[i] = -1 when the margin is below min_margin. The m x n logits are
 * never stored. m % 128 == 0, n % 256 == 0, n <= 4096, k % 64 == 0, k <= 256.
 * groups > 1: A [groups m], B [groups n], bias [groups n], outputs [groups m];
 * a row of group g is scored against group g's n rows of B (indices 0 .. n - 1). */
typedef struct rt_gemm_argmax_desc {
  const void* a;
  uint32_t lda;
  const void* b;
  uint32_t ldb;
  uint32_t m, n, k;
  const float* bias;
  float min_margin;
  int32_t* out_index;
  float* out_value;  /* optional */
  float* out_margin; /* optional */
  uint32_t* error_word;
  uint32_t groups; /* 0 or 1: one product */
} rt_gemm_argmax_desc;
rt_status rt_gemm_argmax_bf16(const rt_gemm_argmax_desc* d, rt_stream stream);

/* The whole proposal network in one launch: features, three hidden layers
 * and the argmax over n logits for each ray, bit-identical to rt_ray_features
 * + 3 x rt_gemm_bf16 (bias, ReLU, BF16 outputs) + rt_gemm_argmax_bf16, with no
 * activation written to memory. Weights BF16, rows contiguous: w1 [groups 128][192],
 * w2, w3 [groups 128][128], w4 [groups n][128]; biases FP32 [groups 128] (b1..b3),
 * [groups n] (b4); all pointers 16-byte aligned. n % 256 == 0, n <= 4096. groups > 1: ray r belongs to group
 * r / group_rows (group_rows % 128 == 0, count == groups * group_rows).
 * tmax (optional): rays with tmax <= 0 (inactive: a bounce of a ray that
 * missed) get -1, and a tile of 128 rays that are all inactive costs no MMA. */
typedef struct rt_mlp_propose_desc {
  const float* orig; /* float4 per ray */
  const float* dir;
  uint32_t count;
  float box_lo[3], box_hi[3];
  const void* w1;
  const void* w2;
  const void* w3;
  const void* w4;
  const float* b1;
  const float* b2;
  const float* b3;
  const float* b4;
  uint32_t n;
  uint32_t groups, group_rows;
  float min_margin;
  int32_t* out_index;
  float* out_value;  /* optional */
  float* out_margin; /* optional */
  uint32_t* error_word;
  const float* tmax; /* optional */
} rt_mlp_propose_desc;
rt_status rt_mlp_propose(const rt_mlp_propose_desc* d, rt_stream stream);

/* Softmax cross-entropy gradient of the logits A B^T + bias without storing
 * them: g[r][j] = (softmax(row r)_j - [j == labels[r]]) * scale in BF16, written
 * row-major (g, [m][ldg]) and transposed (gt, [n][ldgt]); *loss_sum +=
 * scale * (logsumexp(row r) - logit[labels[r]]). Rows whose label is outside
 * [0, n) get g = 0 and add no loss. m % 128 == 0, n % 256 == 0, n <= 4096,
 * k % 64 == 0, k <= 256, ldg % 8 == 0. groups > 1 as for rt_gemm_argmax_bf16;
 * group q's transpose fills rows q n .. q n + n - 1 of gt, columns 0 .. m - 1. */
typedef struct rt_gemm_xent_desc {
  const void* a;
  uint32_t lda;
  const void* b;
  uint32_t ldb;
  uint32_t m, n, k;
  const float* bias;
  const int32_t* labels;
  float scale;
  void* g;
  uint32_t ldg;
  void* gt;
  uint32_t ldgt;
  float* loss_sum; /* optional, accumulated */
  uint32_t* error_word;
  uint32_t groups;
} rt_gemm_xent_desc;
rt_status rt_gemm_xent_bf16(const rt_gemm_xent_desc* d, rt_stream stream);

/* Self-test of the bounded waits of the tensor-core kernels: one warp
 * allocates 32 TMEM columns, waits on a shared-memory barrier that nothing
 * arrives at for limit_us microseconds (1 .. 2,000,000), then releases the TMEM
 * and returns. Results (DEVICE): RT_DEVERR_WAIT_TIMEOUT is OR-ed into
 * *error_word; result[0] = 1 if the wait completed (it cannot), else 0;
 * result[1] = microseconds the kernel waited. The context stays usable. */
rt_status rt_tc_wait_selftest(uint32_t limit_us, uint32_t* error_word, uint32_t* result, rt_stream stream);

/* Ray features: u = ((o - c) * 2 / (hi - lo), d / |d|), c = (lo + hi) / 2;
 * f[24 i + 2 j] = sin(pi 2^j u_i), f[24 i + 2 j + 1] = cos(pi 2^j u_i), j < 12;
 * columns 144 .. 191 are zero. out: BF16 [count][ld_out] (ld_out >= 192, a
 * multiple of 8; 16-byte aligned); out_t: BF16 [192][ld_out_t] (rows 144..191
 * zero). group_rows > 0 (count % group_rows == 0): out_t holds one transpose
 * per group of group_rows rays, group g in rows 192 g .. 192 g + 191, columns
 * 0 .. group_rows - 1 (ld_out_t >= group_rows). */
typedef struct rt_feature_desc {
  const float* orig; /* float4 per ray */
  const float* dir;  /* float4 per ray */
  uint32_t count;
  float box_lo[3], box_hi[3];
  void* out;
  uint32_t ld_out;
  void* out_t;
  uint32_t ld_out_t;
  uint32_t group_rows; /* 0: one group of count rays */
} rt_feature_desc;
rt_status rt_ray_features(const rt_feature_desc* d, rt_stream stream);

/* grad[r][j] = (softmax(logits[r])_j - [j == labels[r]]) * scale (BF16), rows
 * with a label outside [0, cols) get 0; *loss_sum += scale * (logsumexp - logit[label]).
 * cols % 128 == 0. */
rt_status rt_softmax_xent(const float* logits, uint32_t rows, uint32_t cols, const int32_t* labels, float scale, void* grad_bf16,
                          float* loss_sum, rt_stream stream);
/* out[c][r] = in[r][c] (BF16). */
rt_status rt_transpose_bf16(const void* in, uint32_t rows, uint32_t cols, uint32_t ld_in, void* out, uint32_t ld_out, rt_stream stream);
/* out[c] = sum_r in[r][c] (BF16 in, FP32 out; out is overwritten; the
 * summation order is fixed, so the result is deterministic). */
rt_status rt_colsum_bf16(const void* in, uint32_t rows, uint32_t cols, uint32_t ld, float* out, rt_stream stream);
/* Grouped forms: group g's input rows are g rows .. g rows + rows - 1; its
 * output rows (transpose) are g cols .. g cols + cols - 1, and its column sums
 * out[g cols + c]. */
rt_status rt_transpose_bf16_grouped(const void* in, uint32_t groups, uint32_t rows, uint32_t cols, uint32_t ld_in, void* out,
                                    uint32_t ld_out, rt_stream stream);
rt_status rt_colsum_bf16_grouped(const void* in, uint32_t groups, uint32_t rows, uint32_t cols, uint32_t ld, float* out,
                                 rt_stream stream);

/* Training batch of grouped networks. Row g batch + b of the outputs (origin,
 * direction, label) is input row g group_stride + q with
 *   k = ((offset + b) * hop) mod n_g  (hop 0 counts as 1),
 *   q = index[g group_stride + k], n_g = index_count[g]  with an index list,
 *   q = k, n_g = group_stride                            without;
 * a group whose list is empty gives zero rays labelled -1. */
typedef struct rt_batch_gather_desc {
  const float* orig; /* float4 per ray */
  const float* dir;
  const int32_t* labels;
  uint32_t groups, group_stride, offset, batch;
  float* out_orig;
  float* out_dir;
  int32_t* out_labels;
  const uint32_t* index;       /* optional [groups][group_stride] (rt_group_select) */
  const uint32_t* index_count; /* [groups], with index */
  uint32_t hop;
} rt_batch_gather_desc;
rt_status rt_gather_batch(const rt_batch_gather_desc* d, rt_stream stream);

/* Per group g: index[g group_stride + k] = the k-th row r (ascending) with
 * labels[g group_stride + r] >= 0; count[g] = how many. */
rt_status rt_group_select(const int32_t* labels, uint32_t groups, uint32_t group_stride, uint32_t* index, uint32_t* count,
                          rt_stream stream);

/* One Adam step (bias-corrected, step >= 1) on FP32 parameters [rows][cols];
 * refreshes BF16 copies [rows][ld_bf16] and [cols][ld_bf16_t] when given. */
typedef struct rt_adam_desc {
  float* param;
  const float* grad;
  float* m;
  float* v;
  uint32_t rows, cols;
  float lr, beta1, beta2, eps;
  uint32_t step;
  void* out_bf16;
  uint32_t ld_bf16;
  void* out_bf16_t;
  uint32_t ld_bf16_t;
  uint32_t groups; /* > 1: rows hold groups stacked matrices; out_bf16_t holds their transposes stacked (group g in rows g cols ..) */
} rt_adam_desc;
rt_status rt_adam_step(const rt_adam_desc* d, rt_stream stream);

/* Slots of a built tree cut at `depth` (1..16): slot s follows the bits of s
 * (most significant first, 0 = left child) from the root for `depth` levels
 * or until a leaf. slot_ref[s] = traversal-blob reference of the node reached
 * (int32 bits of the blob's child reference). A slot is the "first" slot of
 * its node when the bits below the node's depth are zero; pos_label[p] = the
 * first slot of the node holding face position p. */
typedef struct rt_slot_desc {
  const uint32_t* nodes; /* bvnode array of rt_lbvh_build */
  const void* accel;     /* traversal blob of the same build */
  uint32_t face_count;
  uint32_t depth;
  int32_t* slot_ref;  /* [2^depth] */
  float* slot_box;    /* [2^depth][8], optional: padded box of the slot's node (min xyz, 0, max xyz, 0) */
  int32_t* pos_label; /* [face_count], optional */
  uint32_t* slot_first; /* [2^depth], optional: first face position of the slot's node (first slots), else 0 */
  uint32_t* slot_count; /* [2^depth], optional: face count of the slot's node (first slots), else 0 */
} rt_slot_desc;
rt_status rt_subtree_slots(const rt_slot_desc* d, rt_stream stream);

/* labels[r] = pos_label[hit_pos[r]] for hits (hit_pos >= 0), -1 for misses. */
rt_status rt_hit_labels(const int32_t* hit_pos, uint32_t count, const int32_t* pos_label, int32_t* labels, rt_stream stream);

/* rt_trace_closest (blob path, d->accel and d->tris required) where ray r first
 * walks the subtree slot_ref[proposal[r]] (proposal[r] < 0 or >= slot_count:
 * none), then the whole tree minus that subtree, starting from the best hit the
 * first walk found. With slot_box, a ray that misses the proposed node's box
 * skips the first walk (one box read). Outputs are bit-identical to
 * rt_trace_closest's. */
typedef struct rt_seed_desc {
  const int32_t* proposal;
  const int32_t* slot_ref;
  const float* slot_box; /* optional, rt_slot_desc.slot_box of the same tree */
  uint32_t slot_count;
  int32_t* in_proposal; /* optional [ray_count]: 1 when the final hit lies in the proposed subtree */
} rt_seed_desc;
rt_status rt_trace_closest_seeded(const rt_trace_desc* d, const rt_seed_desc* s, rt_stream stream);

/* Batched forms over the trees of rt_batch_build (mesh m: faces
 * face_offsets[m] .. face_offsets[m + 1], rays ray_offsets[m] .. ray_offsets[m + 1]).
 * Slot tables are per mesh: slot_ref [mesh_count][2^depth], slot_box
 * [mesh_count][2^depth][8], slot_first / slot_count likewise; pos_label is
 * indexed by the global face position and holds mesh-local slots. */
typedef struct rt_batch_slot_desc {
  uint32_t mesh_count;
  const uint32_t* face_offsets; /* DEVICE [mesh_count + 1] */
  const uint32_t* nodes;        /* of rt_batch_build */
  const void* accel;            /* of rt_batch_build */
  uint32_t face_count;          /* total */
  uint32_t depth;
  int32_t* slot_ref;
  float* slot_box;   /* optional */
  int32_t* pos_label; /* optional [face_count] */
  uint32_t* slot_first; /* optional */
  uint32_t* slot_count; /* optional */
} rt_batch_slot_desc;
rt_status rt_batch_subtree_slots(const rt_batch_slot_desc* d, rt_stream stream);

/* labels[r] = pos_label[face_offsets[m] + hit_pos[r]] for the rays r of mesh m
 * that hit (mesh-local positions, as rt_batch_trace writes them), -1 for misses. */
rt_status rt_batch_hit_labels(const int32_t* hit_pos, uint32_t ray_count, uint32_t mesh_count, const uint32_t* ray_offsets,
                              const uint32_t* face_offsets, const int32_t* pos_label, int32_t* labels, rt_stream stream);

/* rt_batch_trace where ray r of mesh m first walks the subtree
 * slot_ref[m slot_count + proposal[r]] (s->slot_ref, s->slot_box per mesh as
 * above); outputs bit-identical to rt_batch_trace's. */
rt_status rt_batch_trace_seeded(const rt_batch_trace_desc* d, const rt_seed_desc* s, rt_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* RT_PROPOSE_H */
