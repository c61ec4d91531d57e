// rt_propose.cu -- the tree side of the learned proposal: the slot table of a
// built tree (which node each of the 2^depth slots reaches, as a traversal-blob
// reference) and per-face-position labels, from which a traced ray's label is
// read off its hit position.
//
// A slot s follows the bits of s from the root, most significant first (0 =
// left child), for `depth` levels or until a leaf. When a leaf is reached at a
// depth d < depth, every slot sharing those d bits maps to that leaf, and its
// label is the first of them (the low depth - d bits zero).
#include "../../include/rt_propose.h"
#include "rt_device.cuh"

namespace rt {
namespace {

struct SlotOut {
  int32_t* slot_ref;
  float4* slot_box;
  int32_t* pos_label;
  uint32_t* slot_first;
  uint32_t* slot_count;
};

// Slot s of one tree: nodes / hdr / tnodes of that tree (node ids, blob
// references and face positions local to it).
__device__ void subtree_slot(const uint32_t* __restrict__ nodes, const uint32_t* __restrict__ hdr, const float4* __restrict__ tnodes,
                             uint32_t depth, uint32_t s, const SlotOut& O) {
  int32_t* const slot_ref = O.slot_ref;
  float4* const slot_box = O.slot_box;
  int32_t* const pos_label = O.pos_label;
  uint32_t* const slot_first = O.slot_first;
  uint32_t* const slot_count = O.slot_count;
  uint32_t x = 0, ref = hdr[0], d = 0;
  // the root has no parent record: its box is everything
  float4 bmin = make_float4(-kHuge, -kHuge, -kHuge, 0.0f), bmax = make_float4(kHuge, kHuge, kHuge, 0.0f);
  while (d < depth) {
    const uint2 w = *(const uint2*)(nodes + 8 * (size_t)x);
    if (w.x & 1u) break;  // leaf
    const uint32_t bit = (s >> (depth - 1 - d)) & 1u;
    const float4* tn = tnodes + 4 * (size_t)ref + 2 * bit;
    const float4 c0 = tn[0], c1 = tn[1];
    ref = __float_as_uint(c0.w);
    bmin = make_float4(c0.x, c0.y, c0.z, 0.0f);
    bmax = make_float4(c1.x, c1.y, c1.z, 0.0f);
    x = w.y + bit;
    ++d;
  }
  slot_ref[s] = (int32_t)ref;
  if (slot_box) {
    slot_box[2 * s] = bmin;
    slot_box[2 * s + 1] = bmax;
  }
  const bool first = (s & ((1u << (depth - d)) - 1u)) == 0u;
  uint32_t lo = 0, hi = 0;
  if (first) {
    uint32_t y = x;
    for (;;) {
      const uint2 w = *(const uint2*)(nodes + 8 * (size_t)y);
      if (w.x & 1u) { lo = w.y; break; }
      y = w.y;
    }
    y = x;
    for (;;) {
      const uint2 w = *(const uint2*)(nodes + 8 * (size_t)y);
      if (w.x & 1u) { hi = w.y + (w.x >> 1); break; }
      y = w.y + 1;
    }
    if (pos_label)
      for (uint32_t p = lo; p < hi; ++p) pos_label[p] = (int32_t)s;
  }
  if (slot_first) slot_first[s] = lo;
  if (slot_count) slot_count[s] = hi - lo;
}

__global__ __launch_bounds__(128) void k_subtree_slots(const uint32_t* __restrict__ nodes, const uint32_t* __restrict__ hdr,
                                                       const float4* __restrict__ tnodes, uint32_t depth, SlotOut O) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < (1u << depth)) subtree_slot(nodes, hdr, tnodes, depth, s, O);
}

// blockIdx.y = mesh of a batched build; its nodes start at 2 F - m, its blob
// header at 64 m words, its two-child records at 4 F float4s (F = faces before m).
__global__ __launch_bounds__(128) void k_batch_subtree_slots(const uint32_t* __restrict__ foff, const uint32_t* __restrict__ nodes,
                                                             BatchAccel acc, uint32_t depth, SlotOut O) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x, m = blockIdx.y;
  const uint32_t S = 1u << depth;
  if (s >= S) return;
  const uint32_t F = __ldg(foff + m);
  SlotOut Om;
  const size_t so = (size_t)m * S;
  Om.slot_ref = O.slot_ref + so;
  Om.slot_box = O.slot_box ? O.slot_box + 2 * so : nullptr;
  Om.pos_label = O.pos_label ? O.pos_label + F : nullptr;
  Om.slot_first = O.slot_first ? O.slot_first + so : nullptr;
  Om.slot_count = O.slot_count ? O.slot_count + so : nullptr;
  subtree_slot(nodes + 8 * (size_t)node_base(F, m), acc.hdr + 64 * (size_t)m, acc.tnodes + 4 * (size_t)F, depth, s, Om);
}

__global__ __launch_bounds__(256) void k_hit_labels(const int32_t* __restrict__ hit_pos, uint32_t count, const int32_t* __restrict__ pos_label,
                                                    int32_t* __restrict__ labels) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < count; r += gridDim.x * blockDim.x) {
    const int32_t p = hit_pos[r];
    labels[r] = p >= 0 ? __ldg(pos_label + p) : -1;
  }
}

__global__ __launch_bounds__(256) void k_batch_hit_labels(const int32_t* __restrict__ hit_pos, uint32_t count, uint32_t M,
                                                          const uint32_t* __restrict__ roff, const uint32_t* __restrict__ foff,
                                                          const int32_t* __restrict__ pos_label, int32_t* __restrict__ labels) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < count; r += gridDim.x * blockDim.x) {
    const int32_t p = hit_pos[r];
    labels[r] = p >= 0 ? __ldg(pos_label + __ldg(foff + find_seg(roff, M, r)) + p) : -1;
  }
}

}  // namespace
}  // namespace rt

using namespace rt;

extern "C" rt_status rt_subtree_slots(const rt_slot_desc* d, rt_stream stream) {
  if (!d || !d->nodes || !d->accel || !d->slot_ref || d->depth < 1 || d->depth > 16 || d->face_count == 0) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  // blob layout of rt_lbvh_build: header (256 B), then the two-child records
  Carve c((void*)d->accel, ~(size_t)0);
  const uint32_t* hdr = c.take<uint32_t>(64);
  const float4* tnodes = c.take<float4>(4 * (size_t)d->face_count);
  const uint32_t slots = 1u << d->depth;
  const SlotOut O{d->slot_ref, (float4*)d->slot_box, d->pos_label, d->slot_first, d->slot_count};
  k_subtree_slots<<<(slots + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d->nodes, hdr, tnodes, d->depth, O);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_hit_labels(const int32_t* hit_pos, uint32_t count, const int32_t* pos_label, int32_t* labels, rt_stream stream) {
  if (!hit_pos || !pos_label || !labels) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (count == 0) return RT_OK;
  const uint32_t blocks = (uint32_t)hmin<uint32_t>((count + 255) / 256, 148u * 16u);
  k_hit_labels<<<blocks, 256, 0, (cudaStream_t)stream>>>(hit_pos, count, pos_label, labels);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_batch_subtree_slots(const rt_batch_slot_desc* d, rt_stream stream) {
  if (!d || !d->face_offsets || !d->nodes || !d->accel || !d->slot_ref || d->depth < 1 || d->depth > 16 || d->mesh_count == 0 ||
      d->mesh_count > 65535u || d->face_count < d->mesh_count)
    return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  Carve c((void*)d->accel, ~(size_t)0);
  BatchAccel acc;
  carve_batch_accel_layout(c, acc, d->mesh_count, d->face_count);
  const uint32_t slots = 1u << d->depth;
  const SlotOut O{d->slot_ref, (float4*)d->slot_box, d->pos_label, d->slot_first, d->slot_count};
  k_batch_subtree_slots<<<dim3((slots + 127) / 128, d->mesh_count), 128, 0, (cudaStream_t)stream>>>(d->face_offsets, d->nodes, acc,
                                                                                                    d->depth, O);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}

extern "C" rt_status rt_batch_hit_labels(const int32_t* hit_pos, uint32_t ray_count, uint32_t mesh_count, const uint32_t* ray_offsets,
                                         const uint32_t* face_offsets, const int32_t* pos_label, int32_t* labels, rt_stream stream) {
  if (!hit_pos || !ray_offsets || !face_offsets || !pos_label || !labels || mesh_count == 0) return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (ray_count == 0) return RT_OK;
  const uint32_t blocks = (uint32_t)hmin<uint32_t>((ray_count + 255) / 256, 148u * 16u);
  k_batch_hit_labels<<<blocks, 256, 0, (cudaStream_t)stream>>>(hit_pos, ray_count, mesh_count, ray_offsets, face_offsets, pos_label,
                                                               labels);
  note_launch();
  RT_CHECK_LAUNCH();
  return RT_OK;
}
