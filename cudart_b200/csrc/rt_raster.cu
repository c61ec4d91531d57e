// rt_raster.cu -- the rasteriser (CUDA_rasterizeMeshTree,
// kernels/CUDA_rasterizeMeshTree.cu:77-297) on sm_100a.
//
// The reference runs 2 x 2 blocks of 8 x 4 threads over the whole screen,
// each block walking every face through a 192-face shared-memory cache. Here
// the work is binned instead: one thread per face transforms its vertices,
// drops faces off screen (and faces the barycentric test always rejects) and
// computes the reference's zone rectangle; every face is appended to the list
// of each zone of its rectangle (a counting sort: count, scan, fill); then one
// warp per 8 x 4 zone (lane = pixel, the reference's thread layout) walks its
// zone's faces, keeping depth / id / (u, v) in registers and taking the
// minimum (depth, face index). The per-pixel result is the reference's: the
// same tests on the same faces, and the face the reference's index-order walk
// with a strict depth test keeps. Faces are processed in chunks, in index
// order, whose pair count fits the scratch (a face can cover many zones); the
// surfaces carry the state across chunks.
#include <cstring>
#include <vector>

#include "../../include/rt_raster.h"
#include "rt_device.cuh"

namespace rt {
namespace {

constexpr float kRasterEps = 0.000001f;  // EPSILON, :31
constexpr uint32_t kFacesPerBlock = 128;  // granularity of the chunking
constexpr uint32_t kMinPairCap = 16u << 20;

struct Mat4 {
  float4 r0, r1, r2, r3;
};

__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// matrixTransform, then /= |w| (a multiply by the reciprocal), w = 0 (:112-117)
__device__ __forceinline__ float4 project(const Mat4& m, float4 v) {
  v.w = 1.0f;
  float4 o = make_float4(dot4(m.r0, v), dot4(m.r1, v), dot4(m.r2, v), dot4(m.r3, v));
  const float inv = 1.0f / fabsf(o.w);
  o = make_float4(o.x * inv, o.y * inv, o.z * inv, o.w * inv);
  o.w = 0.0f;
  return o;
}

struct Zones {
  int zcx, zcy;
  float zsx, zsy;  // zone_scale = 0.5 * zone_count (:94-95)
};

// Per face: projected vertices, the zone rectangle (x0, y0, x1, y1) and the
// number of zones it covers (0 when dropped). Faces naming a vertex past the
// mesh are skipped with an error bit.
__global__ __launch_bounds__(256) void k_raster_setup(const float4* __restrict__ verts, uint32_t vcount, const uint4* __restrict__ faces,
                                                      uint32_t n, Mat4 M, Zones Z, float4* __restrict__ tri, int4* __restrict__ rect,
                                                      uint32_t* __restrict__ cnt, uint32_t* __restrict__ block_sum, uint32_t* err) {
  __shared__ uint32_t s_sum;
  if (threadIdx.x == 0) s_sum = 0;
  __syncthreads();
  const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t c = 0;
  if (f < n) {
    const uint4 fc = __ldg(faces + f);
    if (fc.x >= vcount || fc.y >= vcount || fc.z >= vcount) {
      atomicOr(err, (uint32_t)RT_DEVERR_NODE_CAPACITY);
    } else {
      float4 a = project(M, __ldg(verts + fc.x));
      const float4 b = project(M, __ldg(verts + fc.y)), cc = project(M, __ldg(verts + fc.z));
      // the face's determinant (intersectTriPoint, :52-71, the same arithmetic as the
      // zone pass would do per pixel): a face the test always rejects gets no zone
      // pairs; otherwise its reciprocal rides in a.w
      const float det = (b.x - a.x) * (cc.y - a.y) - (cc.x - a.x) * (b.y - a.y);
      const bool degenerate = det > -kRasterEps && det < kRasterEps;
      a.w = degenerate ? 0.0f : 1.0f / det;
      tri[3 * (size_t)f] = a;
      tri[3 * (size_t)f + 1] = b;
      tri[3 * (size_t)f + 2] = cc;
      const float mnx = fminf(fminf(fminf(kHuge, a.x), b.x), cc.x), mny = fminf(fminf(fminf(kHuge, a.y), b.y), cc.y);
      const float mxx = fmaxf(fmaxf(fmaxf(-kHuge, a.x), b.x), cc.x), mxy = fmaxf(fmaxf(fmaxf(-kHuge, a.y), b.y), cc.y);
      // intersectRectRect with [-1, 1]^2 (:47-50, :150)
      if (!degenerate && mnx < 1.0f && mxx > -1.0f && mny < 1.0f && mxy > -1.0f) {
        const int x0 = max(__float2int_rz(Z.zsx * (mnx + 1.0f)), 0) / 2 * 2;
        const int y0 = max(__float2int_rz(Z.zsy * (1.0f - mxy)), 0) / 2 * 2;
        const int x1 = min(__float2int_rz(Z.zsx * (mxx + 1.0f)), Z.zcx - 1);
        const int y1 = min(__float2int_rz(Z.zsy * (1.0f - mny)), Z.zcy - 1);
        rect[f] = make_int4(x0, y0, x1, y1);
        if (x1 >= x0 && y1 >= y0) c = (uint32_t)(x1 - x0 + 1) * (uint32_t)(y1 - y0 + 1);
      }
    }
    cnt[f] = c;
  }
  // per block of kFacesPerBlock faces (= blockDim) the pair count, for the host's chunking
  atomicAdd(&s_sum, c);
  __syncthreads();
  if (threadIdx.x == 0) block_sum[blockIdx.x] = s_sum;
}

// (zone, face) pairs of faces [f0, f1) at their offsets, in face order.
// The (zone, face) pairs of faces [f0, f1) binned by zone without a sort:
// k_raster_count counts each zone's faces, an exclusive scan turns the counts
// into list starts, and k_raster_fill appends every face to its zones' lists.
// The order inside a list is whatever the atomics give; the zone pass takes
// the minimum (depth, face index), which is what visiting the faces in index
// order with a strict depth test keeps.
__global__ __launch_bounds__(256) void k_raster_count(const int4* __restrict__ rect, const uint32_t* __restrict__ cnt, uint32_t f0,
                                                      uint32_t f1, int zcx, uint32_t* __restrict__ zcount) {
  for (uint32_t f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
    if (!cnt[f]) continue;
    const int4 r = rect[f];
    for (int j = r.y; j <= r.w; ++j)
      for (int i = r.x; i <= r.z; ++i) atomicAdd(zcount + (uint32_t)(j * zcx + i), 1u);
  }
}
__global__ __launch_bounds__(256) void k_raster_fill(const int4* __restrict__ rect, const uint32_t* __restrict__ cnt, uint32_t f0,
                                                     uint32_t f1, int zcx, const uint32_t* __restrict__ zoff, uint32_t* __restrict__ zfill,
                                                     uint32_t* __restrict__ vals) {
  for (uint32_t f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
    const uint32_t c = cnt[f];
    if (!c) continue;
    const int4 r = rect[f];
    int i = r.x, j = r.y;
    // four zones at a time: their atomics are in flight together before the stores
    for (uint32_t q = 0; q < c; q += 4) {
      uint32_t z[4], pos[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        z[k] = q + k < c ? (uint32_t)(j * zcx + i) : ~0u;
        if (++i > r.z) { i = r.x; ++j; }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (z[k] != ~0u) pos[k] = zoff[z[k]] + atomicAdd(zfill + z[k], 1u);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (z[k] != ~0u) vals[pos[k]] = f;
    }
  }
}

// One warp per zone; lane = pixel (x = lane % 8, y = lane / 8 inside the zone).
__global__ __launch_bounds__(256) void k_raster_zones(const float4* __restrict__ tri, const uint32_t* __restrict__ vals,
                                                      const uint32_t* __restrict__ zs, const uint32_t* __restrict__ ze, uint32_t nz,
                                                      int zcx, int width, int height, uint32_t id_mode, int32_t* __restrict__ fid,
                                                      float2* __restrict__ uv, float* __restrict__ depth) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t z = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; z < nz; z += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t s = zs[z], e = ze[z];
    if (s >= e) continue;
    const int x = (int)(z % (uint32_t)zcx) * 8 + (int)(lane & 7u);
    const int y = (int)(z / (uint32_t)zcx) * 4 + (int)(lane >> 3);
    const bool inside = x >= 0 && x < width && y >= 0 && y < height;
    const size_t l = (size_t)y * (size_t)width + (size_t)x;
    const float px = (float)x * 2.0f / (float)width - 1.0f;
    const float py = 1.0f - (float)y * 2.0f / (float)height;
    float best = inside ? depth[l] : 0.0f;
    int32_t bf = -1;
    float bu = 0.0f, bv = 0.0f;
    for (uint32_t p = s; p < e; ++p) {
      const uint32_t f = __ldg(vals + p);
      const float4 a = __ldg(tri + 3 * (size_t)f), b = __ldg(tri + 3 * (size_t)f + 1), c = __ldg(tri + 3 * (size_t)f + 2);
      // intersectTriPoint (:52-71); the face setup pass computed 1 / det (a.w) and
      // emitted no pairs for faces with |det| below the threshold
      const float inv_det = a.w;
      const float u = ((c.x - px) * (a.y - py) - (a.x - px) * (c.y - py)) * inv_det;
      if (u < 0.0f || u > 1.0f) continue;
      const float v = ((a.x - px) * (b.y - py) - (b.x - px) * (a.y - py)) * inv_det;
      if (v < 0.0f || u + v > 1.0f) continue;
      const float t = (1.0f - u - v) * a.z + u * b.z + v * c.z;
      // the earliest face wins a depth tie: faces arrive in any order, and the
      // depth of an earlier chunk (bf < 0) is only beaten by a strictly nearer face
      if (inside && t > 0 && (t < best || (t == best && bf >= 0 && (int32_t)f < bf))) {
        best = t;
        bf = (int32_t)f;
        bu = u;
        bv = v;
      }
    }
    if (bf >= 0) {
      fid[l] = id_mode == 1 ? bf - bf % 192 : bf;
      uv[l] = make_float2(bu, bv);
      depth[l] = best;
    }
  }
}

int sm_count_r() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

Zones zones_of(uint32_t width, uint32_t height) {
  Zones Z;
  Z.zcx = 1 + ((int)width - 1) / 8;
  Z.zcy = 1 + ((int)height - 1) / 4;
  Z.zsx = 0.5f * (float)Z.zcx;
  Z.zsy = 0.5f * (float)Z.zcy;
  return Z;
}

struct RasterLayout {
  float4* tri;
  int4* rect;
  uint32_t *cnt, *block_sum, *vals, *zoff, *zfill, *zsums, *err;
  uint32_t cap;
};

size_t carve_raster(Carve& c, RasterLayout& L, uint32_t n, uint32_t width, uint32_t height, uint32_t pair_capacity) {
  const Zones Z = zones_of(width, height);
  const uint64_t nz = (uint64_t)Z.zcx * (uint64_t)Z.zcy;
  uint64_t cap = pair_capacity ? pair_capacity : kMinPairCap;
  if (cap < (uint64_t)kFacesPerBlock * nz) cap = (uint64_t)kFacesPerBlock * nz;  // one block of faces always fits
  L.cap = (uint32_t)(cap > 0x7FFFFFFFull ? 0x7FFFFFFFull : cap);
  L.tri = c.take<float4>(3 * (size_t)n);
  L.rect = c.take<int4>(n);
  L.cnt = c.take<uint32_t>(n);
  L.block_sum = c.take<uint32_t>(n / kFacesPerBlock + 1);
  L.vals = c.take<uint32_t>(L.cap);
  L.zoff = c.take<uint32_t>(nz + 1);
  L.zfill = c.take<uint32_t>(nz);
  L.zsums = c.take<uint32_t>(nz / 1024 + 2);
  L.err = c.take<uint32_t>(1);
  return c.off + 256;
}

}  // namespace
}  // namespace rt

using namespace rt;

extern "C" rt_status rt_raster_scratch_bytes(uint32_t face_count, uint32_t width, uint32_t height, uint32_t pair_capacity, size_t* bytes) {
  if (!bytes || face_count == 0 || width == 0 || height == 0 || face_count > 0x7FFFFFFFu) return RT_ERR_INVALID_ARGUMENT;
  Carve c(nullptr, 0);
  RasterLayout L;
  *bytes = carve_raster(c, L, face_count, width, height, pair_capacity);
  return RT_OK;
}

extern "C" rt_status rt_rasterize(const rt_raster_desc* d, rt_stream stream) {
  if (!d || !d->vertices || !d->faces || !d->face_id || !d->uv || !d->depth || d->width == 0 || d->height == 0 || d->id_mode > 1)
    return RT_ERR_INVALID_ARGUMENT;
  if (rt_device_check() != RT_OK) return RT_ERR_NO_DEVICE;
  if (d->face_count == 0) return RT_OK;
  size_t need = 0;
  rt_raster_scratch_bytes(d->face_count, d->width, d->height, d->pair_capacity, &need);
  if (!d->scratch || d->scratch_bytes < need) return RT_ERR_SCRATCH_TOO_SMALL;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t n = d->face_count;
  Carve c(d->scratch, d->scratch_bytes);
  RasterLayout L;
  carve_raster(c, L, n, d->width, d->height, d->pair_capacity);
  const Zones Z = zones_of(d->width, d->height);
  const uint32_t nz = (uint32_t)Z.zcx * (uint32_t)Z.zcy;
  Mat4 M;
  memcpy(&M, d->matrix, 64);
  uint32_t* err = d->error_word ? d->error_word : L.err;
  if (!d->error_word && cudaMemsetAsync(L.err, 0, 4, st) != cudaSuccess) return RT_ERR_CUDA;
  const uint32_t nblocks = (n + kFacesPerBlock - 1) / kFacesPerBlock;
  k_raster_setup<<<nblocks, kFacesPerBlock, 0, st>>>((const float4*)d->vertices, d->vertex_count, (const uint4*)d->faces, n, M, Z, L.tri,
                                                      L.rect, L.cnt, L.block_sum, err);
  note_launch();
  RT_CHECK_LAUNCH();
  std::vector<uint32_t> bsum(nblocks);
  if (cudaMemcpyAsync(bsum.data(), L.block_sum, (size_t)nblocks * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return RT_ERR_CUDA;
  const int sms = sm_count_r();
  uint32_t b = 0;
  while (b < nblocks) {
    // the longest run of face blocks whose pairs fit the pair buffer
    uint64_t P = 0;
    uint32_t e = b;
    while (e < nblocks && P + bsum[e] <= L.cap) P += bsum[e++];
    if (e == b) return RT_ERR_CAPACITY;  // cannot happen: one block's pairs always fit
    const uint32_t f0 = b * kFacesPerBlock, f1 = e * kFacesPerBlock < n ? e * kFacesPerBlock : n;
    b = e;
    if (P == 0) continue;
    const uint32_t fblocks = (uint32_t)hmin<uint64_t>((f1 - f0 + 255) / 256, (uint64_t)sms * 8);
    if (cudaMemsetAsync(L.zoff, 0, ((size_t)nz + 1) * 4, st) != cudaSuccess || cudaMemsetAsync(L.zfill, 0, (size_t)nz * 4, st) != cudaSuccess)
      return RT_ERR_CUDA;
    k_raster_count<<<fblocks, 256, 0, st>>>(L.rect, L.cnt, f0, f1, Z.zcx, L.zoff);
    note_launch();
    RT_CHECK_LAUNCH();
    excl_scan(L.zoff, nz + 1, L.zsums, nullptr, st);
    k_raster_fill<<<fblocks, 256, 0, st>>>(L.rect, L.cnt, f0, f1, Z.zcx, L.zoff, L.zfill, L.vals);
    note_launch();
    RT_CHECK_LAUNCH();
    k_raster_zones<<<(uint32_t)hmin<uint64_t>(((uint64_t)nz * 32 + 255) / 256, (uint64_t)sms * 16), 256, 0, st>>>(
        L.tri, L.vals, L.zoff, L.zoff + 1, nz, Z.zcx, (int)d->width, (int)d->height, d->id_mode, d->face_id, (float2*)d->uv, d->depth);
    note_launch();
    RT_CHECK_LAUNCH();
  }
  return RT_OK;
}
