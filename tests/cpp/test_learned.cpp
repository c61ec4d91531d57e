// test_learned.cpp -- C++ host code driving the learned subtree proposal
// through the C ABI of include/rt_propose.h, next to the reference-style
// drop-in (include/cudart_b200/renderkit.hpp) that builds the tree:
//
//   soup mesh -> CUDAMeshTree::buildMeshTreeLBVH -> box rays -> rt_trace_closest
//   -> rt_subtree_slots / rt_hit_labels -> training steps of the network
//   (rt_ray_features, rt_gemm_bf16, rt_gemm_xent_bf16, rt_colsum_bf16,
//   rt_adam_step) -> rt_mlp_propose -> rt_trace_closest_seeded.
//
// Exits 0 when the seeded traversal returns the plain traversal's hits bit
// for bit, the training loss fell, and no device error was raised.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "cudart_b200/renderkit.hpp"
#include "rt_propose.h"

using namespace renderkit;

namespace {

constexpr uint32_t kFeat = 192, kHidden = 128, kClasses = 4096, kDepth = 12, kBatch = 1024;

struct Lcg {  // 64-bit LCG (Knuth's MMIX constants), top 24 bits as a float in [0, 1)
  uint64_t s;
  float next() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return (float)(s >> 40) * (1.0f / 16777216.0f);
  }
};

uint16_t to_bf16(float x) {  // round to nearest even (finite inputs)
  uint32_t u;
  std::memcpy(&u, &x, 4);
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

#define OK(call) RK_OK(call)

// One layer: FP32 master weights [out][in] and biases, Adam moments, BF16 copies [out][in] and [in][out].
struct Layer {
  uint32_t out, in;
  CUDAArray<float> w, b, gw, gb, mw, vw, mb, vb;
  CUDAArray<uint16_t> w16, w16t;
  Layer(uint32_t o, uint32_t i, uint32_t fan_in, Lcg& rng)
      : out(o), in(i), w((size_t)o * i), b(o), gw((size_t)o * i), gb(o), mw((size_t)o * i), vw((size_t)o * i), mb(o), vb(o),
        w16((size_t)o * i), w16t((size_t)o * i) {
    const float bound = 1.0f / std::sqrt((float)fan_in);
    std::vector<float> hw((size_t)o * i), hb(o), zero((size_t)o * i, 0.0f);
    std::vector<uint16_t> h16((size_t)o * i), h16t((size_t)o * i);
    for (uint32_t r = 0; r < o; ++r)
      for (uint32_t c = 0; c < i; ++c) hw[(size_t)r * i + c] = c < fan_in ? (rng.next() * 2.0f - 1.0f) * bound : 0.0f;
    for (uint32_t r = 0; r < o; ++r) hb[r] = (rng.next() * 2.0f - 1.0f) * bound;
    for (uint32_t r = 0; r < o; ++r)
      for (uint32_t c = 0; c < i; ++c) {
        h16[(size_t)r * i + c] = to_bf16(hw[(size_t)r * i + c]);
        h16t[(size_t)c * o + r] = h16[(size_t)r * i + c];
      }
    w.copyDataFromHost(hw.data()); b.copyDataFromHost(hb.data());
    mw.copyDataFromHost(zero.data()); vw.copyDataFromHost(zero.data());
    mb.copyDataFromHost(zero.data()); vb.copyDataFromHost(zero.data());
    w16.copyDataFromHost(h16.data()); w16t.copyDataFromHost(h16t.data());
  }
};

rt_gemm_desc gemm(const void* a, uint32_t lda, const void* b, uint32_t ldb, uint32_t m, uint32_t n, uint32_t k, uint32_t* err) {
  rt_gemm_desc d = {};
  d.a = a; d.lda = lda; d.b = b; d.ldb = ldb; d.m = m; d.n = n; d.k = k; d.alpha = 1.0f; d.error_word = err;
  return d;
}

}  // namespace

int main() {
  Lcg rng{12345};
  // a soup of small triangles in the unit cube, and its box grown 1.5x for the ray origins and the features
  const uint32_t N = 60000;
  std::vector<float4> verts(3 * (size_t)N);
  std::vector<uint4> faces(N);
  for (uint32_t i = 0; i < N; ++i) {
    const float cx = rng.next(), cy = rng.next(), cz = rng.next();
    for (uint32_t k = 0; k < 3; ++k)
      verts[3 * (size_t)i + k] = make_float4(cx + 0.02f * (rng.next() - 0.5f), cy + 0.02f * (rng.next() - 0.5f),
                                             cz + 0.02f * (rng.next() - 0.5f), 0.0f);
    faces[i] = make_uint4(3 * i, 3 * i + 1, 3 * i + 2, 0);
  }
  aabox hitbox;
  hitbox.min = make_float4(-0.01f, -0.01f, -0.01f, 0.0f);
  hitbox.max = make_float4(1.01f, 1.01f, 1.01f, 0.0f);
  CUDAMesh mesh(verts.data(), 3 * N, faces.data(), N, hitbox);
  CUDAMeshTree tree(&mesh);
  tree.buildMeshTreeLBVH(12);
  const float lo[3] = {-0.25f, -0.25f, -0.25f}, hi[3] = {1.25f, 1.25f, 1.25f};

  // rays: origins uniform in the box, directions uniform on the sphere
  const uint32_t R = 1u << 17;
  std::vector<float4> ho(R), hd(R);
  for (uint32_t r = 0; r < R; ++r) {
    ho[r] = make_float4(lo[0] + (hi[0] - lo[0]) * rng.next(), lo[1] + (hi[1] - lo[1]) * rng.next(), lo[2] + (hi[2] - lo[2]) * rng.next(), 0.0f);
    float x, y, z, l;
    do {
      x = 2.0f * rng.next() - 1.0f; y = 2.0f * rng.next() - 1.0f; z = 2.0f * rng.next() - 1.0f;
      l = x * x + y * y + z * z;
    } while (l > 1.0f || l < 1e-6f);
    l = std::sqrt(l);
    hd[r] = make_float4(x / l, y / l, z / l, 0.0f);
  }
  CUDAArray<float4> orig(R), dir(R);
  orig.copyDataFromHost(ho.data());
  dir.copyDataFromHost(hd.data());
  CUDAArray<int32_t> hit_id(R), seed_id(R), labels(R), prop(R);
  CUDAArray<float> hit_t(R), seed_t(R);
  CUDAArray<float2> hit_uv(R), seed_uv(R);
  CUDAArray<uint32_t> err(1);
  const uint32_t zero = 0;
  err.copyDataFromHost(&zero);

  rt_trace_desc td = {};
  td.nodes = (const uint32_t*)tree.getNodesArray()->getPointer();
  td.tris = (const float*)tree.tris->getPointer();
  td.accel = tree.accel->getPointer();
  td.face_count_hint = N;
  td.indices = tree.getIndicesArray()->getPointer();
  td.orig = (const float*)orig.getPointer();
  td.dir = (const float*)dir.getPointer();
  td.ray_count = R;
  td.hit_id = hit_id.getPointer();
  td.hit_t = hit_t.getPointer();
  td.hit_uv = (float*)hit_uv.getPointer();
  td.error_word = err.getPointer();
  td.schedule = RT_TRACE_WHILE_WHILE | RT_TRACE_WIDE;
  OK(rt_trace_closest(&td, nullptr));

  // slot table of the tree cut at depth 12 and the label of every ray's hit
  const uint32_t S = 1u << kDepth;
  CUDAArray<int32_t> slot_ref(S), pos_label(N);
  CUDAArray<float> slot_box(8 * (size_t)S);
  rt_slot_desc sd = {};
  sd.nodes = td.nodes; sd.accel = td.accel; sd.face_count = N; sd.depth = kDepth;
  sd.slot_ref = slot_ref.getPointer(); sd.slot_box = slot_box.getPointer(); sd.pos_label = pos_label.getPointer();
  OK(rt_subtree_slots(&sd, nullptr));
  OK(rt_hit_labels(hit_id.getPointer(), R, pos_label.getPointer(), labels.getPointer(), nullptr));

  // the network: 192 -> 128 -> 128 -> 128 -> 4096
  Layer L1(kHidden, kFeat, 144, rng), L2(kHidden, kHidden, kHidden, rng), L3(kHidden, kHidden, kHidden, rng),
      L4(kClasses, kHidden, kHidden, rng);
  Layer* layers[4] = {&L1, &L2, &L3, &L4};
  const uint32_t B = kBatch;
  CUDAArray<uint16_t> X((size_t)B * kFeat), XT((size_t)kFeat * B), H1((size_t)B * kHidden), H2((size_t)B * kHidden),
      H3((size_t)B * kHidden), H1T((size_t)kHidden * B), H2T((size_t)kHidden * B), H3T((size_t)kHidden * B),
      G((size_t)B * kClasses), GT((size_t)kClasses * B), D3((size_t)B * kHidden), D2((size_t)B * kHidden), D1((size_t)B * kHidden),
      D3T((size_t)kHidden * B), D2T((size_t)kHidden * B), D1T((size_t)kHidden * B);
  CUDAArray<float> loss(1);
  const uint32_t steps = 60;
  float first_loss = 0.0f, last_loss = 0.0f;
  for (uint32_t st = 0; st < steps; ++st) {
    const size_t off = (size_t)(st * B) % (R - B);
    const float* o = (const float*)(orig.getPointer() + off);
    const float* d = (const float*)(dir.getPointer() + off);
    const int32_t* lab = labels.getPointer() + off;
    rt_feature_desc fd = {};
    fd.orig = o; fd.dir = d; fd.count = B;
    std::memcpy(fd.box_lo, lo, sizeof lo); std::memcpy(fd.box_hi, hi, sizeof hi);
    fd.out = X.getPointer(); fd.ld_out = kFeat; fd.out_t = XT.getPointer(); fd.ld_out_t = B;
    OK(rt_ray_features(&fd, nullptr));
    // forward: hidden layers (bias, ReLU, BF16 output and its transpose)
    const void* in[3] = {X.getPointer(), H1.getPointer(), H2.getPointer()};
    uint16_t* hout[3] = {H1.getPointer(), H2.getPointer(), H3.getPointer()};
    uint16_t* hout_t[3] = {H1T.getPointer(), H2T.getPointer(), H3T.getPointer()};
    for (int l = 0; l < 3; ++l) {
      rt_gemm_desc g = gemm(in[l], layers[l]->in, layers[l]->w16.getPointer(), layers[l]->in, B, kHidden, layers[l]->in, err.getPointer());
      g.bias = layers[l]->b.getPointer(); g.relu = 1;
      g.c_bf16 = hout[l]; g.ldc_bf16 = kHidden; g.ct_bf16 = hout_t[l]; g.ldct = B;
      OK(rt_gemm_bf16(&g, nullptr));
    }
    // logits + softmax cross-entropy gradient (mean over the batch)
    float zf = 0.0f;
    loss.copyDataFromHost(&zf);
    rt_gemm_xent_desc xd = {};
    xd.a = H3.getPointer(); xd.lda = kHidden; xd.b = L4.w16.getPointer(); xd.ldb = kHidden; xd.m = B; xd.n = kClasses; xd.k = kHidden;
    xd.bias = L4.b.getPointer(); xd.labels = lab; xd.scale = 1.0f / B;
    xd.g = G.getPointer(); xd.ldg = kClasses; xd.gt = GT.getPointer(); xd.ldgt = B; xd.loss_sum = loss.getPointer();
    xd.error_word = err.getPointer();
    OK(rt_gemm_xent_bf16(&xd, nullptr));
    // backward: dW = dY^T X, db = column sums of dY, dX = dY W masked by ReLU'
    const void* dy[4] = {D1.getPointer(), D2.getPointer(), D3.getPointer(), G.getPointer()};
    const void* dyt[4] = {D1T.getPointer(), D2T.getPointer(), D3T.getPointer(), GT.getPointer()};
    const void* xt[4] = {XT.getPointer(), H1T.getPointer(), H2T.getPointer(), H3T.getPointer()};
    const void* xmask[4] = {nullptr, H1.getPointer(), H2.getPointer(), H3.getPointer()};
    uint16_t* dx[4] = {nullptr, D1.getPointer(), D2.getPointer(), D3.getPointer()};
    uint16_t* dxt[4] = {nullptr, D1T.getPointer(), D2T.getPointer(), D3T.getPointer()};
    for (int l = 3; l >= 0; --l) {
      Layer& Ly = *layers[l];
      rt_gemm_desc gw = gemm(dyt[l], B, xt[l], B, Ly.out, Ly.in, B, err.getPointer());
      gw.c_f32 = Ly.gw.getPointer(); gw.ldc_f32 = Ly.in;
      OK(rt_gemm_bf16(&gw, nullptr));
      OK(rt_colsum_bf16(dy[l], B, Ly.out, Ly.out, Ly.gb.getPointer(), nullptr));
      if (l > 0) {
        rt_gemm_desc gx = gemm(dy[l], Ly.out, Ly.w16t.getPointer(), Ly.out, B, Ly.in, Ly.out, err.getPointer());
        gx.mask = xmask[l]; gx.ldmask = Ly.in;
        gx.c_bf16 = dx[l]; gx.ldc_bf16 = Ly.in; gx.ct_bf16 = dxt[l]; gx.ldct = B;
        OK(rt_gemm_bf16(&gx, nullptr));
      }
    }
    for (Layer* Ly : layers) {
      rt_adam_desc ad = {};
      ad.param = Ly->w.getPointer(); ad.grad = Ly->gw.getPointer(); ad.m = Ly->mw.getPointer(); ad.v = Ly->vw.getPointer();
      ad.rows = Ly->out; ad.cols = Ly->in; ad.lr = 2e-3f; ad.beta1 = 0.9f; ad.beta2 = 0.999f; ad.eps = 1e-8f; ad.step = st + 1;
      ad.out_bf16 = Ly->w16.getPointer(); ad.ld_bf16 = Ly->in; ad.out_bf16_t = Ly->w16t.getPointer(); ad.ld_bf16_t = Ly->out;
      OK(rt_adam_step(&ad, nullptr));
      ad.param = Ly->b.getPointer(); ad.grad = Ly->gb.getPointer(); ad.m = Ly->mb.getPointer(); ad.v = Ly->vb.getPointer();
      ad.rows = 1; ad.cols = Ly->out; ad.out_bf16 = nullptr; ad.out_bf16_t = nullptr;
      OK(rt_adam_step(&ad, nullptr));
    }
    float lv = 0.0f;
    loss.copyDataToHost(&lv);
    if (st == 0) first_loss = lv;
    last_loss = lv;
  }

  // fused proposals for every ray, then the seeded traversal
  rt_mlp_propose_desc pd = {};
  pd.orig = (const float*)orig.getPointer(); pd.dir = (const float*)dir.getPointer(); pd.count = R;
  std::memcpy(pd.box_lo, lo, sizeof lo); std::memcpy(pd.box_hi, hi, sizeof hi);
  pd.w1 = L1.w16.getPointer(); pd.w2 = L2.w16.getPointer(); pd.w3 = L3.w16.getPointer(); pd.w4 = L4.w16.getPointer();
  pd.b1 = L1.b.getPointer(); pd.b2 = L2.b.getPointer(); pd.b3 = L3.b.getPointer(); pd.b4 = L4.b.getPointer();
  pd.n = kClasses; pd.out_index = prop.getPointer(); pd.error_word = err.getPointer();
  OK(rt_mlp_propose(&pd, nullptr));
  rt_trace_desc sdsc = td;
  sdsc.hit_id = seed_id.getPointer(); sdsc.hit_t = seed_t.getPointer(); sdsc.hit_uv = (float*)seed_uv.getPointer();
  rt_seed_desc seed = {};
  seed.proposal = prop.getPointer(); seed.slot_ref = slot_ref.getPointer(); seed.slot_box = slot_box.getPointer(); seed.slot_count = S;
  OK(rt_trace_closest_seeded(&sdsc, &seed, nullptr));
  RK_CHECK(cudaDeviceSynchronize() == cudaSuccess, "device");

  std::vector<int32_t> a(R), b(R), pr(R);
  std::vector<float> ta(R), tb(R);
  hit_id.copyDataToHost(a.data()); seed_id.copyDataToHost(b.data()); prop.copyDataToHost(pr.data());
  hit_t.copyDataToHost(ta.data()); seed_t.copyDataToHost(tb.data());
  uint32_t e = 0;
  err.copyDataToHost(&e);
  size_t diff = 0, hits = 0, proposed = 0;
  for (uint32_t r = 0; r < R; ++r) {
    if (a[r] != b[r] || std::memcmp(&ta[r], &tb[r], 4) != 0) ++diff;
    hits += a[r] >= 0;
    proposed += pr[r] >= 0;
  }
  std::printf("learned proposal from C++: rays %u, hits %zu, proposals %zu, differing hits %zu, loss %.4f -> %.4f, device error %u\n", R, hits, proposed,
              diff, first_loss, last_loss, e);
  if (diff != 0 || e != 0 || !(last_loss < first_loss) || hits == 0) return 1;
  return 0;
}
