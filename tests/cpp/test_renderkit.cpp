// test_renderkit.cpp -- drives the C++ drop-in (include/cudart_b200/renderkit.hpp)
// the way the reference's samples drive CUDAMeshTree / CUDARaytracer
// (samples/02_how_to_use_the_raytracer.cpp:67-85,178-194) and its sorter
// (samples/09_how_to_use_a_sorter.cpp): build, camera lookAt, primary rays,
// trace, radix sort; then SAH and Hybrid builds of fresh copies of the mesh and
// the rasteriser on the LBVH-ordered mesh. Reads a scene file, writes the
// results for tests/test_gpu_renderkit.py to compare with the CPU oracle.
//
// in : u32 V, N, W, H, tree_depth, K; f32 center[3], target[3], fov, ratio, hitbox[8];
//      float4 vertices[V]; uint4 faces[N]; u32 keys[K]
// out: u32 node_count, real_depth; bvnode nodes[node_count]; uint4 faces[N] (reordered);
//      u32 faces_id[W*H]; f32 depths[W*H]; float2 coords[W*H]; u32 keys[K]; u32 indices[K];
//      then for SAH and Hybrid(8): u32 node_count; bvnode nodes[]; uint4 faces[N];
//      then the raster surfaces: u32 faces_id[W*H]; f32 depths[W*H]; float2 coords[W*H]
#include <cstdio>
#include <vector>

#include "cudart_b200/renderkit.hpp"

using namespace renderkit;

template <typename T>
static void rd(FILE* f, T* p, size_t n) { RK_CHECK(fread(p, sizeof(T), n, f) == n, "short read"); }
template <typename T>
static void wr(FILE* f, const T* p, size_t n) { RK_CHECK(fwrite(p, sizeof(T), n, f) == n, "short write"); }

int main(int argc, char** argv) {
  RK_CHECK(argc == 3, "usage: test_renderkit in.bin out.bin");
  FILE* in = fopen(argv[1], "rb");
  RK_CHECK(in != nullptr, "cannot open input");
  uint32_t hdr[6];
  float cam[8], hb[8];
  rd(in, hdr, 6); rd(in, cam, 8); rd(in, hb, 8);
  const uint32_t V = hdr[0], N = hdr[1], W = hdr[2], H = hdr[3], depth = hdr[4], K = hdr[5];
  std::vector<float4> verts(V);
  std::vector<uint4> faces(N);
  std::vector<uint32_t> keys(K);
  rd(in, verts.data(), V); rd(in, faces.data(), N); rd(in, keys.data(), K);
  fclose(in);

  aabox hitbox;
  hitbox.min = make_float4(hb[0], hb[1], hb[2], hb[3]);
  hitbox.max = make_float4(hb[4], hb[5], hb[6], hb[7]);
  const std::vector<uint4> faces0 = faces;
  CUDAMesh mesh(verts.data(), V, faces.data(), N, hitbox);
  CUDAMeshTree tree(&mesh);
  tree.buildMeshTreeLBVH(depth);

  CUDACamera camera;
  camera.setCenter(cam[0], cam[1], cam[2]);
  camera.lookAt(cam[3], cam[4], cam[5]);
  camera.setFOV(cam[6]);
  camera.setRatio(cam[7]);
  CUDABuffer buffer(W, H);
  CUDARaytracer raytracer;
  raytracer.setBuffer(&buffer);
  raytracer.setCamera(&camera);
  buffer.clearOutputSurfaces();
  raytracer.calcPrimaryRays();
  raytracer.raytraceMeshTree(&mesh, &tree);

  const uint32_t nc = tree.getNodeCount(), rd_ = tree.getRealDepth();
  std::vector<bvnode> nodes(nc);
  tree.getNodesArray()->copyDataToHost(nodes.data());
  mesh.getFacesArray()->copyDataToHost(faces.data());
  const size_t R = (size_t)W * H;
  std::vector<uint32_t> ids(R);
  std::vector<float> depths(R);
  std::vector<float2> coords(R);
  buffer.out_faces_id.copyDataToHost(ids.data());
  buffer.out_depths.copyDataToHost(depths.data());
  buffer.out_coords.copyDataToHost(coords.data());

  CUDAArray<uint> dk(K), di(K);
  dk.copyDataFromHost(keys.data());
  CUDA_radixSortGeneral(dk.getPointer(), di.getPointer(), K, 32, true);
  std::vector<uint32_t> sk(K), si(K);
  dk.copyDataToHost(sk.data());
  di.copyDataToHost(si.data());

  FILE* out = fopen(argv[2], "wb");
  RK_CHECK(out != nullptr, "cannot open output");
  wr(out, &nc, 1); wr(out, &rd_, 1);
  wr(out, nodes.data(), nc); wr(out, faces.data(), N);
  wr(out, ids.data(), R); wr(out, depths.data(), R); wr(out, coords.data(), R);
  wr(out, sk.data(), K); wr(out, si.data(), K);

  for (int hybrid = 0; hybrid < 2; ++hybrid) {
    CUDAMesh m2(verts.data(), V, faces0.data(), N, hitbox);
    CUDAMeshTree t2(&m2);
    if (hybrid) t2.buildMeshTreeHybrid(8);
    else t2.buildMeshTreeSAH();
    const uint32_t n2 = t2.getNodeCount();
    std::vector<bvnode> nodes2(n2);
    std::vector<uint4> faces2(N);
    t2.getNodesArray()->copyDataToHost(nodes2.data());
    m2.getFacesArray()->copyDataToHost(faces2.data());
    wr(out, &n2, 1); wr(out, nodes2.data(), n2); wr(out, faces2.data(), N);
  }

  buffer.clearOutputSurfaces();
  raytracer.rasterizeMeshTree(&mesh, &tree);
  buffer.out_faces_id.copyDataToHost(ids.data());
  buffer.out_depths.copyDataToHost(depths.data());
  buffer.out_coords.copyDataToHost(coords.data());
  wr(out, ids.data(), R); wr(out, depths.data(), R); wr(out, coords.data(), R);
  fclose(out);
  std::printf("renderkit ok: %u faces, %u nodes, depth %u\n", N, nc, rd_);
  return 0;
}
