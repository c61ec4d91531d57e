// renderkit.hpp -- C++ drop-in for the reference's host interface of the LBVH
// build / ray-tracing path, implemented over the C ABI of rt_core.h.
//
// Same class and method names, argument meanings and defaults as the
// reference (namespace renderkit):
//   CUDAMesh           CUDAMesh.h:20-155       (device vertices/faces + hit box)
//   CUDAMeshTree       CUDAMeshTree.h:22-164   (nodes, boxes, indices; buildMeshTreeLBVH,
//                                               buildMeshTreeSAH, buildMeshTreeHybrid)
//   CUDACamera         CUDACamera.h:15-321     (center, angles, fov, ratio; lookAt)
//   CUDABuffer         CUDABuffer.h:17-206     (ray in/out surfaces; clearOutputSurfaces)
//   CUDARaytracer      CUDARaytracer.h:58-209  (headless: setBuffer/setCamera,
//                                               calcPrimaryRays, raytraceMeshTree,
//                                               rasterizeMeshTree)
// and the free functions the reference's kernels export (CUDA_radixSortGeneral,
// CUDA_radixSort, CUDA_bubbleSort512, CUDA_bitonicSort, CUDA_bitonicSortGeneral,
// CUDA_calcMeshBoxes, CUDA_reorderMeshFaces, CUDA_buildMeshTreeLBVH,
// CUDA_calcPrimaryRays, CUDA_raytraceMeshTree, CUDA_rasterizeMeshTree).
//
// Error behaviour follows the reference's _assert (CUDACommon.h:123-133): a
// failing call prints the file, line and message and exits, except that this
// shim does not call system("pause"). The calls synchronize before returning,
// as the reference's did (cudaThreadSynchronize after each launch).
// Differences: faces_id of a miss is 0xFFFFFFFF instead of an uninitialised
// value; the LBVH build keeps the pre-gathered triangle stream and traversal
// blob on the tree so that raytraceMeshTree uses the fast traversal; the
// rasteriser writes each pixel's face index (the reference writes the first
// index of the face's 192-face block); buildMeshTreeSAH always builds from the
// mesh (the reference refines the leaves of a tree that already has nodes).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../rt_core.h"
#include "../rt_raster.h"
#include "../rt_sah.h"

namespace renderkit {

typedef unsigned int uint;

inline void rk_assert(bool ok, const char* file, int line, const char* msg) {
  if (!ok) {
    std::printf("Error in %s, line %d : %s\n\n", file, line, msg);
    std::exit(-1);
  }
}
#define RK_CHECK(expr, msg) ::renderkit::rk_assert((expr), __FILE__, __LINE__, (msg))
#define RK_OK(call) RK_CHECK((call) == RT_OK, #call)

// The library must have been built from the same rt_core.h (struct layouts).
inline void rk_check_abi() {
  static const bool ok = rt_abi_version() == RT_ABI_VERSION;
  RK_CHECK(ok, "librt_core was built from a different rt_core.h (RT_ABI_VERSION mismatch)");
}

// Device array owning cudaMalloc'd memory (CUDAArray.h:16-209).
template <typename T>
class CUDAArray {
 public:
  explicit CUDAArray(size_t count) : count_(count) {
    RK_CHECK(cudaMalloc((void**)&ptr_, count * sizeof(T) + (count == 0)) == cudaSuccess, "CUDAArray: cudaMalloc failed");
  }
  ~CUDAArray() { cudaFree(ptr_); }
  CUDAArray(const CUDAArray&) = delete;
  CUDAArray& operator=(const CUDAArray&) = delete;
  T* getPointer() const { return ptr_; }
  size_t getUnitCount() const { return count_; }
  void copyDataFromHost(const T* src) { RK_CHECK(cudaMemcpy(ptr_, src, count_ * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess, "copy"); }
  void copyDataToHost(T* dst) const { RK_CHECK(cudaMemcpy(dst, ptr_, count_ * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess, "copy"); }
  void copyDataFromDevice(const T* src) { RK_CHECK(cudaMemcpy(ptr_, src, count_ * sizeof(T), cudaMemcpyDeviceToDevice) == cudaSuccess, "copy"); }

 private:
  T* ptr_ = nullptr;
  size_t count_;
};

struct aabox { float4 min, max; };  // CUDABox.h:17-148 (32 bytes)
struct bvnode { uint32_t word0, word1; float3 box_min, box_max; };  // CUDANode.h:20-50 (32 bytes)
static_assert(sizeof(bvnode) == 32, "bvnode is 32 bytes");

// ---------------------------------------------------------------------------
class CUDAMesh {
 public:
  // vertices: float4 (w = 0); faces: uint4 (a, b, c, material); hitbox as the
  // model computed it (CUDAModel grows it per vertex).
  CUDAMesh(const float4* vertices, uint vertex_count, const uint4* faces, uint face_count, const aabox& hitbox)
      : verts_(vertex_count), faces_(face_count), hitbox_(hitbox) {
    verts_.copyDataFromHost(vertices);
    faces_.copyDataFromHost(faces);
  }
  uint getVertexCount() const { return (uint)verts_.getUnitCount(); }
  uint getFaceCount() const { return (uint)faces_.getUnitCount(); }
  CUDAArray<float4>* getVerticesArray() { return &verts_; }
  CUDAArray<uint4>* getFacesArray() { return &faces_; }
  aabox getHitbox() const { return hitbox_; }

 private:
  CUDAArray<float4> verts_;
  CUDAArray<uint4> faces_;
  aabox hitbox_;
};

// ---------------------------------------------------------------------------
class CUDAMeshTree {
 public:
  explicit CUDAMeshTree(CUDAMesh* mesh) : mesh(mesh) {
    const uint n = mesh->getFaceCount();
    if (n > 0) {
      boxes = new CUDAArray<aabox>(n);
      indices = new CUDAArray<uint>(n);
    }
  }
  ~CUDAMeshTree() {
    delete nodes; delete boxes; delete indices; delete tris; delete accel;
  }
  CUDAMesh* getMesh() const { return mesh; }
  aabox getHitbox() const { return mesh->getHitbox(); }
  CUDAArray<aabox>* getBoxesArray() const { return boxes; }
  CUDAArray<uint>* getIndicesArray() const { return indices; }
  CUDAArray<bvnode>* getNodesArray() const { return nodes; }
  uint getNodeCount() const { return nodes ? (uint)nodes->getUnitCount() : 0; }
  uint getRealDepth() const { return real_depth; }

  // CUDAMeshTree.cpp:88-91 -> CUDA_buildMeshTreeLBVH(mesh, this, true, tree_depth)
  void buildMeshTreeLBVH(uint tree_depth = 12);
  // CUDAMeshTree.cpp:93-96 -> CUDA_buildMeshTreeSAH(mesh, this)
  void buildMeshTreeSAH();
  // CUDAMeshTree.cpp:98-103: LBVH of lbvh_tree_depth levels without leaf splitting, then SAH in every leaf
  void buildMeshTreeHybrid(uint lbvh_tree_depth = 12);

  void updateNodes(bvnode* nodes_buffer, uint node_count) {  // CUDAMeshTree.cpp:105-112
    delete nodes;
    nodes = new CUDAArray<bvnode>(node_count);
    nodes->copyDataFromDevice(nodes_buffer);
  }

  // traversal data kept from the build (no reference counterpart)
  CUDAArray<float4>* tris = nullptr;
  CUDAArray<unsigned char>* accel = nullptr;

 private:
  friend void CUDA_buildMeshTreeLBVH(CUDAMesh*, CUDAMeshTree*, bool, uint);
  friend void rk_build_sah(CUDAMesh*, CUDAMeshTree*, uint);
  CUDAMesh* mesh;
  CUDAArray<bvnode>* nodes = nullptr;
  CUDAArray<aabox>* boxes = nullptr;
  CUDAArray<uint>* indices = nullptr;
  uint real_depth = 0;
};

// kernels/CUDA_buildMeshTreeLBVH.cu:457
inline void CUDA_buildMeshTreeLBVH(CUDAMesh* mesh, CUDAMeshTree* tree, bool tree_complete = false, uint tree_depth = 32) {
  rk_check_abi();
  const uint n = mesh->getFaceCount();
  rt_build_params p = {tree_depth, tree_complete ? 1u : 0u, 0u, 0u, 32u};
  size_t scratch_bytes = 0, accel_bytes = 0;
  uint32_t max_nodes = 0;
  RK_OK(rt_lbvh_scratch_bytes(n, &p, &scratch_bytes, &max_nodes));
  RK_OK(rt_lbvh_accel_bytes(n, &accel_bytes));
  CUDAArray<unsigned char> scratch(scratch_bytes);
  CUDAArray<bvnode> nodes_buffer(max_nodes);
  CUDAArray<rt_build_info> info(1);
  delete tree->tris; tree->tris = nullptr;
  delete tree->accel; tree->accel = nullptr;
  if (tree_complete) {
    tree->tris = new CUDAArray<float4>(3 * (size_t)n);
    tree->accel = new CUDAArray<unsigned char>(accel_bytes);
  }
  aabox hb = mesh->getHitbox();
  rt_build_desc d = {};
  d.vertices = (const float*)mesh->getVerticesArray()->getPointer();
  d.vertex_count = mesh->getVertexCount();
  d.face_count = n;
  d.faces_in = (const uint32_t*)mesh->getFacesArray()->getPointer();
  d.faces_out = (uint32_t*)mesh->getFacesArray()->getPointer();  // reordered in place (:669-676)
  d.hitbox = (const float*)&hb;
  d.params = p;
  d.boxes = (float*)tree->boxes->getPointer();
  d.indices = tree->indices->getPointer();
  d.nodes = (uint32_t*)nodes_buffer.getPointer();
  d.max_nodes = max_nodes;
  d.tris = tree_complete ? (float*)tree->tris->getPointer() : nullptr;
  d.accel = tree_complete ? tree->accel->getPointer() : nullptr;
  d.accel_bytes = tree_complete ? accel_bytes : 0;
  d.info = info.getPointer();
  d.scratch = scratch.getPointer();
  d.scratch_bytes = scratch_bytes;
  RK_OK(rt_lbvh_build(&d, nullptr));
  rt_build_info h;
  info.copyDataToHost(&h);
  RK_CHECK(h.error == 0, "CUDA_buildMeshTreeLBVH() : device error");
  tree->real_depth = h.real_depth;
  tree->updateNodes(nodes_buffer.getPointer(), h.node_count);
}

inline void CUDAMeshTree::buildMeshTreeLBVH(uint tree_depth) { CUDA_buildMeshTreeLBVH(mesh, this, true, tree_depth); }

// SAH (lbvh_depth 0) or Hybrid build through rt_sah_build; faces reordered in
// the mesh as the reference's CUDA_reorderMeshFaces call leaves them (:777-784).
inline void rk_build_sah(CUDAMesh* mesh, CUDAMeshTree* tree, uint lbvh_depth) {
  rk_check_abi();
  const uint n = mesh->getFaceCount();
  size_t scratch_bytes = 0, accel_bytes = 0;
  uint32_t max_nodes = 0;
  RK_OK(rt_sah_sizes(n, lbvh_depth, &scratch_bytes, &max_nodes));
  RK_OK(rt_lbvh_accel_bytes(n, &accel_bytes));
  CUDAArray<unsigned char> scratch(scratch_bytes);
  CUDAArray<bvnode> nodes_buffer(max_nodes);
  CUDAArray<uint4> faces_out(n);
  CUDAArray<rt_build_info> info(1);
  delete tree->tris; tree->tris = new CUDAArray<float4>(3 * (size_t)n);
  delete tree->accel; tree->accel = new CUDAArray<unsigned char>(accel_bytes);
  aabox hb = mesh->getHitbox();
  rt_sah_desc d = {};
  d.vertices = (const float*)mesh->getVerticesArray()->getPointer();
  d.vertex_count = mesh->getVertexCount();
  d.face_count = n;
  d.faces_in = (const uint32_t*)mesh->getFacesArray()->getPointer();
  d.faces_out = (uint32_t*)faces_out.getPointer();
  d.hitbox = (const float*)&hb;
  d.lbvh_depth = lbvh_depth;
  d.boxes = (float*)tree->boxes->getPointer();
  d.indices = tree->indices->getPointer();
  d.nodes = (uint32_t*)nodes_buffer.getPointer();
  d.max_nodes = max_nodes;
  d.tris = (float*)tree->tris->getPointer();
  d.accel = tree->accel->getPointer();
  d.accel_bytes = accel_bytes;
  d.info = info.getPointer();
  d.scratch = scratch.getPointer();
  d.scratch_bytes = scratch_bytes;
  RK_OK(rt_sah_build(&d, nullptr));
  rt_build_info h;
  info.copyDataToHost(&h);
  RK_CHECK(h.error == 0, "CUDA_buildMeshTreeSAH() : device error");
  RK_CHECK(cudaMemcpy(mesh->getFacesArray()->getPointer(), faces_out.getPointer(), (size_t)n * 16, cudaMemcpyDeviceToDevice) == cudaSuccess,
           "CUDA_buildMeshTreeSAH() : face reorder");
  tree->real_depth = h.real_depth;
  tree->updateNodes(nodes_buffer.getPointer(), h.node_count);
}

// kernels/CUDA_buildMeshTreeSAH.cu:672
inline void CUDA_buildMeshTreeSAH(CUDAMesh* mesh, CUDAMeshTree* tree) { rk_build_sah(mesh, tree, 0); }
inline void CUDAMeshTree::buildMeshTreeSAH() { rk_build_sah(mesh, this, 0); }
inline void CUDAMeshTree::buildMeshTreeHybrid(uint lbvh_tree_depth) { rk_build_sah(mesh, this, lbvh_tree_depth); }

// ---------------------------------------------------------------------------
class CUDACamera {
 public:
  CUDACamera() {  // CUDACamera.cpp:29-50
    cam_.center[0] = cam_.center[1] = cam_.center[2] = 0.0f;
    cam_.angle[0] = 3.14159265359f * 0.5f; cam_.angle[1] = 0.0f; cam_.angle[2] = 0.0f;
    cam_.fov = 3.14159265359f * 0.5f;
    cam_.ratio = 4.0f / 3.0f;
  }
  void setCenter(float x, float y, float z) { cam_.center[0] = x; cam_.center[1] = y; cam_.center[2] = z; }
  float3 getCenter() const { return make_float3(cam_.center[0], cam_.center[1], cam_.center[2]); }
  void setAngle(float x, float y, float z) {  // CUDACamera.cpp:108-115
    cam_.angle[0] = x; cam_.angle[1] = y; cam_.angle[2] = z;
    dirFromAngle();
  }
  float3 getAngle() const { return make_float3(cam_.angle[0], cam_.angle[1], cam_.angle[2]); }
  void lookAt(float x, float y, float z) {  // CUDACamera.cpp:126-132
    float t[3] = {x, y, z};
    RK_OK(rt_camera_view_dir(&cam_, t, dir_));
    RK_OK(rt_camera_look_at(&cam_, t));
  }
  float3 getDir() const { return make_float3(dir_[0], dir_[1], dir_[2]); }
  const float* dirPtr() const { return dir_; }
  void setFOV(float fov) { cam_.fov = fov; }
  float getFOV() const { return cam_.fov; }
  void setRatio(float ratio) { cam_.ratio = ratio; }
  void setRatio(int width, int height) { cam_.ratio = (float)width / (float)height; }
  float getRatio() const { return cam_.ratio; }
  float pitch() const { return cam_.angle[0]; }
  float yaw() const { return cam_.angle[1]; }
  float roll() const { return cam_.angle[2]; }
  const rt_camera* raw() const { return &cam_; }

 private:
  // CUDACamera.cpp:55-68: wrap / clamp the angles, dir = normalize(cos p cos y, sin y, sin p cos y)
  void dirFromAngle() {
    const float pi = 3.14159265359f;
    float* a = cam_.angle;
    if (a[0] < 0.0f) a[0] += pi * 2.0f;
    if (a[0] > pi * 2.0f) a[0] -= pi * 2.0f;
    if (a[1] < -pi * 0.5f + 0.001f) a[1] = -pi * 0.5f + 0.001f;
    if (a[1] > pi * 0.5f - 0.001f) a[1] = pi * 0.5f - 0.001f;
    const float dx = cosf(a[0]) * cosf(a[1]), dy = sinf(a[1]), dz = sinf(a[0]) * cosf(a[1]);
    const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
    dir_[0] = dx * inv; dir_[1] = dy * inv; dir_[2] = dz * inv;
  }
  rt_camera cam_;
  float dir_[3] = {0.0f, 0.0f, 1.0f};  // CUDACamera.cpp:45-47
};

// ---------------------------------------------------------------------------
class CUDABuffer {
 public:
  CUDABuffer(int width, int height)
      : width(width), height(height), in_origins((size_t)width * height), in_directions((size_t)width * height),
        out_faces_id((size_t)width * height), out_coords((size_t)width * height), out_depths((size_t)width * height) {
    RK_CHECK(width > 0 && height > 0, "CUDABuffer::CUDABuffer() : Invalid size, must be positive.");
  }
  int getWidth() const { return width; }
  int getHeight() const { return height; }
  // CUDABuffer.cpp:109-131: ids 0, coords 0, depths CUDART_NORM_HUGE_F
  void clearOutputSurfaces() {
    const size_t n = (size_t)width * height;
    RK_CHECK(cudaMemset(out_faces_id.getPointer(), 0, n * 4) == cudaSuccess, "clear");
    RK_CHECK(cudaMemset(out_coords.getPointer(), 0, n * 8) == cudaSuccess, "clear");
    std::vector<float> huge(n, 3.402823466e+38f);
    out_depths.copyDataFromHost(huge.data());
  }
  int width, height;
  CUDAArray<float4> in_origins, in_directions;
  CUDAArray<uint> out_faces_id;
  CUDAArray<float2> out_coords;
  CUDAArray<float> out_depths;
};

// kernels/CUDA_calcPrimaryRays.cu:38
inline void CUDA_calcPrimaryRays(CUDABuffer* buffer, CUDACamera* camera) {
  rk_check_abi();
  RK_OK(rt_primary_rays(camera->raw(), buffer->getWidth(), buffer->getHeight(), (float*)buffer->in_origins.getPointer(),
                        (float*)buffer->in_directions.getPointer(), nullptr));
  RK_CHECK(cudaDeviceSynchronize() == cudaSuccess, "CUDA_calcPrimaryRays() : Unable to execute CUDA kernel.");
}

// kernels/CUDA_raytraceMeshTree.cu:434. Depths are read as the initial tmax and
// written in place; faces_id is the position in the (reordered) mesh faces.
// coherency (the reference's choice between its packet and per-ray kernels)
// picks the traversal schedule here: 8 x 4 pixel tiles for coherent primary
// rays, one ray per thread otherwise; both descend while-while through the
// 4-wide records. The closest hits do not depend on the schedule.
inline void CUDA_raytraceMeshTree(CUDABuffer* buffer, CUDAMesh* mesh, CUDAMeshTree* tree, bool coherency = true) {
  rk_check_abi();
  rt_trace_desc d = {};
  d.nodes = (const uint32_t*)tree->getNodesArray()->getPointer();
  if (tree->tris) {
    d.tris = (const float*)tree->tris->getPointer();
    d.accel = tree->accel ? tree->accel->getPointer() : nullptr;
    d.face_count_hint = mesh->getFaceCount();
  } else {
    d.vertices = (const float*)mesh->getVerticesArray()->getPointer();
    d.faces = (const uint32_t*)mesh->getFacesArray()->getPointer();
  }
  d.indices = tree->getIndicesArray()->getPointer();
  d.orig = (const float*)buffer->in_origins.getPointer();
  d.dir = (const float*)buffer->in_directions.getPointer();
  d.tmax = buffer->out_depths.getPointer();
  d.hit_t = buffer->out_depths.getPointer();
  d.hit_id = (int32_t*)buffer->out_faces_id.getPointer();
  d.hit_uv = (float*)buffer->out_coords.getPointer();
  d.ray_count = (uint32_t)((size_t)buffer->getWidth() * buffer->getHeight());
  d.id_mode = 0;
  if (d.accel) {
    d.schedule = RT_TRACE_WHILE_WHILE | RT_TRACE_WIDE;
    if (coherency) d.image_width = buffer->getWidth();
  }
  RK_OK(rt_trace_closest(&d, nullptr));
  RK_CHECK(cudaDeviceSynchronize() == cudaSuccess, "CUDA_raytraceMeshTree() : Unable to execute CUDA kernel.");
}

// kernels/CUDA_rasterizeMeshTree.cu:255. faces_id is the face's index in the
// mesh's (current) face order.
inline void CUDA_rasterizeMeshTree(CUDABuffer* buffer, CUDACamera* camera, CUDAMesh* mesh, CUDAMeshTree* tree) {
  rk_check_abi();
  (void)tree;
  rt_raster_desc d = {};
  RK_OK(rt_raster_matrix(camera->raw(), camera->dirPtr(), d.matrix));
  d.vertices = (const float*)mesh->getVerticesArray()->getPointer();
  d.vertex_count = mesh->getVertexCount();
  d.faces = (const uint32_t*)mesh->getFacesArray()->getPointer();
  d.face_count = mesh->getFaceCount();
  d.width = (uint32_t)buffer->getWidth();
  d.height = (uint32_t)buffer->getHeight();
  d.id_mode = 0;
  d.face_id = (int32_t*)buffer->out_faces_id.getPointer();
  d.uv = (float*)buffer->out_coords.getPointer();
  d.depth = buffer->out_depths.getPointer();
  size_t bytes = 0;
  RK_OK(rt_raster_scratch_bytes(d.face_count, d.width, d.height, 0, &bytes));
  CUDAArray<unsigned char> scratch(bytes);
  d.scratch = scratch.getPointer();
  d.scratch_bytes = bytes;
  RK_OK(rt_rasterize(&d, nullptr));
  RK_CHECK(cudaDeviceSynchronize() == cudaSuccess, "CUDA_rasterizeMeshTree() : Unable to execute CUDA kernel.");
}

class CUDARaytracer {
 public:
  void setBuffer(CUDABuffer* buffer) { current_buffer = buffer; }
  CUDABuffer* getBuffer() const { return current_buffer; }
  void setCamera(CUDACamera* camera) { current_camera = camera; }
  CUDACamera* getCamera() const { return current_camera; }
  void calcPrimaryRays() { CUDA_calcPrimaryRays(current_buffer, current_camera); }  // CUDARaytracer.cpp:125-128
  void raytraceMeshTree(CUDAMesh* mesh, CUDAMeshTree* tree, bool coherency = true) {  // CUDARaytracer.cpp:130-135
    if (mesh->getVertexCount() == 0) return;
    CUDA_raytraceMeshTree(current_buffer, mesh, tree, coherency);
  }
  void rasterizeMeshTree(CUDAMesh* mesh, CUDAMeshTree* tree) {  // CUDARaytracer.cpp:137-142
    if (mesh->getVertexCount() == 0) return;
    CUDA_rasterizeMeshTree(current_buffer, current_camera, mesh, tree);
  }

 private:
  CUDABuffer* current_buffer = nullptr;
  CUDACamera* current_camera = nullptr;
};

// ---------------------------------------------------------------------------
// sort family
namespace detail {
inline void sort_pairs(uint* keys, uint* values, uint length, uint bit_depth, bool init) {
  size_t bytes = 0;
  RK_OK(rt_sort_scratch_bytes(length, &bytes));
  CUDAArray<unsigned char> scratch(bytes);
  RK_OK(rt_radix_sort_pairs(keys, values, length, bit_depth, init ? 1 : 0, scratch.getPointer(), bytes, nullptr));
  RK_CHECK(cudaDeviceSynchronize() == cudaSuccess, "sort : Unable to execute CUDA kernel.");
}
}  // namespace detail

// kernels/CUDA_radixSortGeneral.cu:397
inline void CUDA_radixSortGeneral(uint* keys, uint* indices, uint length, uint bit_depth = 32, bool init_indices = false) {
  detail::sort_pairs(keys, indices, length, bit_depth, init_indices);
}
// kernels/CUDA_bubbleSort512.cu:114 (length <= 512 in the reference)
inline void CUDA_bubbleSort512(uint* keys, uint* indices, uint length, bool init_indices = false) {
  RK_CHECK(length <= 512, "CUDA_bubbleSort512() : Unable to execute CUDA kernel.");
  detail::sort_pairs(keys, indices, length, 32, init_indices);
}
// kernels/CUDA_bitonicSortGeneral.cu:505 (32-bit keys and values)
template <typename key_type, typename value_type>
inline void CUDA_bitonicSortGeneral(value_type* keys, value_type* values, uint length) {
  static_assert(sizeof(key_type) == 4 && sizeof(value_type) == 4, "32-bit keys and values");
  detail::sort_pairs((uint*)keys, (uint*)values, length, 32, false);
}
// kernels/CUDA_radixSort.cu:357
inline void CUDA_radixSort(uint* values, uint length, uint bit_depth = 32) {
  size_t bytes = 0;
  RK_OK(rt_sort_scratch_bytes(length, &bytes));
  CUDAArray<unsigned char> scratch(bytes);
  RK_OK(rt_radix_sort_keys(values, length, bit_depth, scratch.getPointer(), bytes, nullptr));
  RK_CHECK(cudaDeviceSynchronize() == cudaSuccess, "CUDA_radixSort() : Unable to execute CUDA kernel.");
}
// kernels/CUDA_bitonicSort.cu:403 (32-bit values)
template <typename value_type>
inline void CUDA_bitonicSort(value_type* values, uint length) {
  static_assert(sizeof(value_type) == 4, "32-bit values");
  CUDA_radixSort((uint*)values, length, 32);
}

// kernels/CUDA_calcMeshBoxes.cu:65
inline void CUDA_calcMeshBoxes(aabox* boxes, uint* indices, uint4* faces, float4* vertices, uint count) {
  RK_OK(rt_mesh_boxes((const float*)vertices, (const uint32_t*)faces, count, (float*)boxes, indices, nullptr));
  RK_CHECK(cudaDeviceSynchronize() == cudaSuccess, "CUDA_calcMeshBoxes() : Unable to execute CUDA kernel.");
}

// kernels/CUDA_reorderMeshFaces.cu:44 (in place through a temporary, as the reference)
inline void CUDA_reorderMeshFaces(uint4* faces, uint* indices, uint count) {
  CUDAArray<uint4> tmp(count);
  RK_OK(rt_reorder_faces((const uint32_t*)faces, indices, count, (uint32_t*)tmp.getPointer(), nullptr));
  RK_CHECK(cudaMemcpy(faces, tmp.getPointer(), (size_t)count * sizeof(uint4), cudaMemcpyDeviceToDevice) == cudaSuccess, "copy");
}

}  // namespace renderkit
