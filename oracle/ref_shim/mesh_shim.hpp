// mesh_shim.hpp -- host stand-ins for CUDAArray / CUDAMesh / CUDAMeshTree with
// the members that the reference's quickLoad / quickSave (CUDAMesh.cpp:134-400,
// CUDAMeshTree.cpp:194-289) use. Arrays live in host memory. _assert records a
// failure instead of exiting. TEST INFRASTRUCTURE ONLY.
static int g_assert_failures = 0;
static inline void _assert(bool ok, const char*, int, const char*) { if (!ok) ++g_assert_failures; }
namespace renderkit {
template <typename T>
struct CUDAArray {
  std::vector<T> data;
  explicit CUDAArray(uint n) : data(n) {}
  uint getUnitCount() const { return (uint)data.size(); }
  void copyDataFromHost(const T* p) { memcpy(data.data(), p, data.size() * sizeof(T)); }
  void copyDataToHost(T* p) const { memcpy(p, data.data(), data.size() * sizeof(T)); }
};
class CUDAMesh {
 public:
  aabox hitbox;
  CUDAArray<float4>* vertices = nullptr;
  CUDAArray<float4>* normals = nullptr;
  CUDAArray<float4>* colors = nullptr;
  CUDAArray<float2>* texcoords = nullptr;
  CUDAArray<uint4>* faces = nullptr;
  void quickLoad(char* path);
  void quickSave(char* path, bool overwrite);
};
class CUDAMeshTree {
 public:
  CUDAArray<bvnode>* nodes = nullptr;
  CUDAArray<aabox>* boxes = nullptr;
  CUDAArray<uint>* indices = nullptr;
  void quickSave(char* path, bool overwrite);
};
}  // namespace renderkit
using namespace renderkit;
