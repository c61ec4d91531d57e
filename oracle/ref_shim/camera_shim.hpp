// camera_shim.hpp -- a CUDACamera with the members that the reference's
// angleFromDir / lookAt (CUDACamera.cpp:70-88,126-133) and CUDA_calcPrimaryRays
// (kernels/CUDA_calcPrimaryRays.cu:43-55) touch. TEST INFRASTRUCTURE ONLY.
namespace renderkit {
class CUDACamera {
 public:
  float fov, ratio;
  float3 center, angle, dir;
  bool dirty;
  void angleFromDir();
  void lookAt(float _x, float _y, float _z);
  float getFOV() { return fov; }
  float getRatio() { return ratio; }
  float3 getCenter() { return center; }
  float pitch() { return angle.x; }
  float yaw() { return angle.y; }
  float roll() { return angle.z; }
};
}  // namespace renderkit
using namespace renderkit;
