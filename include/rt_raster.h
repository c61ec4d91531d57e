/* rt_raster.h -- C ABI of the rasteriser (sm_100a): an alternative primary-
 * visibility producer writing the same per-pixel face id / (u, v) / depth
 * surfaces as the traversal.
 *
 * Replaces CUDA_rasterizeMeshTree (kernels/CUDA_rasterizeMeshTree.cu:255-297),
 * called by CUDARaytracer::rasterizeMeshTree (CUDARaytracer.cpp:137-142).
 * Semantics of its kernel (:77-225): every vertex is transformed by
 * transpose(view * proj) and divided by |w|; a face whose screen rectangle
 * misses [-1, 1]^2 is dropped; otherwise it is tested on the 8 x 4 pixel zones
 * of its zone rectangle (start rounded down to an even zone) at each pixel's
 * corner (x * 2 / width - 1, 1 - y * 2 / height) with a 2-D barycentric test
 * (|det| < 1e-6 rejected); a pixel takes the face of smallest depth t > 0,
 * the earliest face on equal depth (the reference tests faces in index order).
 */
#ifndef RT_RASTER_H
#define RT_RASTER_H

#include "rt_core.h"

#ifdef __cplusplus
extern "C" {
#endif

/* HOST. The camera's view direction after CUDACamera::lookAt(target)
 * (CUDACamera.cpp:126-132, angleFromDir :70-72): (target - center) * (1 / sqrtf(|.|^2)). */
rt_status rt_camera_view_dir(const rt_camera* camera, const float target[3], float dir[3]);
/* HOST. transpose(view * proj) as CUDACamera::update (CUDACamera.cpp:245-266)
 * builds it for a camera at camera->center with view direction `dir`
 * (CUDACamera::dir: rt_camera_view_dir after a lookAt), roll camera->angle[2],
 * camera->fov / ratio, near plane 1.0, far plane 1999.999. A camera looking
 * exactly along z gets a NaN matrix, as in the reference (its roll axis
 * (dir.x, 0, dir.y) is zero). */
rt_status rt_raster_matrix(const rt_camera* camera, const float dir[3], float matrix[16]);

typedef struct rt_raster_desc {
  const float* vertices; /* float4 per vertex */
  uint32_t vertex_count;
  const uint32_t* faces; /* uint4 per face */
  uint32_t face_count;
  float matrix[16];      /* rt_raster_matrix */
  uint32_t width, height;
  uint32_t id_mode;      /* 0: face index; 1: the reference's value, face - face % 192 (it writes its cache block start) */
  int32_t* face_id;      /* [width * height], updated where a face wins (CUDABuffer clears it to 0) */
  float* uv;             /* [width * height] float2, updated with the winner's (u, v) */
  float* depth;          /* [width * height], read and updated (CUDABuffer clears it to +HUGE) */
  uint32_t pair_capacity; /* (zone, face) pairs per chunk; 0 = 16M; at least 128 faces' worth (128 x zone count) */
  void* scratch;          /* rt_raster_scratch_bytes for the same face count, size and pair_capacity */
  size_t scratch_bytes;
  uint32_t* error_word;  /* optional: RT_DEVERR_NODE_CAPACITY when a face names a vertex past vertex_count (the face is skipped) */
} rt_raster_desc;

rt_status rt_raster_scratch_bytes(uint32_t face_count, uint32_t width, uint32_t height, uint32_t pair_capacity, size_t* bytes);
/* Rasterises the faces into the surfaces. Waits for the stream once (it reads
 * the per-block zone counts to cut the faces into chunks that fit the scratch). */
rt_status rt_rasterize(const rt_raster_desc* d, rt_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* RT_RASTER_H */
