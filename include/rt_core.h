/* rt_core.h -- C ABI of the B200 LBVH build + closest-hit traversal core.
 *
 * A drop-in for the reference's LBVH / ray-tracing path (gatouillatpy/cudart):
 * every entry point below names the reference function it replaces
 * (file:line in the reference tree). Conventions:
 *   - all pointers are device pointers unless a comment says "host";
 *   - all calls are asynchronous on the caller's stream and never synchronize
 *     (no host round trips: counts stay on the device);
 *   - the library allocates nothing on its hot paths: callers pass scratch
 *     buffers sized by the *_scratch_bytes queries;
 *   - errors are returned as rt_status (the reference printed and exit()ed,
 *     CUDACommon.h:123-133); device-side failures (stack or capacity overflow)
 *     are reported in rt_build_info.error / the trace error word;
 *   - there is no CPU fallback: without a CUDA device every compute call
 *     returns RT_ERR_NO_DEVICE.
 * Layouts match the reference: vertices are float4 (CUDAMesh.h), faces uint4
 * (a, b, c, material), aabox is float4 min + float4 max (CUDABox.h:17-148),
 * bvnode is 32 bytes (CUDANode.h:20-50): word0 bit0 = leaf flag, bits 1-2 =
 * split axis (internal) or bits 1-31 = triangle count (leaf), word1 = left
 * child id (right = left + 1) or first triangle position, then float3 box_min,
 * float3 box_max.
 */
#ifndef RT_CORE_H
#define RT_CORE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* rt_stream; /* a cudaStream_t; NULL = legacy default stream */

/* Layout version of the structs below. A caller compiled against this header
 * must check rt_abi_version() == RT_ABI_VERSION before passing any struct:
 * a library built from a different header reads different field offsets. */
#define RT_ABI_VERSION 11u

typedef enum rt_status {
  RT_OK = 0,
  RT_ERR_INVALID_ARGUMENT = 1,
  RT_ERR_NO_DEVICE = 2,
  RT_ERR_CUDA = 3,
  RT_ERR_SCRATCH_TOO_SMALL = 4,
  RT_ERR_CAPACITY = 5,
  RT_ERR_UNSUPPORTED = 6
} rt_status;

/* Device-side error bits (rt_build_info.error, trace error word). */
#define RT_DEVERR_NODE_CAPACITY 0x1u  /* more nodes than max_nodes */
#define RT_DEVERR_STACK_OVERFLOW 0x2u /* traversal stack exhausted (result of that ray may be wrong) */
#define RT_DEVERR_MORTON_CAPACITY 0x4u
#define RT_DEVERR_WAIT_TIMEOUT 0x8u    /* a bounded wait inside a kernel ran out (2 s); that kernel's output is invalid */
#define RT_DEVERR_ACCEL_MISSING 0x10u  /* the blob lacks the tree the schedule walks (or was built for other sizes) */

typedef struct rt_build_params {
  uint32_t tree_depth;    /* Morton levels; reference default 12 (CUDAMeshTree.h:118); 1..32 */
  uint32_t tree_complete; /* 1: split leaves above max_leaf by median and reorder faces (CUDAMeshTree.cpp:88-91) */
  uint32_t min_leaf;      /* 16, kernels/CUDA_buildMeshTreeLBVH.cu:39 (0 = default) */
  uint32_t max_leaf;      /* 224, kernels/CUDA_buildMeshTreeLBVH.cu:40 (0 = default) */
  uint32_t morton_bits;   /* 32: reference 11/11/10 interleave; 30: 10/10/10 left-aligned (0 = 32) */
  uint32_t accel_trees;   /* traversal trees written into the blob besides the node records: RT_ACCEL_* bits (0 = none) */
  uint32_t cluster_leaf;  /* RT_ACCEL_CLUSTERS: most positions per cluster tree leaf, 1..8 (0 = 3) */
} rt_build_params;

/* rt_build_params.accel_trees. The blob always holds records of the build's
 * node tree (whose leaves hold ~N / 2^tree_depth triangles). RT_ACCEL_CLUSTERS
 * adds the cluster tree: the binary radix tree of the sorted (Morton code,
 * position) keys, cut at subtrees of at most cluster_leaf positions and stored
 * as 4-wide records (two more launches; scratch grows by ~76 bytes per face;
 * meshes below 2^28 faces), walked by the RT_TRACE_CLUSTERS schedules. No
 * reference counterpart. */
#define RT_ACCEL_CLUSTERS 0x2u

/* Written by rt_lbvh_build on the device. */
typedef struct rt_build_info {
  uint32_t node_count;     /* nodes written (2 * leaf_count - 1) */
  uint32_t leaf_count;
  uint32_t real_depth;     /* max leaf level + 1, as the reference computes it (:450-452) */
  uint32_t split_count;    /* adjacent code pairs that differ */
  uint32_t overrun_visits; /* Morton visits whose split search ran past the level's own list */
  uint32_t nondet_reads;   /* split reads from levels deeper than tree_depth (unordered in the reference) */
  uint32_t past_end_reads; /* split reads past the end of the list (undefined in the reference) */
  uint32_t error;          /* RT_DEVERR_* bits */
} rt_build_info;

typedef struct rt_build_desc {
  const float* vertices;    /* float4[vertex_count] */
  uint32_t vertex_count;
  uint32_t face_count;      /* N */
  const uint32_t* faces_in; /* uint4[N] */
  uint32_t* faces_out;      /* uint4[N]: faces in Morton (position) order; may equal faces_in */
  const float* hitbox;      /* HOST float[8] = min xyzw, max xyzw (CUDAMesh::getHitbox); NULL = min/max of all vertices */
  rt_build_params params;
  float* boxes;             /* aabox[N] per original face (CUDAMeshTree::boxes) */
  uint32_t* indices;        /* uint[N]: position -> original face id (CUDAMeshTree::indices) */
  uint32_t* codes;          /* uint[N]: sorted Morton codes; NULL = kept in scratch */
  uint32_t* nodes;          /* bvnode[max_nodes] (CUDAMeshTree::nodes) */
  uint32_t max_nodes;       /* >= 2N - 1 (rt_lbvh_scratch_bytes' max_nodes); smaller: RT_ERR_CAPACITY before any launch */
  float* tris;              /* float4[3N] {v0, v1 - v0, v2 - v0} per position (w = 0); NULL = not produced */
  rt_build_info* info;      /* device pointer, may be NULL */
  void* scratch;
  size_t scratch_bytes;
  void* accel;              /* optional traversal blob (needs tris and tree_complete); NULL = not produced */
  size_t accel_bytes;       /* >= rt_lbvh_accel_bytes */
} rt_build_desc;

/* Scratch bytes and the node-count bound for an N-face build.
 * Replaces the temporaries CUDA_buildMeshTreeLBVH cudaMalloc'd per call
 * (kernels/CUDA_buildMeshTreeLBVH.cu:462-471). */
rt_status rt_lbvh_scratch_bytes(uint32_t face_count, const rt_build_params* params, size_t* scratch_bytes, uint32_t* max_nodes);

/* Bytes of the optional traversal blob of an N-face build: two-child records
 * of the internal nodes (both children's padded boxes, indexed by pre-order
 * rank), the leaf table, one padded box per 8 consecutive triangles of a
 * leaf, 4-wide records, and room for the cluster tree (RT_ACCEL_CLUSTERS,
 * 128 bytes per face). Derived from the same build; the nodes stay the
 * reference's. No reference counterpart (the reference traverses bvnodes
 * directly). */
rt_status rt_lbvh_accel_bytes(uint32_t face_count, size_t* bytes);

/* LBVH build: boxes, Morton codes, key+index sort, split lists, topology,
 * node boxes, face reorder and triangle pre-gather.
 * Replaces CUDA_buildMeshTreeLBVH (kernels/CUDA_buildMeshTreeLBVH.cu:457-681),
 * called by CUDAMeshTree::buildMeshTreeLBVH (CUDAMeshTree.cpp:88-91). */
rt_status rt_lbvh_build(const rt_build_desc* desc, rt_stream stream);

/* Batched build of M meshes in one set of launches (no per-mesh host work).
 * Faces and vertices of all meshes are concatenated; face_offsets[m] and
 * vertex_offsets[m] (DEVICE arrays of M + 1 entries) delimit mesh m, and its
 * faces index its own vertices from 0; every mesh has at least one face.
 * Every per-mesh output equals what
 * rt_lbvh_build gives for that mesh alone (same bits), stored at fixed
 * offsets derived from F_m = face_offsets[m]:
 *   faces_out, boxes, codes, tris, indices  at position F_m (indices hold mesh-local face ids),
 *   nodes                                   at node 2 F_m - m (capacity 2 n_m - 1),
 *   info                                    at entry m,
 *   accel                                   the batched traversal blob (rt_batch_trace).
 * The hit box of each mesh is the min/max of its vertices. No reference
 * counterpart (the reference builds one mesh per call). */
typedef struct rt_batch_build_desc {
  uint32_t mesh_count;
  uint32_t face_count;            /* total */
  uint32_t vertex_count;          /* total */
  const uint32_t* face_offsets;   /* DEVICE [mesh_count + 1] */
  const uint32_t* vertex_offsets; /* DEVICE [mesh_count + 1] */
  const float* vertices;
  const uint32_t* faces_in;
  uint32_t* faces_out;            /* must not alias faces_in */
  rt_build_params params;         /* tree_complete must be 1 */
  float* boxes;
  uint32_t* indices;
  uint32_t* codes;
  uint32_t* nodes;                /* >= 2 * face_count - mesh_count records */
  float* tris;
  void* accel;
  size_t accel_bytes;
  rt_build_info* info;            /* DEVICE [mesh_count] */
  void* scratch;
  size_t scratch_bytes;
} rt_batch_build_desc;
rt_status rt_batch_sizes(uint32_t mesh_count, uint32_t face_count, const rt_build_params* params, size_t* scratch_bytes,
                         size_t* accel_bytes);
rt_status rt_batch_build(const rt_batch_build_desc* desc, rt_stream stream);

/* One traversal launch for the rays of all meshes of a batched build: the rays
 * of mesh m are ray_offsets[m] .. ray_offsets[m+1] (DEVICE, M + 1 entries).
 * Hit ids are positions (id_mode 0) or face ids (id_mode 1) inside the mesh. */
typedef struct rt_batch_trace_desc {
  uint32_t mesh_count;
  const uint32_t* face_offsets;   /* DEVICE [mesh_count + 1], as given to rt_batch_build */
  const uint32_t* ray_offsets;    /* DEVICE [mesh_count + 1] */
  const void* accel;              /* from rt_batch_build */
  const float* tris;
  const uint32_t* indices;
  uint32_t face_count;            /* total, as given to rt_batch_build */
  const float* orig;
  const float* dir;
  const float* tmax;              /* optional */
  uint32_t ray_count;             /* at most RT_MAX_RAYS */
  uint32_t id_mode;
  int32_t* hit_id;
  float* hit_t;
  float* hit_uv;
  uint32_t* ray_visits;
  uint32_t* ray_tests;
  uint32_t* error_word;
  uint32_t schedule;              /* RT_TRACE_WHILE_WHILE, RT_TRACE_WIDE, RT_TRACE_COOP (with work_counter) */
  uint32_t* work_counter;         /* optional device word: persistent warps fetch rays through it (the call zeroes it) */
  uint32_t persistent_blocks_per_sm; /* with work_counter: CTAs of 128 threads per SM (0 = 8) */
  const uint32_t* ray_order;      /* optional DEVICE permutation of the rays: threads take rays in this order
                                     (rt_batch_ray_order, rt_image_tile_order); results stay in each ray's own slot */
  uint32_t lane_threshold;        /* as in rt_trace_desc */
  /* Optional (all three or none; id_mode 0): each ray's diffuse bounce, as rt_batch_bounce_rays makes it from the
     hits of this call with bounce_seed (float4 origins and directions, float tmax, ray_count entries each; a ray
     that hit nothing gets tmax -1). The packet schedule (RT_TRACE_CLUSTERS | RT_TRACE_PACKET with a work_counter)
     writes them as each ray finishes; every other schedule launches rt_batch_bounce_rays' kernel after the trace.
     They share no byte with each other or with orig, dir, tmax and the hit arrays (else RT_ERR_INVALID_ARGUMENT). */
  uint64_t bounce_seed;
  float* bounce_orig;
  float* bounce_dir;
  float* bounce_tmax;
} rt_batch_trace_desc;
rt_status rt_batch_trace(const rt_batch_trace_desc* desc, rt_stream stream);

/* A tracing order for the rays of a batched trace: ray indices sorted by mesh
 * (ray_offsets, DEVICE, mesh_count + 1 entries), then by direction octant, then
 * by the top morton_bits bits (0, 3, .., 21; fewer when the mesh id, octant and
 * Morton bits would not fit in 32 bits) of the 21-bit Morton code of the
 * origin inside box (min xyz, max xyz, HOST); rays with tmax <= 0 go last; the
 * sort is stable, so rays with equal keys keep their order. Scratch as for
 * rt_ray_order. No reference counterpart. */
rt_status rt_batch_ray_order_scratch_bytes(uint32_t count, size_t* scratch_bytes);
rt_status rt_batch_ray_order(const float* orig, const float* dir, const float* tmax, uint32_t count, const uint32_t* ray_offsets,
                             uint32_t mesh_count, const float box[6], uint32_t morton_bits, uint32_t* order, void* scratch,
                             size_t scratch_bytes, rt_stream stream);

/* A tracing order for `images` row-major width x height images stored one after
 * the other (width % 8 == 0, height % 4 == 0): each run of 32 slots is an 8 x 4
 * pixel tile of one image. No reference counterpart. */
rt_status rt_image_tile_order(uint32_t images, uint32_t width, uint32_t height, uint32_t* order, rt_stream stream);

/* Per-face boxes and indices[k] = k.
 * Replaces CUDA_calcMeshBoxes (kernels/CUDA_calcMeshBoxes.cu:65-104). */
rt_status rt_mesh_boxes(const float* vertices, const uint32_t* faces, uint32_t face_count, float* boxes, uint32_t* indices, rt_stream stream);

/* faces_out[n] = faces_in[indices[n]]; faces_out must not overlap faces_in.
 * Replaces CUDA_reorderMeshFaces (kernels/CUDA_reorderMeshFaces.cu:44-83). */
rt_status rt_reorder_faces(const uint32_t* faces_in, const uint32_t* indices, uint32_t face_count, uint32_t* faces_out, rt_stream stream);

/* Stable LSD radix sort of (key, value) pairs on the low 8*ceil(bit_depth/8)
 * bits of the keys; init_values = 1 sets values to 0..n-1 first.
 * Replaces CUDA_radixSortGeneral (kernels/CUDA_radixSortGeneral.cu:397-482)
 * and its small-size targets CUDA_bubbleSort512 (kernels/CUDA_bubbleSort512.cu:114)
 * and CUDA_bitonicSortGeneral<uint,uint> (kernels/CUDA_bitonicSortGeneral.cu:505),
 * which only guarantee ascending keys; ties here keep the input order. */
rt_status rt_sort_scratch_bytes(uint32_t n, size_t* scratch_bytes);
rt_status rt_radix_sort_pairs(uint32_t* keys, uint32_t* values, uint32_t n, uint32_t bit_depth, int init_values,
                              void* scratch, size_t scratch_bytes, rt_stream stream);
/* Keys only. Replaces CUDA_radixSort (kernels/CUDA_radixSort.cu:357) and
 * CUDA_bitonicSort<uint> (kernels/CUDA_bitonicSort.cu:403). */
rt_status rt_radix_sort_keys(uint32_t* keys, uint32_t n, uint32_t bit_depth, void* scratch, size_t scratch_bytes, rt_stream stream);

/* Allocation-free variant of rt_radix_sort_pairs, for callers that cannot
 * allocate device memory where they sort (a plug-in whose host application
 * owns every device allocation; a frame loop that cannot afford cudaMalloc /
 * cudaFree, which may synchronize the device). No counterpart in the
 * reference. Same results as rt_radix_sort_pairs. Its scratch is a
 * RT_STATIC_SORT_SCRATCH_BYTES array inside the library that every GPU using
 * the library holds until the process exits; n above RT_STATIC_SORT_MAX_N is
 * refused with RT_ERR_CAPACITY. The first call on a device looks up the
 * array's device address (make it before any stream capture). All calls share
 * the array: calls that overlap on the GPU race and must be serialized. */
#define RT_STATIC_SORT_MAX_N (1u << 20)
#define RT_STATIC_SORT_SCRATCH_BYTES ((9u << 20) + (16u << 10))
rt_status rt_radix_sort_pairs_static(uint32_t* keys, uint32_t* values, uint32_t n, uint32_t bit_depth, int init_values,
                                     rt_stream stream);

/* Camera state of CUDACamera (CUDACamera.h:15-321) that ray generation reads. */
typedef struct rt_camera {
  float center[3];
  float angle[3]; /* pitch, yaw, roll (CUDACamera::pitch/yaw/roll) */
  float fov;      /* radians; CUDACamera default PI/2 */
  float ratio;    /* width / height; CUDACamera default 4/3 */
} rt_camera;

/* HOST. CUDACamera::lookAt (CUDACamera.cpp:126-132 -> angleFromDir :70-88). */
rt_status rt_camera_look_at(rt_camera* camera, const float target[3]);
/* HOST. The four float4 (origin, dir, step x, step y) of CUDA_calcPrimaryRays
 * (kernels/CUDA_calcPrimaryRays.cu:43-55). */
rt_status rt_camera_basis(const rt_camera* camera, uint32_t width, uint32_t height, float basis[16]);
/* One pinhole ray per pixel, row-major, float4 origin and direction.
 * Replaces CUDA_calcPrimaryRays (kernels/CUDA_calcPrimaryRays.cu:20-69). */
rt_status rt_primary_rays(const rt_camera* camera, uint32_t width, uint32_t height, float* orig, float* dir, rt_stream stream);
/* The rays of `count` cameras in one launch: camera c's width x height rays at
 * rows c * width * height. `bases` is a DEVICE float[16 * count], camera c's
 * rt_camera_basis at 16 c (made once while the cameras stay put); the rays are
 * bit-identical to rt_primary_rays per camera. No reference counterpart. */
rt_status rt_batch_primary_rays(const float* bases, uint32_t count, uint32_t width, uint32_t height, float* orig, float* dir,
                                rt_stream stream);

typedef struct rt_trace_desc {
  const uint32_t* nodes;    /* bvnode[] from rt_lbvh_build */
  const float* tris;        /* float4[3N] from rt_lbvh_build; NULL = read vertices + faces as the reference does */
  const float* vertices;    /* float4[], used when tris == NULL */
  const uint32_t* faces;    /* uint4[] in position order (the reordered faces), used when tris == NULL */
  const uint32_t* indices;  /* position -> original id, used when id_mode == 1 */
  const float* orig;        /* float4[ray_count] */
  const float* dir;         /* float4[ray_count] */
  const float* tmax;        /* float[ray_count] initial depth; NULL = CUDART_NORM_HUGE_F. A ray with tmax <= 0 misses. */
  uint32_t ray_count;       /* at most RT_MAX_RAYS */
  uint32_t id_mode;         /* 0: position in the reordered faces (the reference's faces_id); 1: original face id */
  int32_t* hit_id;          /* out: -1 on a miss */
  float* hit_t;             /* out: t of the hit, or tmax on a miss (may alias tmax, as CUDABuffer depths do) */
  float* hit_uv;            /* out: float2 (u, v); (0, 0) on a miss */
  uint32_t* ray_visits;     /* optional out: nodes popped per ray */
  uint32_t* ray_tests;      /* optional out: triangles tested per ray */
  uint32_t* error_word;     /* optional device word: RT_DEVERR_* bits are OR-ed in */
  const void* accel;        /* optional traversal blob from rt_lbvh_build (with tris): faster, same results */
  uint32_t face_count_hint; /* the face count the blob was built for (required with accel) */
  /* schedule of the blob traversal (results never depend on it): */
  uint32_t image_width;     /* > 0 and dividing ray_count: rays are a row-major image; a warp takes an 8x4 pixel tile */
  uint32_t* work_counter;   /* optional device word: persistent warps fetch rays through it (the call zeroes it) */
  uint32_t persistent_blocks_per_sm; /* with work_counter: CTAs of 128 threads per SM (0 = 8) */
  uint32_t schedule;        /* RT_TRACE_* bits */
  const uint32_t* ray_order; /* optional permutation from rt_ray_order: threads take rays in this order */
  uint32_t treelet_depth;   /* persistent 4-wide walks: levels of 4-wide records below the root (0..4, at most 85
                               records, 10.9 KB) that each CTA copies to shared memory and reads from there (0: none) */
  uint32_t lane_threshold;  /* RT_TRACE_PACKET: a warp leaves the packet walk for per-lane walks (from the same stacks)
                               once fewer than this many lanes still want the node it is at (0: never);
                               RT_TRACE_REFILL: a warp fetches new rays for its idle lanes once this many are idle */
} rt_trace_desc;

/* The most rays one trace call takes (2^31 - 1, 64 GB of origins and directions): the persistent schedules' slot
   counters then never wrap. A larger ray_count is refused with RT_ERR_INVALID_ARGUMENT before any launch. */
#define RT_MAX_RAYS 0x7FFFFFFFu

#define RT_TRACE_WHILE_WHILE 0x1u /* descend until a leaf is held, then test it (else: interleaved) */
#define RT_TRACE_COOP 0x2u        /* the warp's lanes share the triangle tests of all its rays' leaves */
#define RT_TRACE_WIDE 0x4u /* descend through the blob's 4-wide records */
#define RT_TRACE_CLUSTERS 0x8u /* walk the blob's cluster tree (built with RT_ACCEL_CLUSTERS; else every ray reports a miss
                                  and RT_DEVERR_ACCEL_MISSING is raised); WIDE is ignored */
#define RT_TRACE_PACKET 0x10u  /* with RT_TRACE_CLUSTERS and a work_counter: each warp walks the cluster tree as one packet
                                  (one node sequence for its 32 rays; for coherent rays such as 8 x 4 pixel tiles) */
#define RT_TRACE_REFILL 0x20u  /* with RT_TRACE_CLUSTERS and a work_counter: per-lane walks in which a warp takes new rays
                                  for its idle lanes (lane_threshold of them, 0 = 16) instead of waiting for its slowest ray;
                                  it claims 32 slots per atomic, writes the inactive ones (tmax <= 0) as misses at once and
                                  queues the active ones for its lanes */

/* A tracing order for incoherent rays: ray indices sorted by direction octant,
 * then by the Morton code of the origin inside box (min xyz, max xyz, HOST);
 * rays with tmax <= 0 go last. Feed it to rt_trace_desc.ray_order (results
 * stay in each ray's own slot). No reference counterpart. */
rt_status rt_ray_order_scratch_bytes(uint32_t count, size_t* scratch_bytes);
rt_status rt_ray_order(const float* orig, const float* dir, const float* tmax, uint32_t count, const float box[6], uint32_t* order,
                       void* scratch, size_t scratch_bytes, rt_stream stream);

/* Closest hit per ray: the minimum (t, position) over all triangles that the
 * Moller-Trumbore test of kernels/CUDA_raytraceMeshTree.cu:57-89 accepts with
 * t < tmax. Replaces CUDA_raytraceMeshTree (kernels/CUDA_raytraceMeshTree.cu:434-480)
 * called by CUDARaytracer::raytraceMeshTree (CUDARaytracer.cpp:130-135). */
rt_status rt_trace_closest(const rt_trace_desc* desc, rt_stream stream);

typedef struct rt_interp_desc {
  const int32_t* hit_id;   /* from rt_trace_closest with id_mode 0 (face positions); < 0 = miss */
  const float* hit_uv;     /* float2 per ray */
  uint32_t count;          /* rays */
  const uint32_t* faces;   /* uint4 faces indexed by hit_id (the build's reordered faces) */
  const float* vertices;   /* float4 per vertex */
  const float* normals;    /* optional float4 per vertex (CUDAMesh::getNormalsArray); NULL = face normal */
  const float* colors;     /* optional float4 per vertex; NULL = white */
  const float* texcoords;  /* optional float2 per vertex; NULL = (u, v) */
  float* out_points;       /* optional outputs, one per ray: float4 */
  float* out_normals;      /* float4 */
  float* out_colors;       /* float4 */
  float* out_texcoords;    /* float2 */
  uint32_t* out_materials; /* face.w */
} rt_interp_desc;

/* Hit point, normal, color, texcoord and material per ray from (face, u, v).
 * Replaces CUDA_interpolateData (kernels/CUDA_interpolateData.cu:216-256),
 * called by CUDARaytracer::interpolateOutputSurfaces (CUDARaytracer.cpp:144-162).
 * Misses write zeros. */
rt_status rt_interpolate(const rt_interp_desc* desc, rt_stream stream);

/* One cosine-weighted diffuse bounce per hit (PCG32 stream = ray index);
 * misses give an inactive ray with tmax = -1. Workload generation for the
 * incoherent scene; no reference counterpart. */
rt_status rt_bounce_rays(const float* tris, const float* orig, const float* dir, const int32_t* hit_pos, const float* hit_t,
                         uint32_t ray_count, uint64_t seed, float* orig_out, float* dir_out, float* tmax_out, rt_stream stream);
/* rt_bounce_rays for the rays of a batched build: hit_pos holds positions inside
 * each ray's own mesh (rt_batch_trace, id_mode 0), the rays of mesh m being
 * ray_offsets[m] .. ray_offsets[m+1] (DEVICE, mesh_count + 1 entries), and
 * face_offsets (DEVICE, as given to rt_batch_build) place each mesh in tris.
 * Same rays as rt_bounce_rays given the global positions. Optional order_out
 * (DEVICE, ray_count entries, with order_counters: 2 DEVICE words the call
 * zeroes): a tracing order for rt_batch_trace_desc.ray_order, the active rays
 * first, in runs of neighbouring rays (ray order inside each run of 1024
 * rays). No reference counterpart. */
rt_status rt_batch_bounce_rays(const float* tris, const uint32_t* face_offsets, const uint32_t* ray_offsets, uint32_t mesh_count,
                               const float* orig, const float* dir, const int32_t* hit_pos, const float* hit_t, uint32_t ray_count,
                               uint64_t seed, float* orig_out, float* dir_out, float* tmax_out, uint32_t* order_out,
                               uint32_t* order_counters, rt_stream stream);

/* Hits packed for download: the (t, u, v) of every ray whose hit_id >= 0, in ray order, as float[3 * hits] in
 * `packed` (DEVICE, room for 3 * count floats), and the number of those rays in *packed_count (DEVICE word). With
 * the ids, downloaded as they are, the host rebuilds every hit exactly: a ray with id -1 has t = the tmax it was
 * traced with (CUDART_NORM_HUGE_F without one) and uv = 0. Scratch: rt_pack_hits_scratch_bytes. No reference
 * counterpart. */
rt_status rt_pack_hits_scratch_bytes(uint32_t count, size_t* scratch_bytes);
rt_status rt_pack_hits(const int32_t* hit_id, const float* hit_t, const float* hit_uv, uint32_t count, float* packed,
                       uint32_t* packed_count, void* scratch, size_t scratch_bytes, rt_stream stream);

/* Mesh and tree chunk files (HOST calls; arrays may be device or host memory).
 * Same bytes as CUDAMesh::quickSave / CUDAMeshTree::quickSave with
 * overwrite = true (CUDAMesh.cpp:253-400, CUDAMeshTree.cpp:194-289); readers
 * follow CUDAMesh::quickLoad / CUDAMeshTree::quickLoad (CUDAMesh.cpp:134-251,
 * CUDAMeshTree.cpp:114-192) but require stored counts EQUAL to the buffers'
 * (the reference's tree loader inverts that check), and appending
 * (overwrite = 0) writes whole chunks (the reference's append mode corrupts
 * the chunk lengths). A NULL array pointer skips that chunk; *_info fills the
 * counts (and the hit box) so that the caller can size the buffers. */
typedef struct rt_mesh_file {
  float hitbox[8];
  int32_t has_hitbox;
  uint32_t vertex_count, normal_count, color_count, texcoord_count, face_count;
  float* vertices;   /* float4 */
  float* normals;    /* float4 */
  float* colors;     /* float4 */
  float* texcoords;  /* float2 */
  uint32_t* faces;   /* uint4 */
} rt_mesh_file;
typedef struct rt_tree_file {
  uint32_t node_count, index_count, box_count;
  uint32_t* nodes;    /* bvnode */
  uint32_t* indices;  /* uint */
  float* boxes;       /* aabox */
} rt_tree_file;
rt_status rt_mesh_file_save(const char* path, int overwrite, const rt_mesh_file* mesh);
rt_status rt_mesh_file_info(const char* path, rt_mesh_file* mesh);
rt_status rt_mesh_file_load(const char* path, rt_mesh_file* mesh);
rt_status rt_tree_file_save(const char* path, int overwrite, const rt_tree_file* tree);
rt_status rt_tree_file_info(const char* path, rt_tree_file* tree);
rt_status rt_tree_file_load(const char* path, rt_tree_file* tree);

const char* rt_status_string(rt_status status);
uint32_t rt_version(void);
/* RT_ABI_VERSION of the header the library was built with. */
uint32_t rt_abi_version(void);
/* RT_OK when a CUDA device is usable, RT_ERR_NO_DEVICE otherwise. */
rt_status rt_device_check(void);
/* Kernels this library has launched in this process (to count the kernels of a timed region). */
uint64_t rt_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* RT_CORE_H */
