#!/usr/bin/env bash
# build_ref.sh -- compiles selected functions of the reference's own source
# files into host-side checker libraries under oracle/_ref/ (git-ignored).
#
# The reference cannot be built as a whole here: its kernels use CUDA texture
# references and string-named symbol copies that CUDA 12 removed, and
# CUDACommon.h includes headers of an external project that are not vendored.
# The functions that carry the hot path's arithmetic and control flow are plain
# C/C++ though, so this recipe feeds exact line ranges of the reference files
# (through stdin; no copy is written anywhere) into g++ between the shim pieces
# in oracle/ref_shim/, which stand in for the CUDA 1.x facilities. Each range is
# preceded by a #line directive, so diagnostics point at the reference file.
#
# Output: oracle/_ref/libref_cudart.so exporting ref_mesh_boxes, ref_lbvh_build,
# ref_reorder_faces, ref_trace, ref_camera_rays, ref_interpolate, ref_mesh_quick_save,
# ref_mesh_quick_load, ref_tree_quick_save, ref_sah_build, ref_raster_matrix,
# ref_rasterize. TEST INFRASTRUCTURE ONLY.
#
# Usage: oracle/build_ref.sh [reference_root]   (default: $CUDART_REFERENCE)
set -euo pipefail
REF="${1:-${CUDART_REFERENCE:-}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
SHIM="$HERE/ref_shim"
OUT="$HERE/_ref"
if [ -z "$REF" ] || [ ! -d "$REF/kernels" ]; then
  echo "build_ref.sh: reference not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"

# rng FILE FIRST LAST -- emit a line range of a reference file with a #line marker
rng() { echo "#line $2 \"$1\""; sed -n "$2,$3p" "$REF/$1"; }

CXXFLAGS=(-O2 -ffp-contract=off -fno-strict-aliasing -w -shared -fPIC -std=c++17)

build_tu() {  # build_tu NAME [extra flags]  (reads the TU from stdin)
  local name="$1"; shift
  g++ "${CXXFLAGS[@]}" "$@" -x c++ - -c -o "$OUT/$name.o"
}

S=kernels/CUDA_buildMeshTreeSAH.cu
{
  echo "#define SHIM_THREADED 1"
  cat "$SHIM/prelude.hpp"
  cat "$SHIM/sah_shim.hpp"
  echo "namespace renderkit {"
  rng CUDABin.h 15 113   # bvbin
  echo "}"
  echo "namespace tu_sah {"
  rng "$S" 31 40      # item
  rng "$S" 46 56      # BLOCK_SIZE, SM_BIN_COUNT, STACK_SIZE, costs, leaf sizes
  rng "$S" 62 67      # __device__ mutex, stack, sp, node_count
  rng "$S" 73 73      # texture tex_boxes
  rng "$S" 79 159     # stack_push_global, stack_push, stack_pop, make_node, make_leaf
  rng "$S" 224 666    # kernel_buildMeshTree, kernel_initStack
  cat "$SHIM/sah_epilogue.hpp"
  echo "}"
} | build_tu ref_sah

Z=kernels/CUDA_rasterizeMeshTree.cu
{
  echo "#define SHIM_THREADED 1"
  cat "$SHIM/prelude.hpp"
  cat "$SHIM/sah_shim.hpp"
  cat "$SHIM/raster_shim.hpp"
  echo "namespace tu_raster {"
  rng types/_cuda_float4.h 135 140      # operator/=(float4, float): multiply by the reciprocal
  rng types/_cuda_float4.h 210 227      # cross(float4, float4, float4)
  rng types/_cuda_float4x4.h 11 140     # float4x4, determinant, transpose, inverse
  rng types/_cuda_float4x4.h 142 167    # matrixMultiply
  rng types/_cuda_float4x4.h 183 198    # matrixTransform (both forms)
  rng types/_cuda_float4x4.h 323 350    # matrixRotationAxis
  rng types/_cuda_float4x4.h 398 426    # matrixPerspectiveFov, matrixLookAt
  echo "namespace renderkit {"
  echo "class CUDACamera { public: float3 center, dir, angle; float fov, ratio, zNearPlane, zFarPlane;"
  echo "  float4x4 matView, matProj, matInvView, matInvProj; bool dirty; void update(); };"
  rng CUDACamera.cpp 245 266            # CUDACamera::update
  echo "}"
  rng "$Z" 23 25      # textures
  rng "$Z" 31 41      # EPSILON, CACHE_SIZE, block shape
  rng "$Z" 47 71      # intersectRectRect, intersectTriPoint
  rng "$Z" 77 225     # kernel_rasterizeMeshTree
  cat "$SHIM/raster_epilogue.hpp"
  echo "}"
} | build_tu ref_raster

L=kernels/CUDA_buildMeshTreeLBVH.cu
{
  cat "$SHIM/prelude.hpp"
  echo "namespace tu_lbvh {"
  rng "$L" 35 40      # BLOCK_SIZE, STACK_SIZE, MIN_LEAF_SIZE, MAX_LEAF_SIZE
  rng "$L" 46 48      # __device__ split_count, level_split_count
  cat "$SHIM/lbvh_mid.hpp"
  rng "$L" 54 59      # textures
  rng "$L" 85 109     # make_node, make_leaf
  rng "$L" 115 303    # kernel_calcMortonCodes, kernel_findSplits, kernel_calcBoundingBoxes
  rng "$L" 309 455    # createLeaf/createNode (median)/createNode (Morton)/buildMeshTree
  cat "$SHIM/lbvh_epilogue.hpp"
  echo "}"
} | build_tu ref_lbvh

B=kernels/CUDA_calcMeshBoxes.cu
{
  cat "$SHIM/prelude.hpp"
  echo "namespace tu_boxes {"
  rng "$B" 16 16      # BLOCK_SIZE
  rng "$B" 22 24      # textures
  rng "$B" 30 59      # kernel_initIndices, kernel_calcBoxes
  cat "$SHIM/boxes_epilogue.hpp"
  echo "}"
} | build_tu ref_boxes

R=kernels/CUDA_reorderMeshFaces.cu
{
  cat "$SHIM/prelude.hpp"
  echo "namespace tu_reorder {"
  rng "$R" 12 12      # BLOCK_SIZE
  rng "$R" 18 20      # textures
  rng "$R" 26 38      # kernel_reorderMesh
  cat "$SHIM/reorder_epilogue.hpp"
  echo "}"
} | build_tu ref_reorder

T=kernels/CUDA_raytraceMeshTree.cu
{
  cat "$SHIM/prelude.hpp"
  echo "namespace tu_trace {"
  rng "$T" 23 30      # textures
  rng "$T" 36 51      # EPSILON, block and stack sizes
  rng "$T" 57 219     # intersectTriRay, intersectBoxRay, kernel_raytraceMeshTree
  cat "$SHIM/trace_epilogue.hpp"
  echo "}"
} | build_tu ref_trace

P=kernels/CUDA_calcPrimaryRays.cu
{
  cat "$SHIM/prelude.hpp"
  echo "namespace tu_rays {"
  rng CUDACommon.h 108 108   # PI
  cat "$SHIM/camera_shim.hpp"
  echo "namespace renderkit {"
  rng CUDACamera.cpp 70 88   # CUDACamera::angleFromDir
  rng CUDACamera.cpp 126 133 # CUDACamera::lookAt(float, float, float)
  echo "}"
  rng "$P" 20 32             # kernel_calcPrimaryRays
  cat "$SHIM/rays_head.hpp"
  rng "$P" 43 55             # host camera basis of CUDA_calcPrimaryRays
  cat "$SHIM/rays_tail.hpp"
  echo "}"
} | build_tu ref_rays

I=kernels/CUDA_interpolateData.cu
{
  cat "$SHIM/prelude.hpp"
  echo "namespace tu_interp {"
  rng "$I" 23 31      # textures
  rng "$I" 37 39      # block sizes
  rng "$I" 45 138     # kernel_interpolateData
  cat "$SHIM/interp_epilogue.hpp"
  echo "}"
} | build_tu ref_interp

{
  cat "$SHIM/prelude.hpp"
  echo "#include <stdio.h>"
  echo "namespace tu_file {"
  cat "$SHIM/mesh_shim.hpp"
  echo "namespace renderkit {"
  rng CUDAMesh.cpp 134 400       # CUDAMesh::quickLoad, CUDAMesh::quickSave
  rng CUDAMeshTree.cpp 194 289   # CUDAMeshTree::quickSave
  echo "}"
  cat "$SHIM/file_epilogue.hpp"
  echo "}"
} | build_tu ref_file

g++ -shared -fPIC -o "$OUT/libref_cudart.so" "$OUT"/ref_lbvh.o "$OUT"/ref_boxes.o "$OUT"/ref_reorder.o "$OUT"/ref_trace.o "$OUT"/ref_rays.o "$OUT"/ref_interp.o "$OUT"/ref_file.o "$OUT"/ref_sah.o "$OUT"/ref_raster.o -lpthread
rm -f "$OUT"/*.o
echo "built $OUT/libref_cudart.so"
