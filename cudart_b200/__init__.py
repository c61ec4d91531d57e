"""cudart_b200 -- B200-native LBVH build and closest-hit traversal core.

A drop-in for the LBVH build / ray-tracing path of gatouillatpy/cudart
(CUDAMeshTree::buildMeshTreeLBVH, CUDARaytracer::calcPrimaryRays /
raytraceMeshTree and the sort free functions). The compute lives in
librt_core.so (hand-written sm_100a CUDA behind the C ABI of
include/rt_core.h); ``cudart_b200.core`` is the host side on torch tensors.
"""
from . import scenes  # noqa: F401
