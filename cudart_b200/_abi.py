"""ctypes declarations of the C ABI in include/rt_core.h and include/rt_propose.h
(librt_core.so).

Loading fails loudly when the shared library is missing: there is no CPU
fallback for any compute entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librt_core.so")

RT_OK = 0
ABI_VERSION = 11  # RT_ABI_VERSION of include/rt_core.h that the structs below mirror
STATUS_NAMES = {0: "RT_OK", 1: "RT_ERR_INVALID_ARGUMENT", 2: "RT_ERR_NO_DEVICE", 3: "RT_ERR_CUDA",
                4: "RT_ERR_SCRATCH_TOO_SMALL", 5: "RT_ERR_CAPACITY", 6: "RT_ERR_UNSUPPORTED"}
DEVERR_NODE_CAPACITY = 0x1
DEVERR_STACK_OVERFLOW = 0x2
DEVERR_MORTON_CAPACITY = 0x4
DEVERR_WAIT_TIMEOUT = 0x8
DEVERR_ACCEL_MISSING = 0x10
PROPOSE_ABI_VERSION = 2  # RT_PROPOSE_ABI_VERSION of include/rt_propose.h
TRACE_WHILE_WHILE = 0x1
TRACE_COOP = 0x2
TRACE_WIDE = 0x4
TRACE_CLUSTERS = 0x8
TRACE_PACKET = 0x10
TRACE_REFILL = 0x20
ACCEL_CLUSTERS = 0x2
MAX_RAYS = 0x7FFFFFFF  # RT_MAX_RAYS: the most rays one trace call takes

# every symbol include/rt_core.h declares
EXPORTS = (
    "rt_lbvh_scratch_bytes", "rt_lbvh_accel_bytes", "rt_lbvh_build", "rt_batch_sizes", "rt_batch_build", "rt_batch_trace", "rt_mesh_boxes", "rt_reorder_faces", "rt_sort_scratch_bytes",
    "rt_radix_sort_pairs", "rt_radix_sort_pairs_static", "rt_radix_sort_keys", "rt_camera_look_at", "rt_camera_basis", "rt_primary_rays", "rt_batch_primary_rays",
    "rt_trace_closest", "rt_ray_order_scratch_bytes", "rt_ray_order", "rt_batch_ray_order_scratch_bytes", "rt_batch_ray_order",
    "rt_image_tile_order", "rt_interpolate", "rt_bounce_rays", "rt_batch_bounce_rays", "rt_pack_hits_scratch_bytes", "rt_pack_hits", "rt_mesh_file_save", "rt_mesh_file_info", "rt_mesh_file_load", "rt_tree_file_save", "rt_tree_file_info",
    "rt_tree_file_load", "rt_status_string", "rt_version", "rt_abi_version", "rt_device_check", "rt_launch_count",
)
# every symbol include/rt_sah.h declares
SAH_EXPORTS = ("rt_sah_sizes", "rt_sah_build")
# every symbol include/rt_raster.h declares
RASTER_EXPORTS = ("rt_camera_view_dir", "rt_raster_matrix", "rt_raster_scratch_bytes", "rt_rasterize")
# every symbol include/rt_propose.h declares
PROPOSE_EXPORTS = (
    "rt_propose_abi_version", "rt_gemm_bf16", "rt_gemm_argmax_bf16", "rt_ray_features", "rt_softmax_xent", "rt_transpose_bf16",
    "rt_colsum_bf16", "rt_adam_step", "rt_subtree_slots", "rt_hit_labels", "rt_trace_closest_seeded", "rt_transpose_bf16_grouped",
    "rt_colsum_bf16_grouped", "rt_gather_batch", "rt_batch_subtree_slots", "rt_batch_hit_labels", "rt_batch_trace_seeded",
    "rt_group_select", "rt_mlp_propose", "rt_gemm_xent_bf16", "rt_tc_wait_selftest",
)

_P = C.c_void_p
_U32 = C.c_uint32


class RtError(RuntimeError):
    def __init__(self, fn, status):
        super().__init__(f"{fn} failed: {STATUS_NAMES.get(status, status)}")
        self.status = status


class BuildParams(C.Structure):
    _fields_ = [("tree_depth", _U32), ("tree_complete", _U32), ("min_leaf", _U32), ("max_leaf", _U32), ("morton_bits", _U32),
                ("accel_trees", _U32), ("cluster_leaf", _U32)]


class BuildInfo(C.Structure):
    _fields_ = [(k, _U32) for k in ("node_count", "leaf_count", "real_depth", "split_count", "overrun_visits",
                                     "nondet_reads", "past_end_reads", "error")]


class BuildDesc(C.Structure):
    _fields_ = [("vertices", _P), ("vertex_count", _U32), ("face_count", _U32), ("faces_in", _P), ("faces_out", _P),
                ("hitbox", _P), ("params", BuildParams), ("boxes", _P), ("indices", _P), ("codes", _P), ("nodes", _P),
                ("max_nodes", _U32), ("tris", _P), ("info", _P), ("scratch", _P), ("scratch_bytes", C.c_size_t),
                ("accel", _P), ("accel_bytes", C.c_size_t)]


class TraceDesc(C.Structure):
    _fields_ = [("nodes", _P), ("tris", _P), ("vertices", _P), ("faces", _P), ("indices", _P), ("orig", _P), ("dir", _P),
                ("tmax", _P), ("ray_count", _U32), ("id_mode", _U32), ("hit_id", _P), ("hit_t", _P), ("hit_uv", _P),
                ("ray_visits", _P), ("ray_tests", _P), ("error_word", _P), ("accel", _P), ("face_count_hint", _U32),
                ("image_width", _U32), ("work_counter", _P), ("persistent_blocks_per_sm", _U32), ("schedule", _U32),
                ("ray_order", _P), ("treelet_depth", _U32), ("lane_threshold", _U32)]


class InterpDesc(C.Structure):
    _fields_ = [("hit_id", _P), ("hit_uv", _P), ("count", _U32), ("faces", _P), ("vertices", _P), ("normals", _P),
                ("colors", _P), ("texcoords", _P), ("out_points", _P), ("out_normals", _P), ("out_colors", _P),
                ("out_texcoords", _P), ("out_materials", _P)]


class MeshFile(C.Structure):
    _fields_ = [("hitbox", C.c_float * 8), ("has_hitbox", C.c_int32), ("vertex_count", _U32), ("normal_count", _U32),
                ("color_count", _U32), ("texcoord_count", _U32), ("face_count", _U32), ("vertices", _P), ("normals", _P),
                ("colors", _P), ("texcoords", _P), ("faces", _P)]


class TreeFile(C.Structure):
    _fields_ = [("node_count", _U32), ("index_count", _U32), ("box_count", _U32), ("nodes", _P), ("indices", _P), ("boxes", _P)]


class BatchBuildDesc(C.Structure):
    _fields_ = [("mesh_count", _U32), ("face_count", _U32), ("vertex_count", _U32), ("face_offsets", _P), ("vertex_offsets", _P),
                ("vertices", _P), ("faces_in", _P), ("faces_out", _P), ("params", BuildParams), ("boxes", _P), ("indices", _P),
                ("codes", _P), ("nodes", _P), ("tris", _P), ("accel", _P), ("accel_bytes", C.c_size_t), ("info", _P),
                ("scratch", _P), ("scratch_bytes", C.c_size_t)]


class BatchTraceDesc(C.Structure):
    _fields_ = [("mesh_count", _U32), ("face_offsets", _P), ("ray_offsets", _P), ("accel", _P), ("tris", _P), ("indices", _P),
                ("face_count", _U32), ("orig", _P), ("dir", _P), ("tmax", _P), ("ray_count", _U32), ("id_mode", _U32),
                ("hit_id", _P), ("hit_t", _P), ("hit_uv", _P), ("ray_visits", _P), ("ray_tests", _P), ("error_word", _P),
                ("schedule", _U32), ("work_counter", _P), ("persistent_blocks_per_sm", _U32), ("ray_order", _P),
                ("lane_threshold", _U32), ("bounce_seed", C.c_uint64), ("bounce_orig", _P), ("bounce_dir", _P), ("bounce_tmax", _P)]


class SahDesc(C.Structure):
    _fields_ = [("vertices", _P), ("vertex_count", _U32), ("face_count", _U32), ("faces_in", _P), ("faces_out", _P), ("hitbox", _P),
                ("lbvh_depth", _U32), ("boxes", _P), ("indices", _P), ("nodes", _P), ("max_nodes", _U32), ("tris", _P), ("accel", _P),
                ("accel_bytes", C.c_size_t), ("info", _P), ("scratch", _P), ("scratch_bytes", C.c_size_t)]


class RasterDesc(C.Structure):
    _fields_ = [("vertices", _P), ("vertex_count", _U32), ("faces", _P), ("face_count", _U32), ("matrix", C.c_float * 16),
                ("width", _U32), ("height", _U32), ("id_mode", _U32), ("face_id", _P), ("uv", _P), ("depth", _P), ("pair_capacity", _U32),
                ("scratch", _P), ("scratch_bytes", C.c_size_t), ("error_word", _P)]


class GemmDesc(C.Structure):
    _fields_ = [("a", _P), ("lda", _U32), ("b", _P), ("ldb", _U32), ("m", _U32), ("n", _U32), ("k", _U32), ("alpha", C.c_float),
                ("bias", _P), ("relu", _U32), ("mask", _P), ("ldmask", _U32), ("c_f32", _P), ("ldc_f32", _U32), ("c_bf16", _P),
                ("ldc_bf16", _U32), ("ct_bf16", _P), ("ldct", _U32), ("error_word", _P), ("groups", _U32)]


class GemmArgmaxDesc(C.Structure):
    _fields_ = [("a", _P), ("lda", _U32), ("b", _P), ("ldb", _U32), ("m", _U32), ("n", _U32), ("k", _U32), ("bias", _P),
                ("min_margin", C.c_float), ("out_index", _P), ("out_value", _P), ("out_margin", _P), ("error_word", _P),
                ("groups", _U32)]


class FeatureDesc(C.Structure):
    _fields_ = [("orig", _P), ("dir", _P), ("count", _U32), ("box_lo", C.c_float * 3), ("box_hi", C.c_float * 3), ("out", _P),
                ("ld_out", _U32), ("out_t", _P), ("ld_out_t", _U32), ("group_rows", _U32)]


class AdamDesc(C.Structure):
    _fields_ = [("param", _P), ("grad", _P), ("m", _P), ("v", _P), ("rows", _U32), ("cols", _U32), ("lr", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("step", _U32), ("out_bf16", _P), ("ld_bf16", _U32),
                ("out_bf16_t", _P), ("ld_bf16_t", _U32), ("groups", _U32)]


class SlotDesc(C.Structure):
    _fields_ = [("nodes", _P), ("accel", _P), ("face_count", _U32), ("depth", _U32), ("slot_ref", _P), ("slot_box", _P),
                ("pos_label", _P), ("slot_first", _P), ("slot_count", _P)]


class SeedDesc(C.Structure):
    _fields_ = [("proposal", _P), ("slot_ref", _P), ("slot_box", _P), ("slot_count", _U32), ("in_proposal", _P)]


class BatchGatherDesc(C.Structure):
    _fields_ = [("orig", _P), ("dir", _P), ("labels", _P), ("groups", _U32), ("group_stride", _U32), ("offset", _U32),
                ("batch", _U32), ("out_orig", _P), ("out_dir", _P), ("out_labels", _P), ("index", _P), ("index_count", _P),
                ("hop", _U32)]


class GemmXentDesc(C.Structure):
    _fields_ = [("a", _P), ("lda", _U32), ("b", _P), ("ldb", _U32), ("m", _U32), ("n", _U32), ("k", _U32), ("bias", _P), ("labels", _P),
                ("scale", C.c_float), ("g", _P), ("ldg", _U32), ("gt", _P), ("ldgt", _U32), ("loss_sum", _P), ("error_word", _P),
                ("groups", _U32)]


class MlpProposeDesc(C.Structure):
    _fields_ = [("orig", _P), ("dir", _P), ("count", _U32), ("box_lo", C.c_float * 3), ("box_hi", C.c_float * 3), ("w1", _P), ("w2", _P),
                ("w3", _P), ("w4", _P), ("b1", _P), ("b2", _P), ("b3", _P), ("b4", _P), ("n", _U32), ("groups", _U32),
                ("group_rows", _U32), ("min_margin", C.c_float), ("out_index", _P), ("out_value", _P), ("out_margin", _P),
                ("error_word", _P), ("tmax", _P)]


class BatchSlotDesc(C.Structure):
    _fields_ = [("mesh_count", _U32), ("face_offsets", _P), ("nodes", _P), ("accel", _P), ("face_count", _U32), ("depth", _U32),
                ("slot_ref", _P), ("slot_box", _P), ("pos_label", _P), ("slot_first", _P), ("slot_count", _P)]


class Camera(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("angle", C.c_float * 3), ("fov", C.c_float), ("ratio", C.c_float)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C cudart_b200/csrc` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        L.rt_lbvh_scratch_bytes.argtypes = [_U32, C.POINTER(BuildParams), C.POINTER(C.c_size_t), C.POINTER(_U32)]
        L.rt_lbvh_build.argtypes = [C.POINTER(BuildDesc), _P]
        L.rt_lbvh_accel_bytes.argtypes = [_U32, C.POINTER(C.c_size_t)]
        L.rt_batch_sizes.argtypes = [_U32, _U32, C.POINTER(BuildParams), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        L.rt_batch_build.argtypes = [C.POINTER(BatchBuildDesc), _P]
        L.rt_batch_trace.argtypes = [C.POINTER(BatchTraceDesc), _P]
        L.rt_mesh_boxes.argtypes = [_P, _P, _U32, _P, _P, _P]
        L.rt_reorder_faces.argtypes = [_P, _P, _U32, _P, _P]
        L.rt_sort_scratch_bytes.argtypes = [_U32, C.POINTER(C.c_size_t)]
        L.rt_radix_sort_pairs.argtypes = [_P, _P, _U32, _U32, C.c_int, _P, C.c_size_t, _P]
        L.rt_radix_sort_pairs_static.argtypes = [_P, _P, _U32, _U32, C.c_int, _P]
        L.rt_radix_sort_keys.argtypes = [_P, _U32, _U32, _P, C.c_size_t, _P]
        L.rt_camera_look_at.argtypes = [C.POINTER(Camera), C.POINTER(C.c_float)]
        L.rt_camera_basis.argtypes = [C.POINTER(Camera), _U32, _U32, C.POINTER(C.c_float)]
        L.rt_primary_rays.argtypes = [C.POINTER(Camera), _U32, _U32, _P, _P, _P]
        L.rt_batch_primary_rays.argtypes = [_P, _U32, _U32, _U32, _P, _P, _P]
        L.rt_trace_closest.argtypes = [C.POINTER(TraceDesc), _P]
        L.rt_interpolate.argtypes = [C.POINTER(InterpDesc), _P]
        L.rt_ray_order_scratch_bytes.argtypes = [_U32, C.POINTER(C.c_size_t)]
        L.rt_ray_order.argtypes = [_P, _P, _P, _U32, C.POINTER(C.c_float), _P, _P, C.c_size_t, _P]
        L.rt_batch_ray_order_scratch_bytes.argtypes = [_U32, C.POINTER(C.c_size_t)]
        L.rt_batch_ray_order.argtypes = [_P, _P, _P, _U32, _P, _U32, C.POINTER(C.c_float), _U32, _P, _P, C.c_size_t, _P]
        L.rt_image_tile_order.argtypes = [_U32, _U32, _U32, _P, _P]
        L.rt_bounce_rays.argtypes = [_P, _P, _P, _P, _P, _U32, C.c_uint64, _P, _P, _P, _P]
        L.rt_batch_bounce_rays.argtypes = [_P, _P, _P, _U32, _P, _P, _P, _P, _U32, C.c_uint64, _P, _P, _P, _P, _P, _P]
        L.rt_pack_hits_scratch_bytes.argtypes = [_U32, C.POINTER(C.c_size_t)]
        L.rt_pack_hits.argtypes = [_P, _P, _P, _U32, _P, _P, _P, C.c_size_t, _P]
        for fn, st in (("mesh", MeshFile), ("tree", TreeFile)):
            getattr(L, f"rt_{fn}_file_save").argtypes = [C.c_char_p, C.c_int, C.POINTER(st)]
            getattr(L, f"rt_{fn}_file_info").argtypes = [C.c_char_p, C.POINTER(st)]
            getattr(L, f"rt_{fn}_file_load").argtypes = [C.c_char_p, C.POINTER(st)]
        L.rt_sah_sizes.argtypes = [_U32, _U32, C.POINTER(C.c_size_t), C.POINTER(_U32)]
        L.rt_sah_build.argtypes = [C.POINTER(SahDesc), _P]
        for name in SAH_EXPORTS:
            getattr(L, name).restype = C.c_int
        L.rt_raster_matrix.argtypes = [C.POINTER(Camera), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.rt_camera_view_dir.argtypes = [C.POINTER(Camera), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.rt_raster_scratch_bytes.argtypes = [_U32, _U32, _U32, _U32, C.POINTER(C.c_size_t)]
        L.rt_rasterize.argtypes = [C.POINTER(RasterDesc), _P]
        for name in RASTER_EXPORTS:
            getattr(L, name).restype = C.c_int
        L.rt_gemm_bf16.argtypes = [C.POINTER(GemmDesc), _P]
        L.rt_gemm_argmax_bf16.argtypes = [C.POINTER(GemmArgmaxDesc), _P]
        L.rt_ray_features.argtypes = [C.POINTER(FeatureDesc), _P]
        L.rt_softmax_xent.argtypes = [_P, _U32, _U32, _P, C.c_float, _P, _P, _P]
        L.rt_transpose_bf16.argtypes = [_P, _U32, _U32, _U32, _P, _U32, _P]
        L.rt_colsum_bf16.argtypes = [_P, _U32, _U32, _U32, _P, _P]
        L.rt_adam_step.argtypes = [C.POINTER(AdamDesc), _P]
        L.rt_subtree_slots.argtypes = [C.POINTER(SlotDesc), _P]
        L.rt_hit_labels.argtypes = [_P, _U32, _P, _P, _P]
        L.rt_trace_closest_seeded.argtypes = [C.POINTER(TraceDesc), C.POINTER(SeedDesc), _P]
        L.rt_transpose_bf16_grouped.argtypes = [_P, _U32, _U32, _U32, _U32, _P, _U32, _P]
        L.rt_colsum_bf16_grouped.argtypes = [_P, _U32, _U32, _U32, _U32, _P, _P]
        L.rt_gather_batch.argtypes = [C.POINTER(BatchGatherDesc), _P]
        L.rt_group_select.argtypes = [_P, _U32, _U32, _P, _P, _P]
        L.rt_mlp_propose.argtypes = [C.POINTER(MlpProposeDesc), _P]
        L.rt_gemm_xent_bf16.argtypes = [C.POINTER(GemmXentDesc), _P]
        L.rt_tc_wait_selftest.argtypes = [_U32, _P, _P, _P]
        L.rt_batch_subtree_slots.argtypes = [C.POINTER(BatchSlotDesc), _P]
        L.rt_batch_hit_labels.argtypes = [_P, _U32, _U32, _P, _P, _P, _P, _P]
        L.rt_batch_trace_seeded.argtypes = [C.POINTER(BatchTraceDesc), C.POINTER(SeedDesc), _P]
        for name in PROPOSE_EXPORTS[1:]:
            getattr(L, name).restype = C.c_int
        L.rt_propose_abi_version.restype = _U32
        L.rt_status_string.restype = C.c_char_p
        L.rt_status_string.argtypes = [C.c_int]
        L.rt_version.restype = _U32
        L.rt_device_check.restype = C.c_int
        L.rt_launch_count.restype = C.c_uint64
        L.rt_abi_version.restype = _U32
        for name in EXPORTS:
            if name not in ("rt_status_string", "rt_version", "rt_abi_version", "rt_device_check", "rt_launch_count"):
                getattr(L, name).restype = C.c_int
        if L.rt_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has struct layout version {L.rt_abi_version()}, these bindings expect {ABI_VERSION}: rebuild")
        if L.rt_propose_abi_version() != PROPOSE_ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has proposal struct version {L.rt_propose_abi_version()}, expected {PROPOSE_ABI_VERSION}: rebuild")
        _lib = L
    return _lib


def check(fn: str, status: int):
    if status != RT_OK:
        raise RtError(fn, status)
