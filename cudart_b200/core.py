"""Python host side over the C ABI, on torch CUDA tensors.

Mirrors the reference's host interface for the path: ``build_lbvh`` is
CUDAMeshTree::buildMeshTreeLBVH (CUDAMeshTree.cpp:88-91), ``primary_rays`` is
CUDARaytracer::calcPrimaryRays (CUDARaytracer.cpp:125-128), ``trace`` is
CUDARaytracer::raytraceMeshTree (CUDARaytracer.cpp:130-135), ``sort_pairs`` /
``sort_keys`` are CUDA_radixSortGeneral / CUDA_radixSort. torch only supplies
device memory and streams; every computation runs in librt_core.so. Calls are
asynchronous on the current torch stream; nothing here synchronizes except
the explicit ``*_host`` helpers.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _abi

HUGE = 3.402823466e38


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def _need_cuda(t, name, dtype=None, cols=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if dtype is not None and t.dtype not in dtype:
        raise ValueError(f"{name} has dtype {t.dtype}, expected one of {dtype}")
    if cols is not None and (t.dim() != 2 or t.shape[1] != cols):
        raise ValueError(f"{name} must have shape (*, {cols})")


_I32 = (torch.int32, torch.uint32)
_F32 = (torch.float32,)


class _Scratch:
    """Grow-only scratch buffer per device (the C ABI allocates nothing)."""

    def __init__(self):
        self.buf = {}

    def get(self, nbytes: int, device) -> torch.Tensor:
        key = torch.device(device).index or 0
        b = self.buf.get(key)
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
            self.buf[key] = b
        return b


_SCRATCH = _Scratch()
_ORDER_SCRATCH = _Scratch()
_COUNTERS = {}

# Traversal schedule of the blob path (never changes the results). The
# autotuner in cudart_b200/tune.py can replace it per device.
DEFAULT_SCHEDULE = {"image_width": 0, "persistent": False, "blocks_per_sm": 8, "while_while": False}


def _work_counter(device, stream=None) -> torch.Tensor:
    s = torch.cuda.current_stream() if stream is None else stream
    key = (torch.device(device).index or 0, s.cuda_stream)  # one counter per stream: concurrent traces do not share it
    c = _COUNTERS.get(key)
    if c is None:
        c = torch.zeros(1, dtype=torch.int32, device=device)
        _COUNTERS[key] = c
    return c


def device_check() -> bool:
    return _abi.lib().rt_device_check() == _abi.RT_OK


@dataclass
class Tree:
    """Device state of a built tree (CUDAMeshTree: nodes, boxes, indices) plus
    the reordered faces and the pre-gathered triangle stream."""

    nodes: torch.Tensor  # int32 (max_nodes, 8) bvnode words
    boxes: torch.Tensor  # float32 (N, 8) aabox per original face
    indices: torch.Tensor  # int32 (N,) position -> original face id
    codes: torch.Tensor  # int32 (N,) sorted Morton codes (uint32 bits)
    faces: torch.Tensor  # int32 (N, 4) faces in position order
    tris: torch.Tensor  # float32 (N, 12) {v0, e1, e2}
    info: torch.Tensor  # int32 (8,) rt_build_info, on the device
    accel: torch.Tensor | None = None  # uint8 traversal blob (two-child records, leaf table, group boxes)
    clusters: bool = False  # the blob also holds the cluster tree (schedules with "clusters": True walk it)

    def info_host(self) -> dict:
        vals = self.info.cpu().tolist()
        keys = [f[0] for f in _abi.BuildInfo._fields_]
        return {k: v & 0xFFFFFFFF for k, v in zip(keys, vals)}

    @property
    def node_count(self) -> int:
        return int(self.info[0].item())

    def nodes_host(self):
        return self.nodes[: self.node_count].cpu()


def lbvh_scratch_bytes(face_count: int, tree_depth=12, tree_complete=True, morton_bits=32, min_leaf=0, max_leaf=0, clusters=False):
    params = _abi.BuildParams(tree_depth, int(tree_complete), min_leaf, max_leaf, morton_bits, _abi.ACCEL_CLUSTERS if clusters else 0)
    nb = C.c_size_t(0)
    mx = C.c_uint32(0)
    _abi.check("rt_lbvh_scratch_bytes", _abi.lib().rt_lbvh_scratch_bytes(face_count, C.byref(params), C.byref(nb), C.byref(mx)))
    return nb.value, mx.value


def accel_bytes(face_count: int) -> int:
    nb = C.c_size_t(0)
    _abi.check("rt_lbvh_accel_bytes", _abi.lib().rt_lbvh_accel_bytes(face_count, C.byref(nb)))
    return nb.value


def build_lbvh(vertices: torch.Tensor, faces: torch.Tensor, hitbox=None, tree_depth: int = 12, tree_complete: bool = True,
               morton_bits: int = 32, out: Tree | None = None, accel: bool = True, min_leaf: int = 0, max_leaf: int = 0,
               stream=None, clusters: bool = False, cluster_leaf: int = 0) -> Tree:
    """LBVH build of a mesh given as float4 vertices (V, 4) and uint4 faces (N, 4).
    hitbox: host sequence of 8 floats (min xyzw, max xyzw) or None for the
    vertices' min/max. clusters: also write the cluster tree into the blob
    (RT_ACCEL_CLUSTERS, leaves of at most cluster_leaf positions, 0 = 3), for
    schedules with "clusters": True."""
    _need_cuda(vertices, "vertices", _F32, 4)
    _need_cuda(faces, "faces", _I32, 4)
    n = faces.shape[0]
    dev = vertices.device
    nbytes, max_nodes = lbvh_scratch_bytes(n, tree_depth, tree_complete, morton_bits, min_leaf, max_leaf, clusters=clusters)
    if out is None:
        out = Tree(
            nodes=torch.empty((max_nodes, 8), dtype=torch.int32, device=dev),
            boxes=torch.empty((n, 8), dtype=torch.float32, device=dev),
            indices=torch.empty(n, dtype=torch.int32, device=dev),
            codes=torch.empty(n, dtype=torch.int32, device=dev),
            faces=torch.empty((n, 4), dtype=torch.int32, device=dev),
            tris=torch.empty((n, 12), dtype=torch.float32, device=dev),
            info=torch.zeros(8, dtype=torch.int32, device=dev),
            accel=torch.empty(accel_bytes(n), dtype=torch.uint8, device=dev) if (accel and tree_complete) else None,
        )
    scratch = _SCRATCH.get(nbytes, dev)
    hb = None
    if hitbox is not None:
        hb = (C.c_float * 8)(*[float(x) for x in hitbox])
    d = _abi.BuildDesc()
    d.vertices = vertices.data_ptr()
    d.vertex_count = vertices.shape[0]
    d.face_count = n
    d.faces_in = faces.data_ptr()
    d.faces_out = out.faces.data_ptr()
    d.hitbox = C.cast(hb, C.c_void_p).value if hb is not None else None
    d.params = _abi.BuildParams(tree_depth, int(tree_complete), min_leaf, max_leaf, morton_bits,
                                _abi.ACCEL_CLUSTERS if clusters else 0, cluster_leaf)
    d.boxes = out.boxes.data_ptr()
    d.indices = out.indices.data_ptr()
    d.codes = out.codes.data_ptr()
    d.nodes = out.nodes.data_ptr()
    d.max_nodes = out.nodes.shape[0]
    d.tris = out.tris.data_ptr()
    d.info = out.info.data_ptr()
    d.scratch = scratch.data_ptr()
    d.scratch_bytes = scratch.numel()
    if out.accel is not None:
        d.accel = out.accel.data_ptr()
        d.accel_bytes = out.accel.numel()
    _abi.check("rt_lbvh_build", _abi.lib().rt_lbvh_build(C.byref(d), _stream(stream)))
    out.clusters = bool(clusters and out.accel is not None)
    if hitbox is not None:  # the scene box for ray ordering, known on the host: no device read later
        out._box = [float(hitbox[i]) for i in (0, 1, 2, 4, 5, 6)]
    return out


def sah_sizes(face_count: int, lbvh_depth: int = 0):
    nb = C.c_size_t(0)
    mx = C.c_uint32(0)
    _abi.check("rt_sah_sizes", _abi.lib().rt_sah_sizes(face_count, lbvh_depth, C.byref(nb), C.byref(mx)))
    return nb.value, mx.value


def build_sah(vertices: torch.Tensor, faces: torch.Tensor, hitbox=None, lbvh_depth: int = 0, accel: bool = True,
              out: Tree | None = None, stream=None) -> Tree:
    """SAH build (CUDAMeshTree::buildMeshTreeSAH) or, with lbvh_depth > 0, the
    Hybrid build (buildMeshTreeHybrid(lbvh_depth)). Same Tree layout as
    build_lbvh; `codes` is left unwritten."""
    _need_cuda(vertices, "vertices", _F32, 4)
    _need_cuda(faces, "faces", _I32, 4)
    n = faces.shape[0]
    dev = vertices.device
    nbytes, max_nodes = sah_sizes(n, lbvh_depth)
    if out is None:
        out = Tree(
            nodes=torch.empty((max_nodes, 8), dtype=torch.int32, device=dev),
            boxes=torch.empty((n, 8), dtype=torch.float32, device=dev),
            indices=torch.empty(n, dtype=torch.int32, device=dev),
            codes=torch.zeros(n, dtype=torch.int32, device=dev),
            faces=torch.empty((n, 4), dtype=torch.int32, device=dev),
            tris=torch.empty((n, 12), dtype=torch.float32, device=dev),
            info=torch.zeros(8, dtype=torch.int32, device=dev),
            accel=torch.empty(accel_bytes(n), dtype=torch.uint8, device=dev) if accel else None,
        )
    scratch = _SCRATCH.get(nbytes, dev)
    hb = None
    if hitbox is not None:
        hb = (C.c_float * 8)(*[float(x) for x in hitbox])
    d = _abi.SahDesc()
    d.vertices, d.vertex_count, d.face_count = vertices.data_ptr(), vertices.shape[0], n
    d.faces_in, d.faces_out = faces.data_ptr(), out.faces.data_ptr()
    d.hitbox = C.cast(hb, C.c_void_p).value if hb is not None else None
    d.lbvh_depth = lbvh_depth
    d.boxes, d.indices, d.nodes, d.max_nodes = out.boxes.data_ptr(), out.indices.data_ptr(), out.nodes.data_ptr(), out.nodes.shape[0]
    d.tris = out.tris.data_ptr()
    if out.accel is not None:
        d.accel, d.accel_bytes = out.accel.data_ptr(), out.accel.numel()
    d.info = out.info.data_ptr()
    d.scratch, d.scratch_bytes = scratch.data_ptr(), scratch.numel()
    _abi.check("rt_sah_build", _abi.lib().rt_sah_build(C.byref(d), _stream(stream)))
    return out


def raster_matrix(cam: _abi.Camera, target) -> list:
    """transpose(view * proj) of CUDACamera::update for a camera that looked at `target`."""
    t = (C.c_float * 3)(*[float(x) for x in target])
    d = (C.c_float * 3)()
    _abi.check("rt_camera_view_dir", _abi.lib().rt_camera_view_dir(C.byref(cam), t, d))
    m = (C.c_float * 16)()
    _abi.check("rt_raster_matrix", _abi.lib().rt_raster_matrix(C.byref(cam), d, m))
    return list(m)


def rasterize(vertices: torch.Tensor, faces: torch.Tensor, matrix, width: int, height: int, id_mode: int = 0, out: dict | None = None,
              pair_capacity: int = 0, stream=None) -> dict:
    """CUDARaytracer::rasterizeMeshTree into the surfaces of `out` (created cleared as
    CUDABuffer::clearOutputSurfaces leaves them: id 0, uv 0, depth +HUGE)."""
    _need_cuda(vertices, "vertices", _F32, 4)
    _need_cuda(faces, "faces", _I32, 4)
    P = width * height
    dev = vertices.device
    if out is None:
        out = dict(id=torch.zeros(P, dtype=torch.int32, device=dev), uv=torch.zeros((P, 2), dtype=torch.float32, device=dev),
                   depth=torch.full((P,), HUGE, dtype=torch.float32, device=dev), err=torch.zeros(1, dtype=torch.int32, device=dev))
    nb = C.c_size_t(0)
    _abi.check("rt_raster_scratch_bytes", _abi.lib().rt_raster_scratch_bytes(faces.shape[0], width, height, pair_capacity, C.byref(nb)))
    scratch = _SCRATCH.get(nb.value, dev)
    d = _abi.RasterDesc()
    d.vertices, d.vertex_count, d.faces, d.face_count = vertices.data_ptr(), vertices.shape[0], faces.data_ptr(), faces.shape[0]
    for i in range(16):
        d.matrix[i] = float(matrix[i])
    d.width, d.height, d.id_mode, d.pair_capacity = width, height, id_mode, pair_capacity
    d.face_id, d.uv, d.depth = out["id"].data_ptr(), out["uv"].data_ptr(), out["depth"].data_ptr()
    d.scratch, d.scratch_bytes = scratch.data_ptr(), scratch.numel()
    if "err" in out:
        d.error_word = out["err"].data_ptr()
    _abi.check("rt_rasterize", _abi.lib().rt_rasterize(C.byref(d), _stream(stream)))
    return out


def trace(tree: Tree, orig: torch.Tensor, dir: torch.Tensor, tmax: torch.Tensor | None = None, id_mode: int = 0,
          counters: bool = False, use_tris: bool = True, vertices: torch.Tensor | None = None, out: dict | None = None,
          ray_count: int | None = None, use_accel: bool = True, schedule: dict | None = None, stream=None) -> dict:
    """Closest hit per ray. Returns dict(id=int32, t=float32, uv=float32 (R, 2), err=int32 (1,))."""
    d, out = trace_desc(tree, orig, dir, tmax, id_mode, counters, use_tris, vertices, out, ray_count, use_accel, schedule, stream)
    _abi.check("rt_trace_closest", _abi.lib().rt_trace_closest(C.byref(d), _stream(stream)))
    return out


def trace_desc(tree: Tree, orig, dir, tmax=None, id_mode: int = 0, counters: bool = False, use_tris: bool = True, vertices=None,
               out: dict | None = None, ray_count: int | None = None, use_accel: bool = True, schedule: dict | None = None,
               stream=None):
    """The rt_trace_desc of a trace call and its output tensors (shared by trace and the seeded trace)."""
    _need_cuda(orig, "orig", _F32, 4)
    _need_cuda(dir, "dir", _F32, 4)
    R = orig.shape[0] if ray_count is None else ray_count
    dev = orig.device
    if out is None:
        out = dict(id=torch.empty(R, dtype=torch.int32, device=dev), t=torch.empty(R, dtype=torch.float32, device=dev),
                   uv=torch.empty((R, 2), dtype=torch.float32, device=dev), err=torch.zeros(1, dtype=torch.int32, device=dev))
        if counters:
            out["visits"] = torch.empty(R, dtype=torch.int32, device=dev)
            out["tests"] = torch.empty(R, dtype=torch.int32, device=dev)
    d = _abi.TraceDesc()
    d.nodes = tree.nodes.data_ptr()
    if use_tris:
        d.tris = tree.tris.data_ptr()
    else:
        if vertices is None:
            raise ValueError("use_tris=False needs the mesh vertices")
        d.vertices = vertices.data_ptr()
        d.faces = tree.faces.data_ptr()
    d.indices = tree.indices.data_ptr()
    d.orig = orig.data_ptr()
    d.dir = dir.data_ptr()
    d.tmax = tmax.data_ptr() if tmax is not None else None
    d.ray_count = R
    d.id_mode = id_mode
    d.hit_id = out["id"].data_ptr()
    d.hit_t = out["t"].data_ptr()
    d.hit_uv = out["uv"].data_ptr()
    if "visits" in out:
        d.ray_visits = out["visits"].data_ptr()
        d.ray_tests = out["tests"].data_ptr()
    d.error_word = out["err"].data_ptr()
    if use_accel and use_tris and tree.accel is not None:
        d.accel = tree.accel.data_ptr()
        d.face_count_hint = tree.faces.shape[0]
        sch = DEFAULT_SCHEDULE if schedule is None else schedule
        d.image_width = int(sch.get("image_width", 0))
        if sch.get("persistent", False):
            d.work_counter = _work_counter(dev, stream).data_ptr()
            d.persistent_blocks_per_sm = int(sch.get("blocks_per_sm", 8))
            d.treelet_depth = int(sch.get("treelet", 0))  # top levels staged in shared memory (4-wide walks)
            d.lane_threshold = int(sch.get("lane_threshold", 0))  # packet walks: fall back to per-lane walks
        d.schedule = ((_abi.TRACE_WHILE_WHILE if sch.get("while_while", False) else 0) | (_abi.TRACE_COOP if sch.get("coop", False) else 0)
                      | (_abi.TRACE_WIDE if sch.get("wide", False) else 0) | (_abi.TRACE_CLUSTERS if sch.get("clusters", False) else 0)
                      | (_abi.TRACE_PACKET if sch.get("packet", False) else 0) | (_abi.TRACE_REFILL if sch.get("refill", False) else 0))
        if sch.get("sorted", False):
            order = ray_order(orig, dir, tmax, tree_box(tree), ray_count=R, stream=stream)
            out["_order"] = order  # keep it alive until the trace has run
            d.ray_order = order.data_ptr()
    return d, out


def tree_box(tree: Tree):
    """Scene box for ray ordering (host floats): the hitbox given to build_lbvh,
    else read once from the root node and cached on the tree. A Tree rebuilt
    in place from other geometry without a hitbox keeps the first box; the
    order only affects speed, never the hits."""
    box = getattr(tree, "_box", None)
    if box is None:
        root = tree.nodes[0].cpu().view(torch.float32).tolist()
        box = [root[2], root[3], root[4], root[5], root[6], root[7]]
        if not all(abs(x) < 1e30 for x in box):  # inverted (flat-z quirk) or empty: fall back to the face boxes
            b = tree.boxes.view(-1, 8)
            box = b[:, :3].min(0).values.tolist() + b[:, 4:7].max(0).values.tolist()
        tree._box = box
    return box


def ray_order(orig, dir, tmax, box, ray_count: int | None = None, stream=None) -> torch.Tensor:
    """Permutation of the rays sorted by direction octant and origin Morton code (rt_ray_order)."""
    R = orig.shape[0] if ray_count is None else ray_count
    nb = C.c_size_t(0)
    _abi.lib().rt_ray_order_scratch_bytes(R, C.byref(nb))
    scratch = _ORDER_SCRATCH.get(nb.value, orig.device)
    order = torch.empty(R, dtype=torch.int32, device=orig.device)
    b = (C.c_float * 6)(*[float(x) for x in box])
    _abi.check("rt_ray_order", _abi.lib().rt_ray_order(_p(orig), _p(dir), _p(tmax), R, b, _p(order), _p(scratch), scratch.numel(),
                                                       _stream(stream)))
    return order


def make_camera(center, target=None, angle=None, fov=3.14159265359 * 0.5, ratio=4.0 / 3.0) -> _abi.Camera:
    """CUDACamera state; with a target, the angles come from CUDACamera::lookAt."""
    cam = _abi.Camera()
    cam.center[:] = [float(c) for c in center]
    # CUDACamera's constructor angles (CUDACamera.cpp:41-43)
    cam.angle[:] = [float(a) for a in (angle if angle is not None else (3.14159265359 * 0.5, 0.0, 0.0))]
    cam.fov = fov
    cam.ratio = ratio
    if target is not None:
        tgt = (C.c_float * 3)(*[float(t) for t in target])
        _abi.check("rt_camera_look_at", _abi.lib().rt_camera_look_at(C.byref(cam), tgt))
    return cam


def camera_basis(cam: _abi.Camera, width: int, height: int):
    b = (C.c_float * 16)()
    _abi.check("rt_camera_basis", _abi.lib().rt_camera_basis(C.byref(cam), width, height, b))
    return list(b)


def primary_rays(cam: _abi.Camera, width: int, height: int, out=None, device="cuda", stream=None):
    R = width * height
    if out is None:
        out = (torch.empty((R, 4), dtype=torch.float32, device=device), torch.empty((R, 4), dtype=torch.float32, device=device))
    _abi.check("rt_primary_rays", _abi.lib().rt_primary_rays(C.byref(cam), width, height, _p(out[0]), _p(out[1]), _stream(stream)))
    return out


def camera_bases(cams, width: int, height: int, device="cuda") -> torch.Tensor:
    """The rt_camera_basis of every camera, as the DEVICE float[16 * count] that batch_primary_rays reads."""
    return torch.tensor([camera_basis(c, width, height) for c in cams], dtype=torch.float32, device=device)


def batch_primary_rays(bases: torch.Tensor, width: int, height: int, out=None, stream=None):
    """rt_batch_primary_rays: every camera's rays in one launch (camera c's at rows c * width * height)."""
    count = bases.shape[0]
    R = count * width * height
    if out is None:
        out = (torch.empty((R, 4), dtype=torch.float32, device=bases.device), torch.empty((R, 4), dtype=torch.float32, device=bases.device))
    _abi.check("rt_batch_primary_rays", _abi.lib().rt_batch_primary_rays(_p(bases), count, width, height, _p(out[0]), _p(out[1]),
                                                                         _stream(stream)))
    return out


def bounce_rays(tris, orig, dir, hit_pos, hit_t, seed: int, out=None, ray_count: int | None = None, stream=None):
    R = orig.shape[0] if ray_count is None else ray_count
    dev = orig.device
    if out is None:
        out = (torch.empty((R, 4), dtype=torch.float32, device=dev), torch.empty((R, 4), dtype=torch.float32, device=dev),
               torch.empty(R, dtype=torch.float32, device=dev))
    _abi.check("rt_bounce_rays", _abi.lib().rt_bounce_rays(_p(tris), _p(orig), _p(dir), _p(hit_pos), _p(hit_t), R, C.c_uint64(seed),
                                                           _p(out[0]), _p(out[1]), _p(out[2]), _stream(stream)))
    return out


def batch_bounce_rays(tree, ray_offsets, orig, dir, hit_pos, hit_t, seed: int, out=None, order: bool = False, stream=None):
    """bounce_rays for the rays of a batched build: hit_pos are positions inside each ray's own mesh
    (batch_trace's ids); the same rays as bounce_rays given the global positions. With order=True the result
    has a fourth tensor: a tracing order with the active rays first (for batch_trace's `order`); a given `out`
    with four tensors keeps its fourth unwritten when order=False."""
    R = orig.shape[0]
    dev = orig.device
    if out is None:
        out = (torch.empty((R, 4), dtype=torch.float32, device=dev), torch.empty((R, 4), dtype=torch.float32, device=dev),
               torch.empty(R, dtype=torch.float32, device=dev))
        if order:
            out = out + (torch.empty(R + 2, dtype=torch.int32, device=dev),)  # R order entries, then two counters
    ord_ = out[3] if (order and len(out) > 3) else None
    _abi.check("rt_batch_bounce_rays", _abi.lib().rt_batch_bounce_rays(
        _p(tree.tris), _p(tree.face_offsets), _p(ray_offsets), tree.mesh_count, _p(orig), _p(dir), _p(hit_pos), _p(hit_t), R,
        C.c_uint64(seed), _p(out[0]), _p(out[1]), _p(out[2]), None if ord_ is None else C.c_void_p(ord_.data_ptr()),
        None if ord_ is None else C.c_void_p(ord_[R:].data_ptr()), _stream(stream)))
    return out


def pack_hits(hits: dict, out: dict | None = None, stream=None) -> dict:
    """rt_pack_hits: the (t, u, v) of the rays that hit, in ray order, for a compact download: out["packed"]
    (float32 [3 R]; the first 3 * count entries hold them) and out["count"] (int32 [1]). Rebuild with unpack_hits."""
    ids = hits["id"]
    R = ids.numel()
    if out is None:
        nb = C.c_size_t(0)
        _abi.check("rt_pack_hits_scratch_bytes", _abi.lib().rt_pack_hits_scratch_bytes(R, C.byref(nb)))
        out = dict(packed=torch.empty(3 * max(R, 1), dtype=torch.float32, device=ids.device),
                   count=torch.zeros(1, dtype=torch.int32, device=ids.device),
                   scratch=torch.empty(max(nb.value, 1), dtype=torch.uint8, device=ids.device))
    _abi.check("rt_pack_hits", _abi.lib().rt_pack_hits(_p(ids), _p(hits["t"]), _p(hits["uv"]), R, _p(out["packed"]), _p(out["count"]),
                                                        _p(out["scratch"]), out["scratch"].numel(), _stream(stream)))
    return out


def unpack_hits(ids, packed, count: int, tmax=None):
    """The full hits (t, uv) from the ids and the packed (t, u, v) of the hits (host or device tensors): a miss has
    t = its tmax (CUDART_NORM_HUGE_F without one) and uv = 0."""
    hit = ids >= 0
    R = ids.numel()
    t = torch.full((R,), 3.402823466e38, dtype=torch.float32) if tmax is None else tmax.to(torch.float32).clone()
    t = t.to(ids.device)
    uv = torch.zeros((R, 2), dtype=torch.float32, device=ids.device)
    p = packed[:3 * count].view(count, 3)
    t[hit] = p[:, 0]
    uv[hit] = p[:, 1:]
    return t, uv


def sort_pairs(keys: torch.Tensor, values: torch.Tensor, bit_depth: int = 32, init_values: bool = False, stream=None):
    """In place, stable (CUDA_radixSortGeneral)."""
    _need_cuda(keys, "keys", _I32)
    _need_cuda(values, "values", _I32)
    n = keys.numel()
    nb = C.c_size_t(0)
    _abi.lib().rt_sort_scratch_bytes(n, C.byref(nb))
    s = _SCRATCH.get(nb.value, keys.device)
    _abi.check("rt_radix_sort_pairs", _abi.lib().rt_radix_sort_pairs(_p(keys), _p(values), n, bit_depth, int(init_values), _p(s),
                                                                     s.numel(), _stream(stream)))
    return keys, values


def sort_keys(keys: torch.Tensor, bit_depth: int = 32, stream=None):
    """In place (CUDA_radixSort)."""
    _need_cuda(keys, "keys", _I32)
    n = keys.numel()
    nb = C.c_size_t(0)
    _abi.lib().rt_sort_scratch_bytes(n, C.byref(nb))
    s = _SCRATCH.get(nb.value, keys.device)
    _abi.check("rt_radix_sort_keys", _abi.lib().rt_radix_sort_keys(_p(keys), n, bit_depth, _p(s), s.numel(), _stream(stream)))
    return keys


def mesh_boxes(vertices, faces, stream=None):
    n = faces.shape[0]
    boxes = torch.empty((n, 8), dtype=torch.float32, device=vertices.device)
    idx = torch.empty(n, dtype=torch.int32, device=vertices.device)
    _abi.check("rt_mesh_boxes", _abi.lib().rt_mesh_boxes(_p(vertices), _p(faces), n, _p(boxes), _p(idx), _stream(stream)))
    return boxes, idx


def reorder_faces(faces, indices, stream=None):
    out = torch.empty_like(faces)
    _abi.check("rt_reorder_faces", _abi.lib().rt_reorder_faces(_p(faces), _p(indices), faces.shape[0], _p(out), _stream(stream)))
    return out


def interpolate(tree: Tree, vertices: torch.Tensor, hits: dict, normals=None, colors=None, texcoords=None,
                outputs=("points", "normals", "colors", "texcoords", "materials"), stream=None) -> dict:
    """CUDARaytracer::interpolateOutputSurfaces: per-ray hit point, normal, color,
    texcoord and material from the trace's (position, u, v) (id_mode 0)."""
    R = hits["id"].shape[0]
    dev = vertices.device
    shapes = {"points": (R, 4), "normals": (R, 4), "colors": (R, 4), "texcoords": (R, 2), "materials": (R,)}
    out = {k: torch.empty(shapes[k], dtype=torch.int32 if k == "materials" else torch.float32, device=dev) for k in outputs}
    d = _abi.InterpDesc()
    d.hit_id = hits["id"].data_ptr()
    d.hit_uv = hits["uv"].data_ptr()
    d.count = R
    d.faces = tree.faces.data_ptr()
    d.vertices = vertices.data_ptr()
    d.normals = normals.data_ptr() if normals is not None else None
    d.colors = colors.data_ptr() if colors is not None else None
    d.texcoords = texcoords.data_ptr() if texcoords is not None else None
    for k in outputs:
        setattr(d, "out_" + k, out[k].data_ptr())
    _abi.check("rt_interpolate", _abi.lib().rt_interpolate(C.byref(d), _stream(stream)))
    return out


# ----------------------------------------------------------------------------
# chunk files (CUDAMesh / CUDAMeshTree quickSave / quickLoad)
# ----------------------------------------------------------------------------
def mesh_save(path: str, vertices, faces, hitbox, normals=None, colors=None, texcoords=None, overwrite: bool = True):
    m = _abi.MeshFile()
    m.hitbox[:] = [float(x) for x in hitbox]
    m.has_hitbox = 1
    for name, t in (("vertices", vertices), ("normals", normals), ("colors", colors), ("texcoords", texcoords), ("faces", faces)):
        if t is not None:
            setattr(m, name, t.data_ptr())
            setattr(m, {"vertices": "vertex_count", "normals": "normal_count", "colors": "color_count",
                        "texcoords": "texcoord_count", "faces": "face_count"}[name], t.shape[0])
    torch.cuda.synchronize()
    _abi.check("rt_mesh_file_save", _abi.lib().rt_mesh_file_save(path.encode(), int(overwrite), C.byref(m)))


def mesh_load(path: str, device="cuda") -> dict:
    m = _abi.MeshFile()
    _abi.check("rt_mesh_file_info", _abi.lib().rt_mesh_file_info(path.encode(), C.byref(m)))
    out = {"hitbox": list(m.hitbox) if m.has_hitbox else None}
    spec = (("vertices", "vertex_count", 4, torch.float32), ("normals", "normal_count", 4, torch.float32),
            ("colors", "color_count", 4, torch.float32), ("texcoords", "texcoord_count", 2, torch.float32),
            ("faces", "face_count", 4, torch.int32))
    for name, cnt, cols, dt in spec:
        n = getattr(m, cnt)
        if n:
            t = torch.empty((n, cols), dtype=dt, device=device)
            setattr(m, name, t.data_ptr())
            out[name] = t
    _abi.check("rt_mesh_file_load", _abi.lib().rt_mesh_file_load(path.encode(), C.byref(m)))
    return out


def tree_save(path: str, tree: Tree, overwrite: bool = True):
    t = _abi.TreeFile()
    t.node_count = tree.node_count
    t.index_count = tree.indices.shape[0]
    t.box_count = tree.boxes.shape[0]
    t.nodes, t.indices, t.boxes = tree.nodes.data_ptr(), tree.indices.data_ptr(), tree.boxes.data_ptr()
    torch.cuda.synchronize()
    _abi.check("rt_tree_file_save", _abi.lib().rt_tree_file_save(path.encode(), int(overwrite), C.byref(t)))


def tree_load(path: str, device="cuda") -> dict:
    t = _abi.TreeFile()
    _abi.check("rt_tree_file_info", _abi.lib().rt_tree_file_info(path.encode(), C.byref(t)))
    out = {}
    for name, cnt, cols, dt in (("nodes", "node_count", 8, torch.int32), ("indices", "index_count", 1, torch.int32),
                                ("boxes", "box_count", 8, torch.float32)):
        n = getattr(t, cnt)
        if n:
            x = torch.empty((n, cols) if cols > 1 else (n,), dtype=dt, device=device)
            setattr(t, name, x.data_ptr())
            out[name] = x
    _abi.check("rt_tree_file_load", _abi.lib().rt_tree_file_load(path.encode(), C.byref(t)))
    return out


# ----------------------------------------------------------------------------
# batched meshes (one set of launches for all builds, one launch for all rays)
# ----------------------------------------------------------------------------
@dataclass
class BatchTree:
    face_offsets: torch.Tensor    # int32 (M + 1,) on the device
    vertex_offsets: torch.Tensor  # int32 (M + 1,)
    face_offsets_host: list
    nodes: torch.Tensor           # int32 (2N - M, 8): mesh m's nodes start at 2 F_m - m
    boxes: torch.Tensor
    indices: torch.Tensor         # mesh-local face ids per position
    codes: torch.Tensor
    faces: torch.Tensor           # per mesh, Morton order
    tris: torch.Tensor
    accel: torch.Tensor
    info: torch.Tensor            # int32 (M, 8)
    clusters: bool = False        # the blob also holds every mesh's cluster tree

    @property
    def mesh_count(self) -> int:
        return self.face_offsets.shape[0] - 1

    def mesh_nodes(self, m: int, node_count: int | None = None):
        F = self.face_offsets_host[m]
        nc = int(self.info[m, 0].item()) if node_count is None else node_count
        base = 2 * F - m
        return self.nodes[base: base + nc]


def batch_build(vertices: torch.Tensor, faces: torch.Tensor, face_offsets: list, vertex_offsets: list, tree_depth: int = 12,
                out: BatchTree | None = None, stream=None, clusters: bool = False, cluster_leaf: int = 0) -> BatchTree:
    """Builds every mesh of a concatenated batch (faces index their own mesh's vertices from 0); clusters: also
    every mesh's cluster tree (RT_ACCEL_CLUSTERS), for schedules with "clusters": True."""
    _need_cuda(vertices, "vertices", _F32, 4)
    _need_cuda(faces, "faces", _I32, 4)
    M = len(face_offsets) - 1
    N = faces.shape[0]
    dev = vertices.device
    params = _abi.BuildParams(tree_depth, 1, 0, 0, 32, _abi.ACCEL_CLUSTERS if clusters else 0, cluster_leaf)
    sb, ab = C.c_size_t(0), C.c_size_t(0)
    _abi.check("rt_batch_sizes", _abi.lib().rt_batch_sizes(M, N, C.byref(params), C.byref(sb), C.byref(ab)))
    if out is None:
        out = BatchTree(
            face_offsets=torch.tensor(face_offsets, dtype=torch.int32, device=dev),
            vertex_offsets=torch.tensor(vertex_offsets, dtype=torch.int32, device=dev),
            face_offsets_host=list(face_offsets),
            nodes=torch.empty((2 * N - M, 8), dtype=torch.int32, device=dev),
            boxes=torch.empty((N, 8), dtype=torch.float32, device=dev),
            indices=torch.empty(N, dtype=torch.int32, device=dev),
            codes=torch.empty(N, dtype=torch.int32, device=dev),
            faces=torch.empty((N, 4), dtype=torch.int32, device=dev),
            tris=torch.empty((N, 12), dtype=torch.float32, device=dev),
            accel=torch.empty(ab.value, dtype=torch.uint8, device=dev),
            info=torch.zeros((M, 8), dtype=torch.int32, device=dev),
        )
    scratch = _SCRATCH.get(sb.value, dev)
    d = _abi.BatchBuildDesc()
    d.mesh_count, d.face_count, d.vertex_count = M, N, vertices.shape[0]
    d.face_offsets, d.vertex_offsets = out.face_offsets.data_ptr(), out.vertex_offsets.data_ptr()
    d.vertices, d.faces_in, d.faces_out = vertices.data_ptr(), faces.data_ptr(), out.faces.data_ptr()
    d.params = params
    d.boxes, d.indices, d.codes, d.nodes = out.boxes.data_ptr(), out.indices.data_ptr(), out.codes.data_ptr(), out.nodes.data_ptr()
    d.tris, d.accel, d.accel_bytes = out.tris.data_ptr(), out.accel.data_ptr(), out.accel.numel()
    d.info, d.scratch, d.scratch_bytes = out.info.data_ptr(), scratch.data_ptr(), scratch.numel()
    _abi.check("rt_batch_build", _abi.lib().rt_batch_build(C.byref(d), _stream(stream)))
    out.clusters = bool(clusters)
    return out


_TILE_ORDERS = {}


def image_tile_order(images: int, width: int, height: int, device="cuda", stream=None) -> torch.Tensor:
    """rt_image_tile_order: the slot -> ray permutation that gives each warp an 8 x 4 pixel tile of one of
    `images` consecutive row-major width x height images (made once per shape and device, then reused)."""
    dev = torch.device(device)
    key = (dev.index or 0, images, width, height)
    o = _TILE_ORDERS.get(key)
    if o is None:
        o = torch.empty(images * width * height, dtype=torch.int32, device=dev)
        _abi.check("rt_image_tile_order", _abi.lib().rt_image_tile_order(images, width, height, _p(o), _stream(stream)))
        _TILE_ORDERS[key] = o
    return o


def batch_tree_box(tree: "BatchTree"):
    """Box around every mesh of a batched build (host floats), from the meshes' root nodes; read once and
    cached on the tree. A tree rebuilt in place keeps the first box: it only steers the ray order."""
    box = getattr(tree, "_box", None)
    if box is None:
        M = tree.mesh_count
        F = torch.tensor(tree.face_offsets_host[:M], dtype=torch.int64, device=tree.nodes.device)
        roots = tree.nodes[2 * F - torch.arange(M, device=F.device)].view(torch.float32)[:, 2:8].cpu()
        ok = roots.abs().max(dim=1).values < 1e30
        r = roots[ok] if bool(ok.any()) else tree.boxes.view(-1, 8)[:, [0, 1, 2, 4, 5, 6]].cpu()
        box = r[:, :3].min(0).values.tolist() + r[:, 3:].max(0).values.tolist()
        tree._box = box
    return box


def batch_ray_order(orig, dir, tmax, ray_offsets, mesh_count: int, box, morton_bits: int, ray_count: int | None = None, out=None,
                    stream=None) -> torch.Tensor:
    """rt_batch_ray_order: rays sorted by mesh, direction octant and the top `morton_bits` bits of their origin's
    Morton code in `box`; inactive rays (tmax <= 0) last."""
    R = orig.shape[0] if ray_count is None else ray_count
    nb = C.c_size_t(0)
    _abi.lib().rt_batch_ray_order_scratch_bytes(R, C.byref(nb))
    scratch = _ORDER_SCRATCH.get(nb.value, orig.device)
    order = torch.empty(R, dtype=torch.int32, device=orig.device) if out is None else out
    b = (C.c_float * 6)(*box)
    _abi.check("rt_batch_ray_order", _abi.lib().rt_batch_ray_order(_p(orig), _p(dir), _p(tmax), R, _p(ray_offsets), mesh_count, b,
                                                                   morton_bits, _p(order), _p(scratch), scratch.numel(), _stream(stream)))
    return order


def batch_trace(tree: BatchTree, orig, dir, ray_offsets: torch.Tensor, tmax=None, id_mode: int = 0, counters: bool = False,
                while_while: bool = True, out: dict | None = None, schedule: dict | None = None, order=None, stream=None,
                bounce=None) -> dict:
    """Closest hits for the rays of all meshes (rays of mesh m: ray_offsets[m] .. ray_offsets[m+1]).
    schedule (results never depend on it): while_while, wide (4-wide records),
    persistent + blocks_per_sm (warps fetching 32 rays at a time), coop
    (warp-cooperative leaf tests; always persistent), tiles = (images, width,
    height) (every mesh's rays are one image: warps take 8 x 4 pixel tiles) or
    sorted_bits (rays sorted by mesh, octant and that many bits of their
    origin's Morton code, inactive rays last; the sort is part of the call). `order`: a tracing order given by
    the caller (for instance batch_bounce_rays' order), used in place of the schedule's. `bounce`: (seed, None or
    three tensors) to get each ray's diffuse bounce too, exactly as batch_bounce_rays(..., seed) makes it from these
    hits, as out["b"] = (orig, dir, tmax); the packet schedule writes them as each ray finishes (no second pass
    over the hits)."""
    d, out = batch_trace_desc(tree, orig, dir, ray_offsets, tmax, id_mode, counters, while_while, out, schedule, order)
    if bounce is not None:
        seed, bout = bounce
        if bout is None:
            R = orig.shape[0]
            bout = (torch.empty((R, 4), dtype=torch.float32, device=orig.device), torch.empty((R, 4), dtype=torch.float32, device=orig.device),
                    torch.empty(R, dtype=torch.float32, device=orig.device))
        d.bounce_seed = int(seed)
        d.bounce_orig, d.bounce_dir, d.bounce_tmax = bout[0].data_ptr(), bout[1].data_ptr(), bout[2].data_ptr()
        out["b"] = bout
    _abi.check("rt_batch_trace", _abi.lib().rt_batch_trace(C.byref(d), _stream(stream)))
    return out


def batch_trace_desc(tree: BatchTree, orig, dir, ray_offsets: torch.Tensor, tmax=None, id_mode: int = 0, counters: bool = False,
                     while_while: bool = True, out: dict | None = None, schedule: dict | None = None, order=None):
    """The rt_batch_trace_desc of batch_trace and its output tensors."""
    R = orig.shape[0]
    dev = orig.device
    if out is None:
        out = dict(id=torch.empty(R, dtype=torch.int32, device=dev), t=torch.empty(R, dtype=torch.float32, device=dev),
                   uv=torch.empty((R, 2), dtype=torch.float32, device=dev), err=torch.zeros(1, dtype=torch.int32, device=dev))
        if counters:
            out["visits"] = torch.empty(R, dtype=torch.int32, device=dev)
            out["tests"] = torch.empty(R, dtype=torch.int32, device=dev)
    d = _abi.BatchTraceDesc()
    d.mesh_count = tree.mesh_count
    d.face_offsets, d.ray_offsets = tree.face_offsets.data_ptr(), ray_offsets.data_ptr()
    d.accel, d.tris, d.indices, d.face_count = tree.accel.data_ptr(), tree.tris.data_ptr(), tree.indices.data_ptr(), tree.faces.shape[0]
    d.orig, d.dir, d.tmax, d.ray_count, d.id_mode = orig.data_ptr(), dir.data_ptr(), _p(tmax), R, id_mode
    d.hit_id, d.hit_t, d.hit_uv, d.error_word = out["id"].data_ptr(), out["t"].data_ptr(), out["uv"].data_ptr(), out["err"].data_ptr()
    if "visits" in out:
        d.ray_visits, d.ray_tests = out["visits"].data_ptr(), out["tests"].data_ptr()
    sch = dict(while_while=while_while) if schedule is None else schedule
    d.schedule = ((_abi.TRACE_WHILE_WHILE if sch.get("while_while", False) else 0)
                  | (_abi.TRACE_WIDE if sch.get("wide", False) else 0)
                  | (_abi.TRACE_COOP if sch.get("coop", False) else 0)
                  | (_abi.TRACE_CLUSTERS if sch.get("clusters", False) else 0)
                  | (_abi.TRACE_PACKET if sch.get("packet", False) else 0)
                  | (_abi.TRACE_REFILL if sch.get("refill", False) else 0))
    if order is not None:
        d.ray_order = order.data_ptr()
    elif sch.get("tiles"):  # every mesh's rays are a row-major image of the same size: 8 x 4 pixel tiles per warp
        images, width, height = sch["tiles"]
        key = (int(images), int(width), int(height))
        if out.get("_tile_key") != key:  # the order depends on the image shape only: made once per output set
            out["_order"] = image_tile_order(images, width, height, dev)
            out["_tile_key"] = key
        d.ray_order = out["_order"].data_ptr()
    elif sch.get("sorted_bits") is not None:  # sorted by mesh, octant and origin Morton code (part of the call)
        order = batch_ray_order(orig, dir, tmax, ray_offsets, tree.mesh_count, batch_tree_box(tree), int(sch["sorted_bits"]),
                                ray_count=R)
        out["_order"] = order  # keep it alive until the trace has run
        out.pop("_tile_key", None)
        d.ray_order = order.data_ptr()
    if sch.get("persistent", False) or sch.get("coop", False):
        if "_counter" not in out:
            out["_counter"] = torch.zeros(1, dtype=torch.int32, device=dev)
        d.work_counter = out["_counter"].data_ptr()
        d.persistent_blocks_per_sm = int(sch.get("blocks_per_sm", 8))
    d.lane_threshold = int(sch.get("lane_threshold", 0))
    return d, out
