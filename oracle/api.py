"""ctypes front end of the CPU oracle (oracle/rt_oracle.cpp) and of the
reference checker built from the reference's own sources (oracle/build_ref.sh).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline / reference legs, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "librt_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_cudart.so")

_P = C.c_void_p
_U32 = C.c_uint32
HUGE = np.float32(3.402823466e38)


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _ptr(a):
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("oracle arrays must be C-contiguous")
    return a.ctypes.data_as(_P)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.or_build_topology.restype = _U32
        L.or_lbvh_build.restype = _U32
        L.or_max_threads.restype = C.c_int
        L.or_trace.argtypes = [_P, _P, _P, _P, _P, _P, C.c_long, C.c_long, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P]
        L.or_trace_brute.argtypes = [_P, _U32, _P, _P, _P, C.c_long, _P, _P, _P]
        L.or_bounce_rays.argtypes = [_P, _P, _P, _P, _P, C.c_long, C.c_uint64, _P, _P, _P]
        L.or_camera_basis.argtypes = [_P, _P, C.c_float, C.c_float, C.c_int, C.c_int, _P]
        L.or_primary_rays.argtypes = [_P, C.c_int, C.c_int, _P, _P]
        L.or_lbvh_build.argtypes = [_P, _U32, _P, _U32, _P, _U32, C.c_int, C.c_int, _P, _P, _P, _P, _U32, _P, _P, _P]
        L.or_build_topology.argtypes = [_P, _U32, _U32, C.c_int, _U32, _U32, _P, _U32, _P]
        L.or_interpolate.argtypes = [_P, _P, C.c_long, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.or_raster_matrix.argtypes = [_P, _P, _P, C.c_float, C.c_float, _P]
        L.or_rasterize.argtypes = [_P, _P, _U32, _P, C.c_int, C.c_int, _P, _P, _P]
        L.or_sah_build.restype = C.c_int
        L.or_sah_build.argtypes = [_P, _P, _P, _U32, _P, _U32, _P, _U32, _P, _P]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(REF_SO)
        R.ref_lbvh_build.restype = _U32
        R.ref_lbvh_build.argtypes = [_P, _U32, _P, _U32, C.c_int, _P, _P, _P, _U32, _P]
        R.ref_mesh_boxes.argtypes = [_P, _P, _U32, _P, _P]
        R.ref_reorder_faces.argtypes = [_P, _P, _U32, _P]
        R.ref_trace.argtypes = [_P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P]
        R.ref_camera_rays.argtypes = [_P, _P, C.c_float, C.c_float, C.c_int, C.c_int, _P, _P, _P, _P]
        R.ref_interpolate.argtypes = [_P, _P, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        R.ref_raster_matrix.argtypes = [_P, _P, _P, C.c_float, C.c_float, _P]
        R.ref_rasterize.argtypes = [_P, _P, C.c_int, _P, C.c_int, C.c_int, _P, _P, _P]
        R.ref_sah_build.restype = C.c_int
        R.ref_sah_build.argtypes = [_P, _P, _P, _U32, _P, _U32, _P, _U32, _P]
        _ref = R
    return _ref


# ----------------------------------------------------------------------------
# oracle wrappers
# ----------------------------------------------------------------------------
def hitbox(vertices):
    out = np.zeros(8, np.float32)
    lib().or_hitbox(_ptr(vertices), _U32(len(vertices)), _ptr(out))
    return out


def mesh_boxes(vertices, faces):
    n = len(faces)
    boxes = np.zeros((n, 8), np.float32)
    idx = np.zeros(n, np.uint32)
    lib().or_mesh_boxes(_ptr(vertices), _ptr(faces), _U32(n), _ptr(boxes), _ptr(idx))
    return boxes, idx


def morton(boxes, hit, layout=32):
    codes = np.zeros(len(boxes), np.uint32)
    lib().or_morton(_ptr(boxes), _U32(len(boxes)), _ptr(hit), C.c_int(layout), _ptr(codes))
    return codes


def sort_pairs(keys, vals=None, bit_depth=32, init_vals=False):
    k = np.ascontiguousarray(keys, np.uint32).copy()
    v = None if vals is None and not init_vals else (np.zeros(len(k), np.uint32) if vals is None else np.ascontiguousarray(vals, np.uint32).copy())
    lib().or_sort_pairs(_ptr(k), _ptr(v), _U32(len(k)), _U32(bit_depth), C.c_int(1 if init_vals else 0))
    return k, v


def topology(sorted_codes, tree_depth=12, tree_complete=True, min_leaf=16, max_leaf=224):
    n = len(sorted_codes)
    cap = 2 * n + 64
    nodes = np.zeros((cap, 8), np.float32)
    st = np.zeros(8, np.uint32)
    nc = lib().or_build_topology(_ptr(sorted_codes), _U32(n), _U32(tree_depth), C.c_int(int(tree_complete)),
                                 _U32(min_leaf), _U32(max_leaf), _ptr(nodes), _U32(cap), _ptr(st))
    return nodes[:nc].copy(), st


INFO_KEYS = ("node_count", "leaf_count", "real_depth", "split_count", "overrun_visits", "nondet_reads", "past_end_reads", "error")


def lbvh_build(vertices, faces, hit=None, tree_depth=12, tree_complete=True, layout=32):
    """Full oracle build. Returns dict with boxes, indices (sorted), codes (sorted),
    nodes (node_count x 8 words viewed as float32), faces (reordered), tris, info."""
    n = len(faces)
    cap = 2 * n + 64
    boxes = np.zeros((n, 8), np.float32)
    idx = np.zeros(n, np.uint32)
    codes = np.zeros(n, np.uint32)
    nodes = np.zeros((cap, 8), np.float32)
    faces_out = np.zeros_like(faces)
    tris = np.zeros((n, 12), np.float32)
    info = np.zeros(8, np.uint32)
    nc = lib().or_lbvh_build(_ptr(vertices), _U32(len(vertices)), _ptr(faces), _U32(n), _ptr(hit), _U32(tree_depth),
                             C.c_int(int(tree_complete)), C.c_int(layout), _ptr(boxes), _ptr(idx), _ptr(codes), _ptr(nodes),
                             _U32(cap), _ptr(faces_out), _ptr(tris), _ptr(info))
    return dict(boxes=boxes, indices=idx, codes=codes, nodes=nodes[:nc].copy(), faces=faces_out, tris=tris,
                info=dict(zip(INFO_KEYS, (int(x) for x in info))))


def sah_build(vertices, faces, hit=None, hybrid_depth=None):
    """Full oracle SAH build (CUDAMeshTree::buildMeshTreeSAH) or, with
    hybrid_depth, the Hybrid build (LBVH of that depth without leaf splitting
    or reorder, then SAH on every leaf). Returns dict with boxes, indices,
    nodes, faces (reordered), tris, no_split (leaves made because no bin
    boundary splits a node of >= 224 faces)."""
    n = len(faces)
    if hit is None:
        hit = np.zeros(8, np.float32)
        lib().or_hitbox(_ptr(vertices), _U32(len(vertices)), _ptr(hit))
    hit = np.ascontiguousarray(hit, np.float32)
    cap = 2 * n + 64
    if hybrid_depth is None:
        boxes = np.zeros((n, 8), np.float32)
        idx = np.zeros(n, np.uint32)
        lib().or_mesh_boxes(_ptr(vertices), _ptr(faces), _U32(n), _ptr(boxes), _ptr(idx))
        nodes_in, nc_in = None, 0
    else:
        lb = lbvh_build(vertices, faces, hit, tree_depth=hybrid_depth, tree_complete=False)
        boxes, idx = lb["boxes"], lb["indices"].copy()
        nodes_in, nc_in = np.ascontiguousarray(lb["nodes"]), lb["info"]["node_count"]
        cap += nc_in
    nodes = np.zeros((cap, 8), np.float32)
    nc = np.zeros(1, np.uint32)
    stats = np.zeros(4, np.uint32)
    rc = lib().or_sah_build(_ptr(boxes), _ptr(hit), _ptr(idx), _U32(n), _ptr(nodes_in), _U32(nc_in), _ptr(nodes), _U32(cap),
                            _ptr(nc), _ptr(stats))
    if rc != 0:
        raise RuntimeError(f"or_sah_build failed ({rc})")
    faces_out = np.zeros_like(faces)
    lib().or_reorder_faces(_ptr(faces), _ptr(idx), _U32(n), _ptr(faces_out))
    tris = np.zeros((n, 12), np.float32)
    lib().or_pack_tris(_ptr(vertices), _ptr(faces_out), _U32(n), _ptr(tris))
    return dict(boxes=boxes, indices=idx, nodes=nodes[: int(nc[0])].copy(), faces=faces_out, tris=tris, no_split=int(stats[0]))


def look_dir(center, target):
    """CUDACamera::lookAt's direction: (target - center) * (1 / sqrtf(|.|^2)) in float32."""
    c = np.asarray(center, np.float32)
    t = np.asarray(target, np.float32)
    d = (t - c).astype(np.float32)
    inv = np.float32(1.0) / np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])))
    return (d * inv).astype(np.float32)


def raster_matrix(center, dir3, angle, fov, ratio):
    out = np.zeros(16, np.float32)
    lib().or_raster_matrix(_ptr(np.asarray(center, np.float32)), _ptr(np.asarray(dir3, np.float32)), _ptr(np.asarray(angle, np.float32)),
                           C.c_float(fov), C.c_float(ratio), _ptr(out))
    return out


def rasterize(vertices, faces, matrix, width, height, faces_id=None, coords=None, depths=None):
    """Oracle rasteriser; buffers start as CUDABuffer::clearOutputSurfaces leaves them
    (id 0, uv 0, depth +HUGE) unless given. Returns (faces_id, coords, depths)."""
    P = width * height
    fid = np.zeros(P, np.uint32) if faces_id is None else faces_id.copy()
    uv = np.zeros((P, 2), np.float32) if coords is None else coords.copy()
    dep = np.full(P, HUGE, np.float32) if depths is None else depths.copy()
    lib().or_rasterize(_ptr(vertices), _ptr(faces), _U32(len(faces)), _ptr(np.asarray(matrix, np.float32)), C.c_int(width),
                       C.c_int(height), _ptr(fid), _ptr(uv), _ptr(dep))
    return fid, uv, dep


def ref_raster_matrix(center, dir3, angle, fov, ratio):
    out = np.zeros(16, np.float32)
    ref().ref_raster_matrix(_ptr(np.asarray(center, np.float32)), _ptr(np.asarray(dir3, np.float32)), _ptr(np.asarray(angle, np.float32)),
                            C.c_float(fov), C.c_float(ratio), _ptr(out))
    return out


def ref_rasterize(vertices, faces, matrix, width, height):
    P = width * height
    fid = np.zeros(P, np.uint32)
    uv = np.zeros((P, 2), np.float32)
    dep = np.full(P, HUGE, np.float32)
    ref().ref_rasterize(_ptr(vertices), _ptr(faces), C.c_int(len(faces)), _ptr(np.asarray(matrix, np.float32)), C.c_int(width),
                        C.c_int(height), _ptr(fid), _ptr(uv), _ptr(dep))
    return fid, uv, dep


def camera_look_at(center, target):
    out = np.zeros(3, np.float32)
    lib().or_camera_look_at(_ptr(np.asarray(center, np.float32)), _ptr(np.asarray(target, np.float32)), _ptr(out))
    return out


def camera_basis(center, angle, fov, ratio, width, height):
    out = np.zeros(16, np.float32)
    lib().or_camera_basis(_ptr(np.asarray(center, np.float32)), _ptr(np.asarray(angle, np.float32)), C.c_float(fov),
                          C.c_float(ratio), C.c_int(width), C.c_int(height), _ptr(out))
    return out


def primary_rays(cam):
    ang = camera_look_at(cam.center, cam.target)
    basis = camera_basis(cam.center, ang, cam.fov, cam.ratio, cam.width, cam.height)
    R = cam.width * cam.height
    o = np.zeros((R, 4), np.float32)
    d = np.zeros((R, 4), np.float32)
    lib().or_primary_rays(_ptr(basis), C.c_int(cam.width), C.c_int(cam.height), _ptr(o), _ptr(d))
    return o, d, basis, ang


def trace(nodes, tris, indices, orig, dir, depth=None, mode=0, id_mode=0, begin=0, end=None, threads=0, counters=False):
    R = len(orig)
    end = R if end is None else end
    ids = np.full(R, -1, np.int32)
    t = np.zeros(R, np.float32)
    uv = np.zeros((R, 2), np.float32)
    vis = np.zeros(R, np.uint32) if counters else None
    tst = np.zeros(R, np.uint32) if counters else None
    lib().or_trace(_ptr(nodes), _ptr(tris), _ptr(indices), _ptr(orig), _ptr(dir), _ptr(depth), C.c_long(begin), C.c_long(end),
                   C.c_int(mode), C.c_int(id_mode), C.c_int(threads), _ptr(ids), _ptr(t), _ptr(uv), _ptr(vis), _ptr(tst))
    out = dict(id=ids, t=t, uv=uv)
    if counters:
        out.update(visits=vis, tests=tst)
    return out


def trace_brute(tris, orig, dir, depth=None):
    R = len(orig)
    ids = np.zeros(R, np.int32)
    t = np.zeros(R, np.float32)
    uv = np.zeros((R, 2), np.float32)
    lib().or_trace_brute(_ptr(tris), _U32(len(tris)), _ptr(orig), _ptr(dir), _ptr(depth), C.c_long(R), _ptr(ids), _ptr(t), _ptr(uv))
    return dict(id=ids, t=t, uv=uv)


def bounce_rays(tris, orig, dir, hit_pos, hit_t, seed):
    R = len(orig)
    o = np.zeros((R, 4), np.float32)
    d = np.zeros((R, 4), np.float32)
    dep = np.zeros(R, np.float32)
    lib().or_bounce_rays(_ptr(tris), _ptr(orig), _ptr(dir), _ptr(hit_pos), _ptr(hit_t), C.c_long(R), C.c_uint64(seed),
                         _ptr(o), _ptr(d), _ptr(dep))
    return o, d, dep


def interpolate(hit_id, hit_uv, faces, vertices, normals=None, colors=None, texcoords=None):
    R = len(hit_id)
    out = dict(points=np.zeros((R, 4), np.float32), normals=np.zeros((R, 4), np.float32), colors=np.zeros((R, 4), np.float32),
               texcoords=np.zeros((R, 2), np.float32), materials=np.zeros(R, np.uint32))
    lib().or_interpolate(_ptr(hit_id), _ptr(hit_uv), C.c_long(R), _ptr(faces), _ptr(vertices), _ptr(normals), _ptr(colors),
                         _ptr(texcoords), _ptr(out["points"]), _ptr(out["normals"]), _ptr(out["colors"]), _ptr(out["texcoords"]),
                         _ptr(out["materials"]))
    return out


def max_threads() -> int:
    return int(lib().or_max_threads())


def set_threads(n: int) -> None:
    """Thread count of the oracle's parallel loops (n <= 0: all processors)."""
    lib().or_set_threads(C.c_int(n))


# ----------------------------------------------------------------------------
# reference checker wrappers (functions compiled from the reference sources)
# ----------------------------------------------------------------------------
def ref_mesh_boxes(vertices, faces):
    n = len(faces)
    boxes = np.zeros((n, 8), np.float32)
    idx = np.zeros(n, np.uint32)
    ref().ref_mesh_boxes(_ptr(vertices), _ptr(faces), _U32(n), _ptr(boxes), _ptr(idx))
    return boxes, idx


def ref_lbvh_build(boxes, hit, tree_depth=12, tree_complete=True):
    n = len(boxes)
    cap = 2 * n + 64
    codes = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    nodes = np.zeros((cap, 8), np.float32)
    info = np.zeros(3, np.uint32)
    nc = ref().ref_lbvh_build(_ptr(boxes), _U32(n), _ptr(hit), _U32(tree_depth), C.c_int(int(tree_complete)),
                              _ptr(codes), _ptr(idx), _ptr(nodes), _U32(cap), _ptr(info))
    return dict(codes=codes, indices=idx, nodes=nodes[:nc].copy(), real_depth=int(info[1]), split_count=int(info[2]))


def ref_sah_build(boxes, root_box, indices, nodes_in=None, capacity=None):
    """The reference's SAH kernels (emulated blocks, serial order) on face boxes
    and an index order; nodes_in refines an existing tree's leaves (Hybrid).
    Returns (status, nodes, indices): status 0 ok, 1 stack overflow, 2 node
    capacity exceeded (the reference does not terminate)."""
    n = len(boxes)
    idx = np.ascontiguousarray(indices, np.uint32).copy()
    nc_in = 0 if nodes_in is None else len(nodes_in)
    cap = capacity or (2 * n + 64 + nc_in)
    nodes = np.zeros((cap, 8), np.float32)
    nc = np.zeros(1, np.uint32)
    root = np.ascontiguousarray(root_box, np.float32)
    st = ref().ref_sah_build(_ptr(np.ascontiguousarray(boxes, np.float32)), _ptr(root), _ptr(idx), _U32(n),
                             _ptr(None if nodes_in is None else np.ascontiguousarray(nodes_in, np.float32)), _U32(nc_in),
                             _ptr(nodes), _U32(cap), _ptr(nc))
    return int(st), nodes[: min(int(nc[0]), cap)].copy(), idx


def ref_reorder_faces(faces, indices):
    out = np.zeros_like(faces)
    ref().ref_reorder_faces(_ptr(faces), _ptr(indices), _U32(len(faces)), _ptr(out))
    return out


def ref_trace(nodes, vertices, faces_reordered, orig, dir, width, height):
    R = width * height
    ids = np.zeros(R, np.uint32)
    uv = np.zeros((R, 2), np.float32)
    depth = np.full(R, HUGE, np.float32)
    ref().ref_trace(_ptr(nodes), _ptr(vertices), _ptr(faces_reordered), _ptr(orig), _ptr(dir), C.c_int(width), C.c_int(height),
                    _ptr(ids), _ptr(uv), _ptr(depth))
    return dict(id=ids, uv=uv, t=depth)


def ref_camera_rays(cam):
    R = cam.width * cam.height
    ang = np.zeros(3, np.float32)
    basis = np.zeros(16, np.float32)
    o = np.zeros((R, 4), np.float32)
    d = np.zeros((R, 4), np.float32)
    ref().ref_camera_rays(_ptr(np.asarray(cam.center, np.float32)), _ptr(np.asarray(cam.target, np.float32)), C.c_float(cam.fov),
                          C.c_float(cam.ratio), C.c_int(cam.width), C.c_int(cam.height), _ptr(ang), _ptr(basis), _ptr(o), _ptr(d))
    return o, d, basis, ang


def ref_interpolate(hit_id, hit_uv, width, height, faces, vertices, normals=None, colors=None, texcoords=None):
    """The reference kernel_interpolateData run per pixel (ids must be valid face positions)."""
    R = width * height
    out = dict(points=np.zeros((R, 4), np.float32), normals=np.zeros((R, 4), np.float32), colors=np.zeros((R, 4), np.float32),
               texcoords=np.zeros((R, 2), np.float32), materials=np.zeros(R, np.uint32))
    ref().ref_interpolate(_ptr(hit_id), _ptr(hit_uv), C.c_int(width), C.c_int(height), _ptr(faces), _ptr(vertices), _ptr(normals),
                          _ptr(colors), _ptr(texcoords), _ptr(out["points"]), _ptr(out["normals"]), _ptr(out["colors"]),
                          _ptr(out["texcoords"]), _ptr(out["materials"]))
    return out
