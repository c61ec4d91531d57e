"""Mesh / tree chunk files: bytes identical to the reference's own quickSave
(CUDAMesh.cpp:253-400, CUDAMeshTree.cpp:194-289, compiled from its sources into
oracle/_ref), files readable by the reference's quickLoad, and the loader's
count check the right way round. Host arrays, so no GPU is needed."""
import ctypes as C
import os

import numpy as np
import pytest

from cudart_b200 import _abi, scenes

REF = pytest.importorskip("oracle.api").ref_available()


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _mesh_file(hitbox, v, f, n=None, c=None, t=None):
    m = _abi.MeshFile()
    m.hitbox[:] = [float(x) for x in hitbox]
    m.has_hitbox = 1
    m.vertices, m.vertex_count = _p(v), len(v)
    m.faces, m.face_count = _p(f), len(f)
    if n is not None:
        m.normals, m.normal_count = _p(n), len(n)
    if c is not None:
        m.colors, m.color_count = _p(c), len(c)
    if t is not None:
        m.texcoords, m.texcoord_count = _p(t), len(t)
    return m


@pytest.fixture()
def mesh_data():
    mesh = scenes.terrain(40, 5)
    rng = np.random.default_rng(0)
    V = mesh.vertex_count
    n = rng.normal(size=(V, 4)).astype(np.float32)
    c = rng.uniform(size=(V, 4)).astype(np.float32)
    t = rng.uniform(size=(V, 2)).astype(np.float32)
    return mesh, mesh.hitbox(), n, c, t


@pytest.mark.skipif(not REF, reason="reference checker not built")
def test_mesh_file_bytes_match_reference(oracle, tmp_path, mesh_data):
    mesh, hb, n, c, t = mesh_data
    lib = _abi.lib()
    for attrs in ((None, None, None), (n, c, t)):
        ours, theirs = str(tmp_path / "ours.mesh"), str(tmp_path / "ref.mesh")
        m = _mesh_file(hb, mesh.vertices, mesh.faces, *attrs)
        assert lib.rt_mesh_file_save(ours.encode(), 1, C.byref(m)) == 0
        counts = [len(a) if a is not None else 0 for a in attrs]
        oracle.ref().ref_mesh_quick_save.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                                     C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]
        oracle.ref().ref_mesh_quick_save(theirs.encode(), _p(hb), _p(mesh.vertices), len(mesh.vertices), _p(attrs[0]), counts[0],
                                         _p(attrs[1]), counts[1], _p(attrs[2]), counts[2], _p(mesh.faces), len(mesh.faces))
        assert open(ours, "rb").read() == open(theirs, "rb").read()
        # the reference's quickLoad reads our file back
        R = oracle.ref()
        R.ref_mesh_quick_load.argtypes = [C.c_char_p] + [C.c_void_p] * 7
        hb2 = np.zeros(8, np.float32)
        cnt = np.zeros(5, np.uint32)
        v2 = np.zeros_like(mesh.vertices)
        f2 = np.zeros_like(mesh.faces)
        R.ref_mesh_quick_load(ours.encode(), _p(hb2), _p(cnt), _p(v2), None, None, None, _p(f2))
        assert list(cnt) == [len(mesh.vertices)] + counts + [len(mesh.faces)]
        assert np.array_equal(hb2, hb) and np.array_equal(v2, mesh.vertices) and np.array_equal(f2, mesh.faces)


@pytest.mark.skipif(not REF, reason="reference checker not built")
def test_tree_file_bytes_match_reference(oracle, tmp_path):
    mesh = scenes.soup(3000, seed=2)
    r = oracle.lbvh_build(mesh.vertices, mesh.faces)
    nodes = np.ascontiguousarray(r["nodes"]).view(np.uint32)
    lib = _abi.lib()
    ours, theirs = str(tmp_path / "ours.tree"), str(tmp_path / "ref.tree")
    t = _abi.TreeFile()
    t.node_count, t.index_count, t.box_count = len(nodes), len(r["indices"]), len(r["boxes"])
    t.nodes, t.indices, t.boxes = _p(nodes), _p(r["indices"]), _p(r["boxes"])
    assert lib.rt_tree_file_save(ours.encode(), 1, C.byref(t)) == 0
    R = oracle.ref()
    R.ref_tree_quick_save.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]
    R.ref_tree_quick_save(theirs.encode(), _p(nodes), len(nodes), _p(r["indices"]), len(r["indices"]), _p(r["boxes"]), len(r["boxes"]))
    assert open(ours, "rb").read() == open(theirs, "rb").read()


def test_file_round_trip_append_and_checks(tmp_path, mesh_data):
    mesh, hb, n, c, t = mesh_data
    lib = _abi.lib()
    path = str(tmp_path / "scene.bin")
    m = _mesh_file(hb, mesh.vertices, mesh.faces, n, c, t)
    assert lib.rt_mesh_file_save(path.encode(), 1, C.byref(m)) == 0
    # a tree appended to the same file (chunks of both kinds share a file)
    nodes = np.arange(8 * 5, dtype=np.uint32).reshape(5, 8)
    idx = np.arange(7, dtype=np.uint32)
    boxes = np.ones((7, 8), np.float32)
    tf = _abi.TreeFile()
    tf.node_count, tf.index_count, tf.box_count = 5, 7, 7
    tf.nodes, tf.indices, tf.boxes = _p(nodes), _p(idx), _p(boxes)
    assert lib.rt_tree_file_save(path.encode(), 0, C.byref(tf)) == 0
    info = _abi.MeshFile()
    assert lib.rt_mesh_file_info(path.encode(), C.byref(info)) == 0
    assert (info.vertex_count, info.normal_count, info.color_count, info.texcoord_count, info.face_count) == (
        mesh.vertex_count, mesh.vertex_count, mesh.vertex_count, mesh.vertex_count, mesh.face_count)
    out = {k: np.zeros_like(a) for k, a in (("v", mesh.vertices), ("f", mesh.faces), ("n", n), ("c", c), ("t", t))}
    info.vertices, info.faces, info.normals, info.colors, info.texcoords = (_p(out[k]) for k in ("v", "f", "n", "c", "t"))
    assert lib.rt_mesh_file_load(path.encode(), C.byref(info)) == 0
    assert np.array_equal(out["v"], mesh.vertices) and np.array_equal(out["f"], mesh.faces)
    assert np.array_equal(out["n"], n) and np.array_equal(out["c"], c) and np.array_equal(out["t"], t)
    assert np.array_equal(np.array(list(info.hitbox), np.float32), hb)
    ti = _abi.TreeFile()
    assert lib.rt_tree_file_info(path.encode(), C.byref(ti)) == 0
    assert (ti.node_count, ti.index_count, ti.box_count) == (5, 7, 7)
    n2, i2, b2 = np.zeros_like(nodes), np.zeros_like(idx), np.zeros_like(boxes)
    ti.nodes, ti.indices, ti.boxes = _p(n2), _p(i2), _p(b2)
    assert lib.rt_tree_file_load(path.encode(), C.byref(ti)) == 0  # the reference's inverted count check would abort here
    assert np.array_equal(n2, nodes) and np.array_equal(i2, idx) and np.array_equal(b2, boxes)
    # a buffer of the wrong size is refused
    ti.index_count = 6
    assert lib.rt_tree_file_load(path.encode(), C.byref(ti)) == 5  # RT_ERR_CAPACITY
    # truncated file is refused
    data = open(path, "rb").read()
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(data[:-3])
    assert lib.rt_mesh_file_info(bad.encode(), C.byref(_abi.MeshFile())) == 1
