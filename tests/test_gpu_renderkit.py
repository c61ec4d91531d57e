"""The C++ drop-in (include/cudart_b200/renderkit.hpp), driven by
tests/cpp/test_renderkit.cpp the way the reference's samples drive
CUDAMeshTree / CUDARaytracer / CUDA_radixSortGeneral, compared bit for bit
with the CPU oracle."""
import os
import subprocess

import numpy as np
import pytest

from cudart_b200 import scenes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cpp", "_build", "test_renderkit")


@pytest.mark.parametrize("scene", ["terrain", "soup"])
def test_renderkit_dropin(oracle, tmp_path, scene):
    import __graft_entry__
    __graft_entry__.build_cpp_tests()  # rebuilds when older than the headers or the library
    if scene == "terrain":
        mesh, cam = scenes.terrain_small_scene(256, 192)
    else:
        mesh, cam = scenes.soup(60000, seed=41), scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 160, 96)
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 21, 100003, dtype=np.int64).astype(np.uint32)
    hit = oracle.hitbox(mesh.vertices)
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([mesh.vertex_count, mesh.face_count, cam.width, cam.height, 12, keys.size], np.uint32).tofile(f)
        np.array(list(cam.center) + list(cam.target) + [cam.fov, cam.ratio], np.float32).tofile(f)
        hit.tofile(f)
        mesh.vertices.tofile(f)
        mesh.faces.tofile(f)
        keys.tofile(f)
    r = subprocess.run([EXE, str(inp), str(outp)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = np.fromfile(outp, np.uint8)
    off = 0

    def take(dtype, count):
        nonlocal off
        a = raw[off: off + count * np.dtype(dtype).itemsize].view(dtype)
        off += count * np.dtype(dtype).itemsize
        return a

    nc, real_depth = take(np.uint32, 2)
    nodes = take(np.uint32, 8 * nc).reshape(nc, 8)
    faces = take(np.uint32, 4 * mesh.face_count).reshape(-1, 4)
    R = cam.width * cam.height
    ids = take(np.uint32, R)
    depths = take(np.float32, R)
    coords = take(np.float32, 2 * R).reshape(R, 2)
    sk, si = take(np.uint32, keys.size), take(np.uint32, keys.size)

    ref = oracle.lbvh_build(mesh.vertices, mesh.faces, hit)
    assert nc == ref["info"]["node_count"] and real_depth == ref["info"]["real_depth"]
    assert np.array_equal(nodes, ref["nodes"].view(np.uint32))
    assert np.array_equal(faces, ref["faces"])
    o, d, _, _ = oracle.primary_rays(cam)
    e = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], o, d)
    hitm = e["id"] >= 0
    assert np.array_equal(ids.view(np.int32)[hitm], e["id"][hitm])
    assert np.all(ids[~hitm] == 0xFFFFFFFF)
    assert np.array_equal(depths.view(np.uint32), e["t"].view(np.uint32))
    assert np.array_equal(coords.view(np.uint32), e["uv"].view(np.uint32))
    ek, ev = oracle.sort_pairs(keys, None, 32, init_vals=True)
    assert np.array_equal(sk, ek) and np.array_equal(si, ev)

    for depth in (None, 8):  # buildMeshTreeSAH, buildMeshTreeHybrid(8)
        n2 = int(take(np.uint32, 1)[0])
        nodes2 = take(np.uint32, 8 * n2).reshape(n2, 8)
        faces2 = take(np.uint32, 4 * mesh.face_count).reshape(-1, 4)
        o2 = oracle.sah_build(mesh.vertices, mesh.faces, hit, hybrid_depth=depth)
        assert np.array_equal(nodes2, o2["nodes"].view(np.uint32))
        assert np.array_equal(faces2, o2["faces"])

    rid, rdep = take(np.uint32, R), take(np.float32, R)
    ruv = take(np.float32, 2 * R).reshape(R, 2)
    ang = oracle.camera_look_at(cam.center, cam.target)
    m = oracle.raster_matrix(cam.center, oracle.look_dir(cam.center, cam.target), np.array([ang[0], ang[1], 0], np.float32),
                             cam.fov, cam.ratio)
    fo, uo, do = oracle.rasterize(mesh.vertices, ref["faces"], m, cam.width, cam.height)
    assert np.array_equal(rdep.view(np.uint32), do.view(np.uint32))
    assert np.array_equal(ruv.view(np.uint32), uo.view(np.uint32))
    assert np.array_equal(rid, fo)
    if scene == "terrain":
        assert (do != oracle.HUGE).mean() > 0.1


def test_learned_proposal_from_cpp():
    """tests/cpp/test_learned.cpp: C++ host code trains the proposal network
    through the C ABI (features, tensor-core GEMMs, fused cross-entropy, Adam),
    proposes a slot per ray with rt_mlp_propose and traces with
    rt_trace_closest_seeded; the hits equal rt_trace_closest's bit for bit."""
    import __graft_entry__
    __graft_entry__.build_cpp_tests()
    exe = os.path.join(ROOT, "tests", "cpp", "_build", "test_learned")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "differing hits 0" in r.stdout, r.stdout
