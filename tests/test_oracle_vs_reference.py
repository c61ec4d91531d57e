"""The CPU oracle against the reference's own functions compiled from its
sources (oracle/_ref, built by oracle/build_ref.sh). Skipped when the checker
library is absent."""
import numpy as np
import pytest

from cudart_b200 import scenes

pytestmark = pytest.mark.skipif(not __import__("oracle.api", fromlist=["x"]).ref_available(),
                                reason="reference checker (oracle/_ref) not built")


def _u32(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _check(oracle, mesh, cam=None, depth=12):
    v, f = mesh.vertices, mesh.faces
    hit = oracle.hitbox(v)
    b, idx = oracle.mesh_boxes(v, f)
    rb, ridx = oracle.ref_mesh_boxes(v, f)
    assert np.array_equal(_u32(b), _u32(rb)) and np.array_equal(idx, ridx)
    res = oracle.lbvh_build(v, f, hit, tree_depth=depth)
    ref = oracle.ref_lbvh_build(b, hit, tree_depth=depth)
    assert np.array_equal(res["codes"], ref["codes"])
    assert np.array_equal(res["indices"], ref["indices"])
    assert np.array_equal(_u32(res["nodes"]), _u32(ref["nodes"]))
    assert res["info"]["real_depth"] == ref["real_depth"]
    assert np.array_equal(res["faces"], oracle.ref_reorder_faces(f, res["indices"]))
    if cam is not None:
        o, d, basis, ang = oracle.primary_rays(cam)
        ro, rd, rbasis, rang = oracle.ref_camera_rays(cam)
        assert np.array_equal(_u32(d), _u32(rd)) and np.array_equal(_u32(o), _u32(ro))
        ref_mode = oracle.trace(res["nodes"], res["tris"], res["indices"], o, d, mode=1)
        contract = oracle.trace(res["nodes"], res["tris"], res["indices"], o, d, mode=0)
        rt = oracle.ref_trace(res["nodes"], v, res["faces"], o, d, cam.width, cam.height)
        hm = rt["t"] != oracle.HUGE
        # the oracle's reference-semantics mode reproduces the reference kernel
        assert np.array_equal(_u32(ref_mode["t"]), _u32(rt["t"]))
        assert np.array_equal(ref_mode["id"][hm], rt["id"][hm].astype(np.int32))
        assert np.array_equal(_u32(ref_mode["uv"][hm]), _u32(rt["uv"][hm]))
        # this build's (t, position) contract agrees with it on these scenes
        assert np.array_equal(contract["id"] < 0, ~hm)
        assert np.array_equal(contract["id"][hm], rt["id"][hm].astype(np.int32))
        assert np.array_equal(_u32(contract["t"]), _u32(rt["t"]))
    return res


CAM = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 64, 48)


@pytest.mark.parametrize("n", [1, 2, 15, 16, 17, 223, 224, 225, 511, 512, 513, 1000, 32768, 32769])
def test_soup_sizes(oracle, n):
    _check(oracle, scenes.soup(n, seed=1000 + n), CAM if n <= 5000 else None)


def test_terrain_c0(oracle):
    mesh, cam = scenes.terrain_small_scene(128, 128)
    r = _check(oracle, mesh, cam)
    assert r["info"]["overrun_visits"] > 0  # the split-pointer overrun path is exercised


@pytest.mark.parametrize("depth", [1, 3, 7, 20, 31])
def test_tree_depths(oracle, depth):
    _check(oracle, scenes.soup(20000, seed=11), None, depth=depth)


def test_degenerate_inputs(oracle):
    _check(oracle, scenes.soup(3000, seed=5, lo=(0.3, 0.3, 0.3), hi=(0.3, 0.3, 0.3), sigma=0.0))  # all centroids equal
    m = scenes.terrain(32, 3)
    v = m.vertices.copy()
    v[:, [1, 2]] = v[:, [2, 1]]
    v[:, 2] = 0.5
    _check(oracle, scenes.Mesh(v, m.faces), scenes.Camera((0, 0, -2), (0, 0, 0.5), scenes.FOV_60, 32, 32))  # flat z
    m = scenes.soup(500, seed=9)
    v = m.vertices.copy()
    v[1::3] = v[0::3]  # collinear / degenerate triangles (two equal vertices)
    _check(oracle, scenes.Mesh(v, m.faces), CAM)


def test_interpolation_matches_reference(oracle):
    """kernels/CUDA_interpolateData.cu:45-138 (compiled from the reference) vs the
    oracle, with and without per-vertex normals / colors / texcoords."""
    mesh, cam = scenes.terrain_small_scene(96, 64)
    res = oracle.lbvh_build(mesh.vertices, mesh.faces)
    o, d, _, _ = oracle.primary_rays(cam)
    tr = oracle.trace(res["nodes"], res["tris"], res["indices"], o, d)
    hit = tr["id"] >= 0
    assert hit.any()
    ids = np.where(hit, tr["id"], 0).astype(np.int32)  # the reference reads some face on a miss; compare hits only
    rng = np.random.default_rng(1)
    V = mesh.vertex_count
    normals = rng.normal(size=(V, 4)).astype(np.float32)
    normals[:, 3] = 0
    colors = rng.uniform(size=(V, 4)).astype(np.float32)
    texc = rng.uniform(size=(V, 2)).astype(np.float32)
    for attrs in ((None, None, None), (normals, colors, texc)):
        e = oracle.interpolate(ids, tr["uv"], res["faces"], mesh.vertices, *attrs)
        r = oracle.ref_interpolate(ids.view(np.uint32), tr["uv"], cam.width, cam.height, res["faces"], mesh.vertices, *attrs)
        for k in ("points", "normals", "colors", "texcoords", "materials"):
            assert np.array_equal(_u32(e[k][hit]), _u32(r[k][hit])), k
