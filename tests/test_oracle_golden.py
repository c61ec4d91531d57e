"""The CPU oracle against the golden fixtures produced by the reference's own
code (tests/golden/make_golden.py). Runs without the reference tree."""
import hashlib
import os

import numpy as np
import pytest

from cudart_b200 import scenes

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _u32(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_terrain_c0_build_matches_golden(oracle):
    g = np.load(os.path.join(GOLD, "terrain_c0.npz"))
    mesh, cam = scenes.terrain_small_scene()
    hit = oracle.hitbox(mesh.vertices)
    assert np.array_equal(_u32(hit), _u32(g["hitbox"]))
    boxes, _ = oracle.mesh_boxes(mesh.vertices, mesh.faces)
    assert hashlib.sha256(boxes.tobytes()).digest() == g["boxes_sha256"].tobytes()
    r = oracle.lbvh_build(mesh.vertices, mesh.faces, hit)
    assert np.array_equal(r["codes"], g["codes"])
    assert np.array_equal(r["indices"], g["indices"])
    assert np.array_equal(_u32(r["nodes"]), g["nodes"])
    assert np.array_equal(r["faces"], g["faces"])
    assert r["info"]["real_depth"] == int(g["real_depth"])
    assert r["info"]["split_count"] == int(g["split_count"])


def test_terrain_c0_rays_and_hits_match_golden(oracle):
    g = np.load(os.path.join(GOLD, "terrain_c0.npz"))
    mesh, cam = scenes.terrain_small_scene()
    o, d, basis, ang = oracle.primary_rays(cam)
    assert np.array_equal(_u32(basis), _u32(g["basis"]))
    assert np.array_equal(_u32(ang), _u32(g["angle"]))
    assert hashlib.sha256(d.tobytes()).digest() == g["dirs_sha256"].tobytes()
    r = oracle.lbvh_build(mesh.vertices, mesh.faces)
    sel = g["ray_sel"]
    tr = oracle.trace(r["nodes"], r["tris"], r["indices"], np.ascontiguousarray(o[sel]), np.ascontiguousarray(d[sel]))
    assert np.array_equal(tr["id"], g["hit_id"])
    assert np.array_equal(_u32(tr["t"]), _u32(g["hit_t"]))
    assert np.array_equal(_u32(tr["uv"]), _u32(g["hit_uv"]))


@pytest.mark.parametrize("n", [1, 16, 17, 224, 225, 513, 5000])
def test_soup_nodes_match_golden(oracle, n):
    g = np.load(os.path.join(GOLD, "soup_small.npz"))
    m = scenes.soup(n, seed=n)
    r = oracle.lbvh_build(m.vertices, m.faces)
    assert np.array_equal(_u32(r["nodes"]), g[f"nodes_{n}"])
    assert np.array_equal(r["indices"], g[f"indices_{n}"])


def test_flat_z_quirk_matches_golden(oracle):
    from tests.golden.make_golden import flat_z_mesh
    g = np.load(os.path.join(GOLD, "flatz.npz"))
    m = flat_z_mesh()
    r = oracle.lbvh_build(m.vertices, m.faces)
    nodes = _u32(r["nodes"])
    assert np.array_equal(nodes, g["nodes"])
    # every internal node keeps the inverted initial box (z extent of the leaves is 0)
    internal = (nodes[:, 0] & 1) == 0
    assert internal.any()
    assert np.all(r["nodes"][internal, 2:5] == np.float32(3.402823466e38))
