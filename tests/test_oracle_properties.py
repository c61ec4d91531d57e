"""Structural properties of the oracle's outputs (no reference needed)."""
import numpy as np
import pytest

from cudart_b200 import scenes


def test_sort_is_stable_permutation(oracle):
    rng = np.random.default_rng(0)
    keys = rng.integers(0, 64, 10000).astype(np.uint32)
    k, v = oracle.sort_pairs(keys, None, 32, init_vals=True)
    assert np.all(k[1:] >= k[:-1])
    assert np.array_equal(np.sort(v), np.arange(10000))
    expect = np.argsort(keys, kind="stable")
    assert np.array_equal(v, expect)


def test_sort_bit_depth_uses_low_bytes(oracle):
    keys = np.array([0x100, 0x1, 0x200, 0x0], np.uint32)
    k, v = oracle.sort_pairs(keys, None, 8, init_vals=True)  # one byte: high bits ignored, stable
    assert list(v) == [0, 2, 3, 1]


@pytest.mark.parametrize("n", [17, 1000, 40000])
def test_tree_invariants(oracle, n):
    m = scenes.soup(n, seed=n)
    r = oracle.lbvh_build(m.vertices, m.faces)
    nodes = np.ascontiguousarray(r["nodes"]).view(np.uint32)
    nc = len(nodes)
    assert nc == 2 * r["info"]["leaf_count"] - 1
    leaf = (nodes[:, 0] & 1) == 1
    first, cnt = nodes[leaf, 1], nodes[leaf, 0] >> 1
    order = np.argsort(first)
    assert first[order][0] == 0
    assert np.array_equal(first[order][1:], (first + cnt)[order][:-1])  # disjoint, covering
    assert (first + cnt).max() == n
    ch = nodes[~leaf, 1]
    assert np.all(ch + 1 < nc) and np.all(ch % 2 == 1)
    boxes = r["nodes"][:, 2:8]
    for k in np.nonzero(~leaf)[0]:
        c = nodes[k, 1]
        assert np.array_equal(boxes[k, :3], np.minimum(boxes[c, :3], boxes[c + 1, :3]))
        assert np.array_equal(boxes[k, 3:], np.maximum(boxes[c, 3:], boxes[c + 1, 3:]))


def test_traversal_equals_brute_force(oracle):
    m = scenes.soup(3000, seed=3)
    cam = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 64, 64)
    r = oracle.lbvh_build(m.vertices, m.faces)
    o, d, _, _ = oracle.primary_rays(cam)
    tr = oracle.trace(r["nodes"], r["tris"], r["indices"], o, d)
    bf = oracle.trace_brute(r["tris"], o, d)
    assert np.array_equal(tr["id"], bf["id"])
    assert np.array_equal(tr["t"].view(np.uint32), bf["t"].view(np.uint32))
    orig_ids = oracle.trace(r["nodes"], r["tris"], r["indices"], o, d, id_mode=1)["id"]
    hit = tr["id"] >= 0
    assert np.array_equal(orig_ids[hit], r["indices"][tr["id"][hit]])


def test_bounce_rays_deterministic_and_unit(oracle):
    m = scenes.soup(5000, seed=4)
    cam = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 48, 32)
    r = oracle.lbvh_build(m.vertices, m.faces)
    o, d, _, _ = oracle.primary_rays(cam)
    tr = oracle.trace(r["nodes"], r["tris"], r["indices"], o, d)
    a = oracle.bounce_rays(r["tris"], o, d, tr["id"], tr["t"], 1234)
    b = oracle.bounce_rays(r["tris"], o, d, tr["id"], tr["t"], 1234)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    hit = tr["id"] >= 0
    lens = np.linalg.norm(a[1][hit, :3], axis=1)
    assert np.allclose(lens, 1.0, atol=1e-5)
    assert np.all(a[2][~hit] == -1.0)
