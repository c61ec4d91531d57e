"""SAH / Hybrid builder oracle (oracle/rt_oracle.cpp or_sah_build) pinned to the
reference's own SAH kernels (kernels/CUDA_buildMeshTreeSAH.cu:224-666, run as
emulated 32-thread blocks one after another by oracle/build_ref.sh):
bit-exact nodes (internal nodes compared on bits 0-2 of their first word, the
only bits the reference sets) and indices. Against the committed fixtures
always; against the reference code itself when the reference tree is here."""
import os

import numpy as np
import pytest

from cudart_b200 import scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _masked(nodes):
    w = np.ascontiguousarray(nodes).view(np.uint32).copy()
    internal = (w[:, 0] & 1) == 0
    w[internal, 0] &= 7
    return w


def _golden_cases():
    return {"terrain": (scenes.terrain(64, 2), None), "soup": (scenes.soup(5000, 4), None), "hybrid": (scenes.terrain(64, 2), 4)}


@pytest.mark.parametrize("name", ["terrain", "soup", "hybrid"])
def test_sah_matches_golden(oracle, name):
    g = np.load(os.path.join(GOLD, "sah.npz"))
    m, depth = _golden_cases()[name]
    o = oracle.sah_build(m.vertices, m.faces, hybrid_depth=depth)
    assert np.array_equal(o["indices"], g[f"indices_{name}"])
    assert np.array_equal(_masked(o["nodes"]), g[f"nodes_{name}"])
    assert o["no_split"] == 0


def test_sah_tree_invariants(oracle):
    m = scenes.soup(20000, 8)
    o = oracle.sah_build(m.vertices, m.faces)
    w = o["nodes"].view(np.uint32)
    n = len(m.faces)
    leaf = (w[:, 0] & 1) == 1
    counts = w[leaf, 0] >> 1
    firsts = w[leaf, 1]
    order = np.argsort(firsts)
    assert firsts[order][0] == 0 and np.array_equal(firsts[order][1:], (firsts + counts)[order][:-1])
    assert int(counts.sum()) == n
    assert (counts >= 1).all() and (counts <= 224).all()
    assert np.array_equal(np.sort(o["indices"]), np.arange(n, dtype=np.uint32))
    assert 2 * leaf.sum() - 1 == len(w)
    # children ids: the k-th split in pre-order gets 2k + 1, 2k + 2
    internal = np.nonzero(~leaf)[0]
    assert np.array_equal(np.sort(w[internal, 1]), np.arange(1, len(w), 2, dtype=np.uint32))


def test_sah_no_usable_boundary_makes_a_leaf(oracle):
    """300 copies of one triangle: every centroid falls in one bin, so no bin
    boundary separates two non-empty sides. The reference never terminates
    there (it splits off an empty left child forever); the contract makes a leaf."""
    t = scenes.soup(1, 3)
    v = np.tile(t.vertices, (300, 1))
    f = np.zeros((300, 4), np.uint32)
    f[:, :3] = (np.arange(300)[:, None] * 3 + np.arange(3)).astype(np.uint32)
    o = oracle.sah_build(v, f)
    w = o["nodes"].view(np.uint32)
    assert len(w) == 1 and (w[0, 0] & 1) and (w[0, 0] >> 1) == 300
    assert o["no_split"] == 1


_ref = pytest.mark.skipif(not __import__("oracle.api", fromlist=["x"]).ref_available(), reason="reference tree not present")


def _ref_sah(oracle, m, depth=None):
    hit = oracle.hitbox(m.vertices)
    boxes, idx = oracle.ref_mesh_boxes(m.vertices, m.faces)
    if depth is None:
        return oracle.ref_sah_build(boxes, hit, idx)
    lb = oracle.ref_lbvh_build(boxes, hit, tree_depth=depth, tree_complete=False)
    return oracle.ref_sah_build(boxes, hit, lb["indices"], nodes_in=lb["nodes"])


@_ref
@pytest.mark.parametrize("case", ["soup17", "soup224", "soup225", "soup2000", "terrain32", "terrain64-hyb1", "terrain64-hyb6",
                                  "soup3000-hyb12", "clustered"])
def test_sah_matches_reference_code(oracle, case):
    depth = None
    if case.startswith("soup") and "hyb" not in case:
        m = scenes.soup(int(case[4:]), 11)
    elif case == "terrain32":
        m = scenes.terrain(32, 5)
    elif case.startswith("terrain64"):
        m, depth = scenes.terrain(64, 6), int(case.split("hyb")[1])
    elif case == "soup3000-hyb12":
        m, depth = scenes.soup(3000, 12), 12
    else:  # two tight clusters far apart plus a sparse band: lopsided splits
        a = scenes.soup(1500, 1, lo=(0, 0, 0), hi=(0.01, 0.01, 0.01), sigma=0.001)
        b = scenes.soup(1500, 2, lo=(5, 5, 5), hi=(5.01, 5.01, 5.01), sigma=0.001)
        c = scenes.soup(300, 3, lo=(0, 0, 0), hi=(5, 0.1, 0.1))
        m = scenes.concat(a, b, c)
    st, nodes, idx = _ref_sah(oracle, m, depth)
    assert st == 0
    o = oracle.sah_build(m.vertices, m.faces, hybrid_depth=depth)
    assert np.array_equal(idx, o["indices"])
    assert np.array_equal(_masked(nodes), _masked(o["nodes"]))


@_ref
def test_reference_does_not_terminate_without_a_boundary(oracle):
    t = scenes.soup(1, 3)
    v = np.tile(t.vertices, (300, 1))
    f = np.zeros((300, 4), np.uint32)
    f[:, :3] = (np.arange(300)[:, None] * 3 + np.arange(3)).astype(np.uint32)
    hit = oracle.hitbox(v)
    boxes, idx = oracle.ref_mesh_boxes(v, f)
    st, _, _ = oracle.ref_sah_build(boxes, hit, idx, capacity=64)
    assert st == 2  # node capacity runs out: the reference keeps splitting off empty children
