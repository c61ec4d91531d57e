"""GPU parity: every stage of the CUDA path, called through the C ABI, against
the CPU oracle (which is pinned to the reference's own code) and the golden
fixtures. Integer/byte/index outputs and the pinned FP32 outputs are compared
bit for bit (tolerance: exact)."""
import os

import numpy as np
import pytest

from cudart_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def T():
    import torch
    assert torch.cuda.is_available()
    from cudart_b200 import core
    assert core.device_check()
    return torch


def _u32(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _dev(T, a):
    return T.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(t):
    return t.cpu().numpy()


def _build(T, mesh, **kw):
    from cudart_b200 import core
    v = _dev(T, mesh.vertices)
    f = _dev(T, mesh.faces.view(np.int32))
    tree = core.build_lbvh(v, f, **kw)
    T.cuda.synchronize()
    return v, f, tree


def _check_build(T, oracle, mesh, tree_depth=12, morton_bits=32, hitbox=None):
    v, f, tree = _build(T, mesh, tree_depth=tree_depth, morton_bits=morton_bits, hitbox=hitbox)
    ref = oracle.lbvh_build(mesh.vertices, mesh.faces, hitbox if hitbox is not None else oracle.hitbox(mesh.vertices),
                            tree_depth=tree_depth, layout=morton_bits)
    info = tree.info_host()
    for k in ("node_count", "leaf_count", "real_depth", "split_count", "overrun_visits", "nondet_reads", "past_end_reads"):
        assert info[k] == ref["info"][k], (k, info[k], ref["info"][k])
    assert info["error"] == 0
    nc = info["node_count"]
    assert np.array_equal(_u32(_host(tree.codes)), ref["codes"])
    assert np.array_equal(_u32(_host(tree.indices)), ref["indices"])
    assert np.array_equal(_u32(_host(tree.boxes)), _u32(ref["boxes"]))
    assert np.array_equal(_u32(_host(tree.nodes)[:nc]), _u32(ref["nodes"]))
    assert np.array_equal(_u32(_host(tree.faces)), _u32(ref["faces"]))
    assert np.array_equal(_u32(_host(tree.tris)), _u32(ref["tris"]))
    return v, f, tree, ref


# ----------------------------------------------------------------------------- sort
@pytest.mark.parametrize("n", [1, 2, 100, 4096, 4097, 100000, 1 << 20])
@pytest.mark.parametrize("bits", [8, 21, 32])
def test_sort_pairs_matches_oracle(T, oracle, n, bits):
    from cudart_b200 import core
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, 1 << min(bits, 31), n, dtype=np.int64).astype(np.uint32)
    if n > 10:
        keys[: n // 3] = keys[0]  # many ties
    k, v = _dev(T, keys.view(np.int32)), T.empty(n, dtype=T.int32, device="cuda")
    core.sort_pairs(k, v, bits, init_values=True)
    ek, ev = oracle.sort_pairs(keys, None, bits, init_vals=True)
    assert np.array_equal(_u32(_host(k)), ek)
    assert np.array_equal(_u32(_host(v)), ev)


def test_sort_keys_and_given_values(T, oracle):
    from cudart_b200 import core
    rng = np.random.default_rng(7)
    keys = rng.integers(0, 1 << 21, 1397121, dtype=np.int64).astype(np.uint32)  # samples/09_how_to_use_a_sorter.cpp:54
    vals = rng.integers(0, 1 << 30, keys.size, dtype=np.int64).astype(np.uint32)
    k = _dev(T, keys.view(np.int32))
    core.sort_keys(k, 21)
    assert np.array_equal(_u32(_host(k)), np.sort(keys))
    k, v = _dev(T, keys.view(np.int32)), _dev(T, vals.view(np.int32))
    core.sort_pairs(k, v, 32)
    ek, ev = oracle.sort_pairs(keys, vals, 32)
    assert np.array_equal(_u32(_host(k)), ek) and np.array_equal(_u32(_host(v)), ev)


# ----------------------------------------------------------------------------- build
def test_build_terrain_c0_matches_golden(T, oracle):
    g = np.load(os.path.join(GOLD, "terrain_c0.npz"))
    mesh, _ = scenes.terrain_small_scene()
    v, f, tree, ref = _check_build(T, oracle, mesh, hitbox=g["hitbox"])
    nc = tree.node_count
    assert np.array_equal(_u32(_host(tree.nodes)[:nc]), g["nodes"])
    assert np.array_equal(_u32(_host(tree.codes)), g["codes"])
    assert np.array_equal(_u32(_host(tree.faces)), g["faces"])
    assert tree.info_host()["overrun_visits"] > 0


@pytest.mark.parametrize("n", [1, 2, 15, 16, 17, 223, 224, 225, 511, 512, 513, 4096, 4097, 32768, 32769, 100000])
def test_build_soup_sizes(T, oracle, n):
    _check_build(T, oracle, scenes.soup(n, seed=1000 + n))


@pytest.mark.parametrize("depth", [1, 3, 7, 20, 31, 32])
def test_build_tree_depths(T, oracle, depth):
    _check_build(T, oracle, scenes.soup(20000, seed=11), tree_depth=depth)


def test_build_morton30_and_device_hitbox(T, oracle):
    mesh = scenes.soup(50000, seed=12)
    _check_build(T, oracle, mesh, morton_bits=30)
    _check_build(T, oracle, mesh, hitbox=None)


def test_build_degenerate_inputs(T, oracle):
    from tests.golden.make_golden import flat_z_mesh
    _, _, tree, _ = _check_build(T, oracle, flat_z_mesh())
    g = np.load(os.path.join(GOLD, "flatz.npz"))
    assert np.array_equal(_u32(_host(tree.nodes)[: tree.node_count]), g["nodes"])
    _check_build(T, oracle, scenes.soup(3000, seed=5, lo=(0.3, 0.3, 0.3), hi=(0.3, 0.3, 0.3), sigma=0.0))
    m = scenes.soup(500, seed=9)
    vv = m.vertices.copy()
    vv[1::3] = vv[0::3]
    _check_build(T, oracle, scenes.Mesh(vv, m.faces))


def test_build_terrain_large_overrun(T, oracle):
    _check_build(T, oracle, scenes.terrain(256, 4))


def test_build_in_place_faces(T, oracle):
    from cudart_b200 import core
    mesh = scenes.soup(30000, seed=3)
    v = _dev(T, mesh.vertices)
    f = _dev(T, mesh.faces.view(np.int32))
    tree = core.build_lbvh(v, f)
    tree2 = core.Tree(nodes=T.empty_like(tree.nodes), boxes=T.empty_like(tree.boxes), indices=T.empty_like(tree.indices),
                      codes=T.empty_like(tree.codes), faces=f, tris=T.empty_like(tree.tris), info=T.zeros_like(tree.info))
    core.build_lbvh(v, f, out=tree2)  # faces_out == faces_in: reordered in place, as the reference does
    T.cuda.synchronize()
    assert T.equal(tree2.faces, tree.faces) and T.equal(tree2.nodes[: tree.node_count], tree.nodes[: tree.node_count])


# ----------------------------------------------------------------------------- rays and traversal
def _rays(T, cam):
    from cudart_b200 import core
    c = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    o, d = core.primary_rays(c, cam.width, cam.height)
    T.cuda.synchronize()
    return o, d


@pytest.mark.parametrize("scene", ["terrain", "soup"])
def test_primary_rays_match_oracle(T, oracle, scene):
    cam = scenes.terrain_small_scene()[1] if scene == "terrain" else scenes.soup_1m_scene()[1]
    o, d = _rays(T, cam)
    eo, ed, _, _ = oracle.primary_rays(cam)
    assert np.array_equal(_u32(_host(o)), _u32(eo))
    assert np.array_equal(_u32(_host(d)), _u32(ed))


def test_batch_primary_rays_equal_per_camera(T):
    """rt_batch_primary_rays (all cameras in one launch) gives each camera's rays bit for bit as
    rt_primary_rays (which the oracle pins), for an image size that is no multiple of anything."""
    from cudart_b200 import core
    cams = [core.make_camera((0.1 * i, 0.5, -1.0 - i), (0.5, 0.4, 0.5), fov=0.9 + 0.1 * i, ratio=1.3) for i in range(5)]
    w, h = 37, 23
    o, d = core.batch_primary_rays(core.camera_bases(cams, w, h), w, h)
    T.cuda.synchronize()
    for i, c in enumerate(cams):
        po, pd = core.primary_rays(c, w, h)
        T.cuda.synchronize()
        sl = slice(i * w * h, (i + 1) * w * h)
        assert T.equal(o[sl].view(T.int32), po.view(T.int32)) and T.equal(d[sl].view(T.int32), pd.view(T.int32)), i


def _check_trace(T, oracle, tree, ref, o, d, tmax=None, id_mode=0, use_tris=True, vertices=None, sel=None):
    from cudart_b200 import core
    out = core.trace(tree, o, d, tmax=tmax, id_mode=id_mode, counters=True, use_tris=use_tris, vertices=vertices, use_accel=False)
    fast = core.trace(tree, o, d, tmax=tmax, id_mode=id_mode, use_tris=use_tris, vertices=vertices, use_accel=True)
    T.cuda.synchronize()
    # the traversal-blob path returns the same bits as the reference-node walk
    assert T.equal(fast["id"], out["id"]) and T.equal(fast["t"], out["t"]) and T.equal(fast["uv"], out["uv"])
    assert int(_host(fast["err"])[0]) == 0
    oo, dd = _host(o), _host(d)
    tm = None if tmax is None else _host(tmax)
    e = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], oo, dd, tm, mode=0, id_mode=id_mode, counters=True)
    assert int(_host(out["err"])[0]) == 0
    assert np.array_equal(_host(out["id"]), e["id"])
    assert np.array_equal(_u32(_host(out["t"])), _u32(e["t"]))
    assert np.array_equal(_u32(_host(out["uv"])), _u32(e["uv"]))
    assert np.array_equal(_u32(_host(out["visits"])), e["visits"])
    assert np.array_equal(_u32(_host(out["tests"])), e["tests"])
    return out, e


def test_trace_terrain_c0_matches_golden_and_oracle(T, oracle):
    g = np.load(os.path.join(GOLD, "terrain_c0.npz"))
    mesh, cam = scenes.terrain_small_scene()
    v, f, tree, ref = _check_build(T, oracle, mesh)
    o, d = _rays(T, cam)
    out, _ = _check_trace(T, oracle, tree, ref, o, d)
    sel = g["ray_sel"]
    assert np.array_equal(_host(out["id"])[sel], g["hit_id"])
    assert np.array_equal(_u32(_host(out["t"])[sel]), _u32(g["hit_t"]))
    assert np.array_equal(_u32(_host(out["uv"])[sel]), _u32(g["hit_uv"]))
    # reference data path (vertices + reordered faces, edges computed per test) gives the same bits
    _check_trace(T, oracle, tree, ref, o, d, use_tris=False, vertices=v)
    # original ids
    _check_trace(T, oracle, tree, ref, o, d, id_mode=1)


def test_trace_soup_incoherent(T, oracle):
    mesh = scenes.soup(200000, seed=21)
    v, f, tree, ref = _check_build(T, oracle, mesh)
    cam = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 320, 240)
    o, d = _rays(T, cam)
    out, e = _check_trace(T, oracle, tree, ref, o, d)
    assert (e["id"] >= 0).mean() > 0.95
    # bounce rays: bit-exact with the oracle, then traced
    from cudart_b200 import core
    bo, bd, bt = core.bounce_rays(tree.tris, o, d, out["id"], out["t"], 1234)
    T.cuda.synchronize()
    eo, ed, et = oracle.bounce_rays(ref["tris"], _host(o), _host(d), e["id"], e["t"], 1234)
    assert np.array_equal(_u32(_host(bo)), _u32(eo)) and np.array_equal(_u32(_host(bd)), _u32(ed))
    assert np.array_equal(_u32(_host(bt)), _u32(et))
    _check_trace(T, oracle, tree, ref, bo, bd, tmax=bt)


def test_trace_tmax_and_degenerate_rays(T, oracle):
    mesh = scenes.soup(20000, seed=22)
    v, f, tree, ref = _check_build(T, oracle, mesh)
    cam = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 64, 64)
    o, d = _rays(T, cam)
    dd = d.clone()
    dd[::7, 0] = 0.0  # exactly zero direction components
    dd[::11, 1] = 0.0
    dd[::13] = 0.0
    tm = T.full((o.shape[0],), 3.402823466e38, dtype=T.float32, device="cuda")
    tm[::5] = 0.3
    tm[::17] = 0.0
    tm[::19] = -1.0
    _check_trace(T, oracle, tree, ref, o, dd.contiguous(), tmax=tm)


def test_trace_matches_brute_force(T, oracle):
    mesh = scenes.soup(3000, seed=23)
    v, f, tree, ref = _check_build(T, oracle, mesh)
    cam = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 96, 64)
    o, d = _rays(T, cam)
    from cudart_b200 import core
    out = core.trace(tree, o, d)
    T.cuda.synchronize()
    bf = oracle.trace_brute(ref["tris"], _host(o), _host(d))
    assert np.array_equal(_host(out["id"]), bf["id"])
    assert np.array_equal(_u32(_host(out["t"])), _u32(bf["t"]))


def test_soup_1m_full_size(T, oracle):
    """The 2^20-triangle workload at full size: the whole build bit-exact, all
    1920x1080 primary rays bit-exact, a bounded sample of bounce rays bit-exact."""
    mesh, cam = scenes.soup_1m_scene()
    v, f, tree, ref = _check_build(T, oracle, mesh)
    o, d = _rays(T, cam)
    from cudart_b200 import core
    out = core.trace(tree, o, d)
    T.cuda.synchronize()
    oo, dd = _host(o), _host(d)
    e = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], oo, dd)
    assert np.array_equal(_host(out["id"]), e["id"])
    assert np.array_equal(_u32(_host(out["t"])), _u32(e["t"]))
    assert (e["id"] >= 0).mean() > 0.99
    bo, bd, bt = core.bounce_rays(tree.tris, o, d, out["id"], out["t"], 99)
    out2 = core.trace(tree, bo, bd, tmax=bt)
    T.cuda.synchronize()
    sel = np.arange(0, oo.shape[0], 37)
    eo, ed, et = oracle.bounce_rays(ref["tris"], oo, dd, e["id"], e["t"], 99)
    assert np.array_equal(_u32(_host(bo)), _u32(eo))
    e2 = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], np.ascontiguousarray(eo[sel]), np.ascontiguousarray(ed[sel]),
                      np.ascontiguousarray(et[sel]))
    assert np.array_equal(_host(out2["id"])[sel], e2["id"])
    assert np.array_equal(_u32(_host(out2["t"])[sel]), _u32(e2["t"]))


def test_trace_schedules_identical(T, oracle):
    """Every traversal schedule of the blob path returns the same bits."""
    from cudart_b200 import core, tune
    mesh = scenes.soup(100000, seed=31)
    v, f, tree, ref = _check_build(T, oracle, mesh)
    cam = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 200, 120)
    o, d = _rays(T, cam)
    base = core.trace(tree, o, d, use_accel=False)
    bo, bd, bt = core.bounce_rays(tree.tris, o, d, base["id"], base["t"], 5)
    base2 = core.trace(tree, bo, bd, tmax=bt, use_accel=False)
    for sch in tune.candidates(cam.width):
        out = core.trace(tree, o, d, schedule=sch)
        out2 = core.trace(tree, bo, bd, tmax=bt, schedule=sch)
        T.cuda.synchronize()
        assert int(_host(out["err"])[0]) == 0, sch
        for a, b in ((out, base), (out2, base2)):
            assert T.equal(a["id"], b["id"]) and T.equal(a["t"], b["t"]) and T.equal(a["uv"], b["uv"]), sch


@pytest.mark.parametrize("wide", [False, True])
def test_coop_counters_follow_the_ray(T, oracle, wide):
    """The cooperative schedules count each ray's own box reads and triangle
    tests, whichever lanes ran them: persistent warps (with and without ray
    sorting, so other warp compositions) give every ray the counts of the
    one-launch-slot-per-ray schedule."""
    from cudart_b200 import core
    mesh = scenes.soup(60000, seed=32)
    v, f, tree, ref = _check_build(T, oracle, mesh)
    cam = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 160, 96)
    o, d = _rays(T, cam)
    h = core.trace(tree, o, d)
    bo, bd, bt = core.bounce_rays(tree.tris, o, d, h["id"], h["t"], 9)
    base = core.trace(tree, bo, bd, tmax=bt, counters=True, schedule=dict(coop=True, wide=wide))
    for sch in (dict(coop=True, persistent=True, blocks_per_sm=2, wide=wide),
                dict(coop=True, persistent=True, blocks_per_sm=8, sorted=True, while_while=True, wide=wide)):
        out = core.trace(tree, bo, bd, tmax=bt, counters=True, schedule=sch)
        T.cuda.synchronize()
        assert T.equal(out["id"], base["id"]) and T.equal(out["t"], base["t"]), sch
        assert T.equal(out["visits"], base["visits"]) and T.equal(out["tests"], base["tests"]), sch
    assert int(base["tests"].sum()) > 0


@pytest.mark.parametrize("attrs", [False, True])
def test_interpolate_matches_oracle(T, oracle, attrs):
    from cudart_b200 import core
    mesh, cam = scenes.terrain_small_scene(256, 160)
    v, f, tree, ref = _check_build(T, oracle, mesh)
    o, d = _rays(T, cam)
    hits = core.trace(tree, o, d)
    rng = np.random.default_rng(2)
    V = mesh.vertex_count
    nrm = rng.normal(size=(V, 4)).astype(np.float32) if attrs else None
    col = rng.uniform(size=(V, 4)).astype(np.float32) if attrs else None
    tex = rng.uniform(size=(V, 2)).astype(np.float32) if attrs else None
    out = core.interpolate(tree, v, hits, *(None if a is None else _dev(T, a) for a in (nrm, col, tex)))
    T.cuda.synchronize()
    e = oracle.interpolate(_host(hits["id"]), _host(hits["uv"]), ref["faces"], mesh.vertices, nrm, col, tex)
    for k in ("points", "normals", "colors", "texcoords", "materials"):
        assert np.array_equal(_u32(_host(out[k])), _u32(e[k])), k


def test_file_round_trip_device(T, oracle, tmp_path):
    """quickSave/quickLoad-format files from and into device buffers."""
    from cudart_b200 import core
    mesh = scenes.soup(20000, seed=51)
    v, f, tree, ref = _check_build(T, oracle, mesh)
    hb = oracle.hitbox(mesh.vertices)
    path = str(tmp_path / "scene.bin")
    core.mesh_save(path, v, f, hb)
    core.tree_save(path, tree, overwrite=False)
    m = core.mesh_load(path)
    t = core.tree_load(path)
    assert np.array_equal(np.array(m["hitbox"], np.float32), hb)
    assert T.equal(m["vertices"], v) and T.equal(m["faces"], f)
    nc = tree.node_count
    assert T.equal(t["nodes"], tree.nodes[:nc]) and T.equal(t["indices"], tree.indices) and T.equal(t["boxes"], tree.boxes)


def test_batch_build_and_trace_match_single_mesh(T, oracle):
    """Every mesh of a batched build equals its single-mesh build bit for bit,
    and one batched trace launch equals the per-mesh traces."""
    from cudart_b200 import core
    meshes = [scenes.soup(1, seed=1), scenes.soup(17, seed=2), scenes.terrain(9, 3), scenes.soup(224, seed=4),
              scenes.soup(5000, seed=5), scenes.terrain(64, 6), scenes.soup(33000, seed=7), scenes.soup(2, seed=8)]
    verts, faces, fo, vo = scenes.concat_batch(meshes)
    bt = core.batch_build(_dev(T, verts), _dev(T, faces.view(np.int32)), fo, vo)
    rays = [scenes.sphere_rays(m, 24 + 8 * i, seed=100 + i) for i, m in enumerate(meshes)]
    ro = [0]
    for o, _ in rays:
        ro.append(ro[-1] + len(o))
    O = _dev(T, np.concatenate([o for o, _ in rays]))
    D = _dev(T, np.concatenate([d for _, d in rays]))
    hits = core.batch_trace(bt, O, D, T.tensor(ro, dtype=T.int32, device="cuda"))
    T.cuda.synchronize()
    info = _host(bt.info)
    assert np.all(info[:, 7] == 0), info
    for m, mesh in enumerate(meshes):
        v, f, tree = _build(T, mesh)
        nc = tree.node_count
        assert int(info[m, 0]) == nc
        F0, F1 = fo[m], fo[m + 1]
        assert T.equal(bt.mesh_nodes(m, nc), tree.nodes[:nc]), m
        assert T.equal(bt.indices[F0:F1], tree.indices), m
        assert T.equal(bt.codes[F0:F1], tree.codes), m
        assert T.equal(bt.faces[F0:F1], tree.faces), m
        assert T.equal(bt.tris[F0:F1], tree.tris), m
        assert T.equal(bt.boxes[F0:F1], tree.boxes), m
        single = core.trace(tree, _dev(T, rays[m][0]), _dev(T, rays[m][1]))
        T.cuda.synchronize()
        sl = slice(ro[m], ro[m + 1])
        assert T.equal(hits["id"][sl], single["id"]) and T.equal(hits["t"][sl], single["t"]) and T.equal(hits["uv"][sl], single["uv"]), m
    assert int(_host(hits["err"])[0]) == 0
    # every schedule of the batched traversal (4-wide records, persistent warps) returns the same bits
    from cudart_b200 import tune
    roff = T.tensor(ro, dtype=T.int32, device="cuda")
    for sch in tune.batch_candidates():
        h = core.batch_trace(bt, O, D, roff, schedule=sch)
        T.cuda.synchronize()
        assert int(_host(h["err"])[0]) == 0, sch
        assert T.equal(h["id"], hits["id"]) and T.equal(h["t"], hits["t"]) and T.equal(h["uv"], hits["uv"]), sch


def test_ray_order_puts_inactive_rays_last(T):
    """rt_ray_order returns a permutation of the rays with the active ones grouped by direction octant
    (ascending) and the inactive ones (tmax <= 0) strictly last, also beside an octant-7 ray whose origin is
    the box's max corner, the largest key an active ray can have."""
    from cudart_b200 import core
    rng = np.random.default_rng(12)
    R = 5000
    o = np.zeros((R, 4), np.float32)
    d = np.zeros((R, 4), np.float32)
    o[:, :3] = rng.uniform(0.0, 1.0, (R, 3))
    d[:, :3] = rng.normal(size=(R, 3))
    tmax = np.full(R, 3.0e38, np.float32)
    tmax[::3] = -1.0
    tmax[7::11] = 0.0
    for r in (5, 17, 4999):  # active, octant 7, origin at the max corner
        o[r, :3] = 1.0
        d[r, :3] = -1.0
        tmax[r] = 3.0e38
    tmax[6] = tmax[18] = -1.0
    order = _host(core.ray_order(_dev(T, o), _dev(T, d), _dev(T, tmax), [0.0, 0.0, 0.0, 1.0, 1.0, 1.0])).astype(np.int64)
    assert np.array_equal(np.sort(order), np.arange(R))
    active = tmax[order] > 0
    n_act = int((tmax > 0).sum())
    assert active[:n_act].all() and not active[n_act:].any()
    dd = d[order[:n_act]]
    oct_ = (dd[:, 0] < 0).astype(int) | 2 * (dd[:, 1] < 0) | 4 * (dd[:, 2] < 0)
    assert np.all(np.diff(oct_) >= 0)


@pytest.mark.parametrize("R", [1, 7, 2047, 2048, 2049, 100003])
def test_pack_hits_round_trip(T, R):
    """rt_pack_hits keeps the (t, u, v) of exactly the rays that hit, in ray order (blocks of 2048 rays and
    partial last blocks), and the ids plus the packed hits rebuild every hit bit for bit."""
    from cudart_b200 import core
    rng = np.random.default_rng(R)
    ids = rng.integers(-1, 5, R).astype(np.int32)
    ids[rng.random(R) < 0.6] = -1
    t = rng.uniform(0.0, 10.0, R).astype(np.float32)
    tmax = rng.uniform(0.0, 10.0, R).astype(np.float32)
    t[ids < 0] = tmax[ids < 0]
    uv = rng.uniform(0.0, 1.0, (R, 2)).astype(np.float32)
    uv[ids < 0] = 0.0
    h = dict(id=_dev(T, ids), t=_dev(T, t), uv=_dev(T, uv))
    p = core.pack_hits(h)
    T.cuda.synchronize()
    n = int(_host(p["count"])[0])
    hit = ids >= 0
    assert n == int(hit.sum())
    packed = _host(p["packed"])[:3 * n].reshape(n, 3)
    assert np.array_equal(_u32(packed[:, 0]), _u32(t[hit]))
    assert np.array_equal(_u32(packed[:, 1:]), _u32(uv[hit]))
    t2, uv2 = core.unpack_hits(T.from_numpy(ids), T.from_numpy(_host(p["packed"])), n, tmax=T.from_numpy(tmax))
    assert np.array_equal(_u32(t2.numpy()), _u32(t)) and np.array_equal(_u32(uv2.numpy()), _u32(uv))
    q = core.pack_hits(h, out=p)  # the same outputs again, in place
    T.cuda.synchronize()
    assert int(_host(q["count"])[0]) == n
