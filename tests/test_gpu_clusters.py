"""The cluster tree (RT_ACCEL_CLUSTERS build, RT_TRACE_CLUSTERS walks) against
the oracle: every walk of the cluster tree returns the closest hit bit for bit
(id, t, u, v) as the oracle's restatement of the reference traversal, for mesh
sizes from one face (a single cluster) through a few records to hundreds of
thousands of faces, every leaf size, meshes whose Morton codes are all equal
or run in long ties, degenerate rays and tmax cut-offs, face-id output,
counters, ray orders and batched meshes of mixed sizes. A blob built without
the cluster tree reports RT_DEVERR_ACCEL_MISSING and misses instead of reading
stale records."""
import numpy as np
import pytest

from cudart_b200 import scenes

pytestmark = pytest.mark.gpu

CLUSTER_SCHEDULES = [
    dict(clusters=True),                                                    # per-lane, one thread per ray
    dict(clusters=True, while_while=True),                                  # per-lane, descend-then-test
    dict(clusters=True, persistent=True, blocks_per_sm=8),                   # per-lane, persistent warps
    dict(clusters=True, persistent=True, blocks_per_sm=8, while_while=True, sorted=True),
    dict(clusters=True, persistent=True, blocks_per_sm=16, coop=True),       # warp-cooperative cluster tests
    dict(clusters=True, persistent=True, blocks_per_sm=16, coop=True, sorted=True),
    dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True),     # warp packets
    dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True, sorted=True),
    dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True, lane_threshold=16, sorted=True),  # packet, then per lane
    dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True, lane_threshold=32),
    dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, lane_threshold=16),  # warps refill idle lanes
    dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, lane_threshold=1, sorted=True),
    dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, lane_threshold=8, while_while=True),
]


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


def _build(T, oracle, mesh, clusters=True, cluster_leaf=0):
    from cudart_b200 import core
    v = _dev(T, mesh.vertices)
    f = _dev(T, mesh.faces.view(np.int32))
    tree = core.build_lbvh(v, f, clusters=clusters, cluster_leaf=cluster_leaf)
    T.cuda.synchronize()
    ref = oracle.lbvh_build(mesh.vertices, mesh.faces, oracle.hitbox(mesh.vertices))
    assert np.array_equal(_u32(_host(tree.tris)), _u32(ref["tris"]))
    return tree, ref


def _expect(oracle, ref, o, d, tmax=None, id_mode=0):
    return oracle.trace(ref["nodes"], ref["tris"], ref["indices"], _host(o), _host(d), None if tmax is None else _host(tmax),
                        mode=0, id_mode=id_mode)


def _same(T, out, e):
    assert int(_host(out["err"])[0]) == 0
    assert np.array_equal(_host(out["id"]), e["id"])
    assert np.array_equal(_u32(_host(out["t"])), _u32(e["t"]))
    assert np.array_equal(_u32(_host(out["uv"])), _u32(e["uv"]))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 15, 16, 17, 63, 64, 65, 255, 256, 257, 1023, 1024, 1025, 4095, 4097, 65537, 300001])
def test_cluster_walks_match_oracle(T, oracle, n):
    from cudart_b200 import core
    mesh = scenes.soup(n, seed=500 + n)
    tree, ref = _build(T, oracle, mesh)
    o, d = (_dev(T, a) for a in scenes.sphere_rays(mesh, 48, seed=n))
    e = _expect(oracle, ref, o, d)
    if n >= 64:
        assert (e["id"] >= 0).any()
    for sch in CLUSTER_SCHEDULES:
        out = core.trace(tree, o, d, schedule=sch)
        T.cuda.synchronize()
        _same(T, out, e)


@pytest.mark.parametrize("leaf", [1, 2, 3, 8])
def test_cluster_leaf_sizes(T, oracle, leaf):
    from cudart_b200 import core
    mesh = scenes.soup(20000, seed=41)
    tree, ref = _build(T, oracle, mesh, cluster_leaf=leaf)
    o, d = (_dev(T, a) for a in scenes.sphere_rays(mesh, 64, seed=leaf))
    e = _expect(oracle, ref, o, d)
    for sch in CLUSTER_SCHEDULES:
        _same(T, core.trace(tree, o, d, schedule=sch), e)


def test_cluster_tree_of_identical_triangles(T, oracle):
    """Every triangle the same (all Morton codes equal: the keys differ only by position) and a mesh whose
    triangles shrink geometrically towards one corner (long runs of equal codes beside distinct ones)."""
    from cudart_b200 import core
    n = 5000
    tri = np.array([[0.1, 0.2, 0.3, 0.0], [0.9, 0.25, 0.35, 0.0], [0.5, 0.8, 0.3, 0.0]], np.float32)
    same = scenes.Mesh(np.tile(tri, (n, 1)).astype(np.float32), np.stack([np.arange(n) * 3, np.arange(n) * 3 + 1, np.arange(n) * 3 + 2,
                                                                           np.zeros(n, np.int64)], 1).astype(np.uint32))
    k = np.arange(n) % 40
    sc = (0.5 ** k).astype(np.float32)[:, None]
    geo = scenes.Mesh(np.concatenate([(tri[None, :, :3] * sc[:, :, None]).reshape(-1, 3), np.zeros((3 * n, 1), np.float32)], 1)
                      .astype(np.float32), same.faces)
    for mesh in (same, geo):
        tree, ref = _build(T, oracle, mesh)
        o, d = (_dev(T, a) for a in scenes.sphere_rays(mesh, 40, seed=9))
        e = _expect(oracle, ref, o, d)
        for sch in CLUSTER_SCHEDULES:
            _same(T, core.trace(tree, o, d, schedule=sch), e)


def test_cluster_walks_camera_tmax_degenerate_and_ids(T, oracle):
    """Primary rays of a camera (coherent) and bounce rays (incoherent, with tmax), zero direction
    components, tmax = 0 / negative / short, and original face ids."""
    from cudart_b200 import core
    mesh = scenes.soup(200000, seed=21)
    tree, ref = _build(T, oracle, mesh)
    cam = scenes.Camera((0.5, 0.5, -0.4), (0.5, 0.5, 0.5), scenes.FOV_60, 160, 120)
    c = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    o, d = core.primary_rays(c, cam.width, cam.height)
    dd = d.clone()
    dd[::7, 0] = 0.0
    dd[::11, 1] = 0.0
    dd[::13] = 0.0
    dd = dd.contiguous()
    tm = T.full((o.shape[0],), 3.402823466e38, dtype=T.float32, device="cuda")
    tm[::5] = 0.3
    tm[::17] = 0.0
    tm[::19] = -1.0
    e = _expect(oracle, ref, o, dd, tm)
    e1 = _expect(oracle, ref, o, d, id_mode=1)
    base = core.trace(tree, o, d)
    bo, bd, bt = core.bounce_rays(tree.tris, o, d, base["id"], base["t"], 77)
    eb = _expect(oracle, ref, bo, bd, bt)
    for sch in CLUSTER_SCHEDULES + [dict(clusters=True, image_width=cam.width), dict(clusters=True, persistent=True, image_width=cam.width,
                                                                                     coop=True),
                                    dict(clusters=True, persistent=True, image_width=cam.width, packet=True)]:
        _same(T, core.trace(tree, o, dd, tmax=tm, schedule=sch), e)
        _same(T, core.trace(tree, o, d, id_mode=1, schedule=sch), e1)
        _same(T, core.trace(tree, bo, bd, tmax=bt, schedule=sch), eb)


@pytest.mark.parametrize("coop", [False, True])
def test_cluster_counters_leave_hits_unchanged(T, oracle, coop):
    """Counting runs return the same hits; every ray reads whole records (4 boxes each), at least the root's,
    and every ray with a hit tested at least one triangle."""
    from cudart_b200 import core
    mesh = scenes.soup(50000, seed=33)
    tree, ref = _build(T, oracle, mesh)
    o, d = (_dev(T, a) for a in scenes.sphere_rays(mesh, 64, seed=3))
    sch = dict(clusters=True, persistent=True, blocks_per_sm=8, coop=coop)
    plain = core.trace(tree, o, d, schedule=sch)
    counted = core.trace(tree, o, d, schedule=sch, counters=True)
    T.cuda.synchronize()
    assert T.equal(plain["id"], counted["id"]) and T.equal(plain["t"], counted["t"])
    v = _host(counted["visits"])
    t = _host(counted["tests"])
    assert (v >= 4).all() and (v % 4 == 0).all()
    assert (t[_host(counted["id"]) >= 0] >= 1).all()


def test_blob_without_cluster_tree_reports_it(T, oracle):
    """A cluster schedule on a blob built without the cluster tree (or rebuilt without it) misses every ray
    and raises RT_DEVERR_ACCEL_MISSING; the records' walk of the same blob is unaffected."""
    from cudart_b200 import _abi, core
    mesh = scenes.soup(5000, seed=34)
    tree, ref = _build(T, oracle, mesh, clusters=False)
    o, d = (_dev(T, a) for a in scenes.sphere_rays(mesh, 32, seed=4))
    for sch in CLUSTER_SCHEDULES:
        out = core.trace(tree, o, d, schedule=sch)
        T.cuda.synchronize()
        assert int(_host(out["err"])[0]) & _abi.DEVERR_ACCEL_MISSING, sch
        assert (_host(out["id"]) == -1).all()
    # built with it, then rebuilt in place without it: the valid word is cleared again
    v = _dev(T, mesh.vertices)
    f = _dev(T, mesh.faces.view(np.int32))
    t2 = core.build_lbvh(v, f, clusters=True)
    good = core.trace(t2, o, d, schedule=CLUSTER_SCHEDULES[0])
    T.cuda.synchronize()
    assert int(_host(good["err"])[0]) == 0
    core.build_lbvh(v, f, clusters=False, out=t2)
    stale = core.trace(t2, o, d, schedule=CLUSTER_SCHEDULES[0])
    recs = core.trace(t2, o, d)
    T.cuda.synchronize()
    assert int(_host(stale["err"])[0]) & _abi.DEVERR_ACCEL_MISSING
    _same(T, recs, _expect(oracle, ref, o, d))


def test_batched_cluster_walks_match_single_mesh(T, oracle):
    """A batched build with cluster trees: one batched launch per cluster schedule (with and without ray
    orders) equals the oracle's hits of every mesh."""
    from cudart_b200 import core
    meshes = [scenes.soup(1, seed=1), scenes.soup(17, seed=2), scenes.terrain(9, 3), scenes.soup(224, seed=4),
              scenes.soup(5000, seed=5), scenes.terrain(64, 6), scenes.soup(33000, seed=7), scenes.soup(2, seed=8),
              scenes.soup(70000, seed=9), scenes.soup(1025, seed=10)]
    verts, faces, fo, vo = scenes.concat_batch(meshes)
    bt = core.batch_build(_dev(T, verts), _dev(T, faces.view(np.int32)), fo, vo, clusters=True)
    rays = [scenes.sphere_rays(m, 24 + 8 * i, seed=100 + i) for i, m in enumerate(meshes)]
    ro = [0]
    for o, _ in rays:
        ro.append(ro[-1] + len(o))
    O = _dev(T, np.concatenate([o for o, _ in rays]))
    D = _dev(T, np.concatenate([d for _, d in rays]))
    roff = T.tensor(ro, dtype=T.int32, device="cuda")
    exp_id, exp_t, exp_uv = [], [], []
    for m, mesh in enumerate(meshes):
        ref = oracle.lbvh_build(mesh.vertices, mesh.faces, oracle.hitbox(mesh.vertices))
        e = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], rays[m][0], rays[m][1], None, mode=0)
        exp_id.append(e["id"]); exp_t.append(e["t"]); exp_uv.append(e["uv"])
    e = dict(id=np.concatenate(exp_id), t=np.concatenate(exp_t), uv=np.concatenate(exp_uv))
    schedules = [dict(clusters=True), dict(clusters=True, while_while=True), dict(clusters=True, persistent=True, blocks_per_sm=8),
                 dict(clusters=True, persistent=True, blocks_per_sm=8, while_while=True, sorted_bits=12),
                 dict(clusters=True, persistent=True, blocks_per_sm=16, coop=True),
                 dict(clusters=True, persistent=True, blocks_per_sm=16, coop=True, sorted_bits=12),
                 dict(clusters=True, persistent=True, blocks_per_sm=8, sorted_bits=0),
                 dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True),  # warps spanning meshes: per-lane walks
                 dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True, sorted_bits=21),
                 dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True, lane_threshold=16, sorted_bits=21),
                 dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, lane_threshold=8),
                 dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, lane_threshold=32, sorted_bits=12),
                 dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, lane_threshold=4, while_while=True)]
    for sch in schedules:
        h = core.batch_trace(bt, O, D, roff, schedule=sch)
        T.cuda.synchronize()
        _same(T, h, e)
    # a batched build without cluster trees: refused per ray, no stale reads
    from cudart_b200 import _abi
    b2 = core.batch_build(_dev(T, verts), _dev(T, faces.view(np.int32)), fo, vo)
    for sch in schedules:
        h = core.batch_trace(b2, O, D, roff, schedule=sch)
        T.cuda.synchronize()
        assert int(_host(h["err"])[0]) & _abi.DEVERR_ACCEL_MISSING, sch
        assert (_host(h["id"]) == -1).all(), sch


def test_batched_trace_writes_bounce_rays(T, oracle):
    """rt_batch_trace with bounce outputs: the packet walks write each ray's bounce as it finishes (warps whose rays
    span meshes through the per-lane fallback), every other schedule through one rt_batch_bounce_rays launch after
    the trace; either way the bounces equal rt_batch_bounce_rays' from the written hits bit for bit, inactive rays
    (tmax <= 0) and misses included, and the hits are unchanged."""
    from cudart_b200 import core
    meshes = [scenes.soup(1, seed=1), scenes.terrain(9, 3), scenes.soup(5000, seed=5), scenes.terrain(64, 6),
              scenes.soup(33000, seed=7), scenes.soup(1025, seed=10)]
    verts, faces, fo, vo = scenes.concat_batch(meshes)
    bt = core.batch_build(_dev(T, verts), _dev(T, faces.view(np.int32)), fo, vo, clusters=True)
    rays = [scenes.sphere_rays(m, 40 + 8 * i, seed=200 + i) for i, m in enumerate(meshes)]
    ro = [0]
    for o, _ in rays:
        ro.append(ro[-1] + len(o))
    O = _dev(T, np.concatenate([o for o, _ in rays]))
    D = _dev(T, np.concatenate([d for _, d in rays]))
    R = O.shape[0]
    tmax = T.full((R,), 1e30, dtype=T.float32, device="cuda")
    tmax[3::11] = 0.5  # short reach
    tmax[::7] = -1.0  # inactive rays
    roff = T.tensor(ro, dtype=T.int32, device="cuda")
    plain = core.batch_trace(bt, O, D, roff, tmax=tmax, schedule=dict(clusters=True))
    for sch in [dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True),
                dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True, sorted_bits=21),
                dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True, lane_threshold=16, sorted_bits=21),
                dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, lane_threshold=8),
                dict(clusters=True), dict(persistent=True, blocks_per_sm=8, coop=True, wide=True)]:
        for seed in (5, 1234567):
            h = core.batch_trace(bt, O, D, roff, tmax=tmax, schedule=sch, bounce=(seed, None))
            ref = core.batch_bounce_rays(bt, roff, O, D, h["id"], h["t"], seed)
            T.cuda.synchronize()
            for k in ("id", "t", "uv"):
                assert T.equal(h[k], plain[k]), (sch, k)
            for a, b in zip(h["b"], ref[:3]):
                assert T.equal(a.view(T.int32), b.view(T.int32)), (sch, seed)
            assert (h["b"][2][::7] == -1.0).all()
