"""Parity at the benchmark's full sizes: the trees and hits of the large
workloads (the 4,022,242-triangle learned scene, the 1024-mesh batch, the
64-instance frame) set beside the CPU oracle, which is pinned to the
reference's own code. Builds are compared whole; hits on every 16th ray (c3),
on up to 4096 rays of each of 32 meshes spread over the size range (c2) and on
all rays of two instances (c4, through the cluster trees and the node records), bit for bit (tolerance:
exact)."""
import numpy as np
import pytest
import torch

from cudart_b200 import scenes

pytestmark = pytest.mark.gpu

# the schedules the autotuner picks on these workloads (results never depend on the schedule)
C3_SCHEDULE = dict(image_width=0, persistent=True, blocks_per_sm=8, while_while=True, sorted=True, coop=True, wide=True)
BATCH_SCHEDULE = dict(while_while=True, wide=True, persistent=True, blocks_per_sm=8, coop=True)
# the instanced frame's picks on the cluster trees (primary: 8 x 4 pixel tiles; bounce: rays ordered by mesh, octant, Morton)
C4_PRIMARY = dict(clusters=True, persistent=True, blocks_per_sm=8, tiles=[64, 960, 540])
C4_BOUNCE = dict(clusters=True, persistent=True, blocks_per_sm=16, sorted_bits=12)


def _u32(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _h(t):
    return t.cpu().numpy()


def _same_tree(ref, nodes, indices, codes, faces, tris, boxes):
    nc = ref["info"]["node_count"]
    assert np.array_equal(_u32(_h(nodes)[:nc]), _u32(ref["nodes"]))
    assert np.array_equal(_u32(_h(indices)), ref["indices"])
    assert np.array_equal(_u32(_h(codes)), ref["codes"])
    assert np.array_equal(_u32(_h(faces)), _u32(ref["faces"]))
    assert np.array_equal(_u32(_h(tris)), _u32(ref["tris"]))
    assert np.array_equal(_u32(_h(boxes)), _u32(ref["boxes"]))


def _same_hits(gpu_id, gpu_t, gpu_uv, e):
    assert np.array_equal(_h(gpu_id), e["id"])
    assert np.array_equal(_u32(_h(gpu_t)), _u32(e["t"]))
    assert np.array_equal(_u32(_h(gpu_uv)), _u32(e["uv"]))


def test_c3_full_scene_build_and_sampled_rays(oracle):
    """The 4,022,242-triangle terrain + soup scene built whole, and the 8M evaluation rays traced with the
    tuned schedule (persistent, cooperative, ray-sorted, 4-wide records); every 16th ray against the oracle."""
    from cudart_b200 import core
    mesh = scenes.learned_scene(1.0)
    assert mesh.face_count == 4022242
    v = torch.from_numpy(mesh.vertices).cuda()
    f = torch.from_numpy(mesh.faces.view(np.int32)).cuda()
    tree = core.build_lbvh(v, f)
    torch.cuda.synchronize()
    ref = oracle.lbvh_build(mesh.vertices, mesh.faces, oracle.hitbox(mesh.vertices))
    info = tree.info_host()
    for k in ("node_count", "leaf_count", "real_depth", "split_count"):
        assert info[k] == ref["info"][k], k
    assert info["error"] == 0
    _same_tree(ref, tree.nodes, tree.indices, tree.codes, tree.faces, tree.tris, tree.boxes)
    box = scenes.scene_box(mesh, 1.5)
    eo, ed = scenes.box_rays_torch(8 << 20, box, seed=2)
    hits = core.trace(tree, eo, ed, schedule=C3_SCHEDULE)
    torch.cuda.synchronize()
    assert int(hits["err"].item()) == 0
    sel = slice(0, eo.shape[0], 16)
    e = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], np.ascontiguousarray(_h(eo[sel])), np.ascontiguousarray(_h(ed[sel])))
    _same_hits(hits["id"][sel], hits["t"][sel], hits["uv"][sel], e)
    assert 0.2 < (e["id"] >= 0).mean() < 0.6


def test_c2_full_batch_sampled_meshes(oracle):
    """The whole 1024-mesh batch (9.9M faces, 59.6M rays) built and traced in one launch each; 32 meshes
    spread over the size range (64 .. 65,536 faces) compared with their own oracle builds and traces."""
    from cudart_b200 import core
    meshes = scenes.batch_meshes(1024, seed=3)
    verts, faces, fo, vo = scenes.concat_batch(meshes)
    orig, dirs, ro = scenes.batch_sphere_rays_torch(meshes)
    bt = core.batch_build(torch.from_numpy(verts).cuda(), torch.from_numpy(faces.view(np.int32)).cuda(), fo, vo)
    roff = torch.tensor(ro.astype(np.int32), device="cuda")
    hits = core.batch_trace(bt, orig, dirs, roff, schedule=BATCH_SCHEDULE)
    torch.cuda.synchronize()
    assert int(hits["err"].item()) == 0
    info = _h(bt.info)
    assert np.all(info[:, 7] == 0)
    sizes = np.array([m.face_count for m in meshes])
    pick = np.argsort(sizes, kind="stable")[np.linspace(0, len(meshes) - 1, 32).astype(int)]
    assert sizes[pick].min() <= 128 and sizes[pick].max() >= 32768
    for m in pick:
        mesh = meshes[m]
        ref = oracle.lbvh_build(mesh.vertices, mesh.faces, oracle.hitbox(mesh.vertices))
        nc = ref["info"]["node_count"]
        assert int(info[m, 0]) == nc, m
        F0, F1 = fo[m], fo[m + 1]
        _same_tree(ref, bt.mesh_nodes(m, nc), bt.indices[F0:F1], bt.codes[F0:F1], bt.faces[F0:F1], bt.tris[F0:F1], bt.boxes[F0:F1])
        r0, r1 = int(ro[m]), int(ro[m + 1])
        step = max(1, (r1 - r0) // 4096)
        sel = slice(r0, r1, step)
        e = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], np.ascontiguousarray(_h(orig[sel])), np.ascontiguousarray(_h(dirs[sel])))
        _same_hits(hits["id"][sel], hits["t"][sel], hits["uv"][sel], e)


def test_c4_instances_of_one_frame(oracle):
    """One frame of the 64-instance workload at full size (16,097,152 faces, 33,177,600 primary rays):
    instances 0 and 37 built by the oracle from the frame's displaced vertices and compared with the batched
    build; all their primary rays (equal to the oracle's camera rays) and the bounce rays the GPU made from
    the hits traced by the oracle; instance 0's bounce rays equal the oracle's bounce generator."""
    from cudart_b200.instances import InstancedFrames
    w = InstancedFrames(64, 1 / 16, 960, 540)
    assert w.face_count == 16097152 and w.ray_count == 33177600
    w.displace(1)
    w.build()
    w.schedule_primary, w.schedule_bounce = C4_PRIMARY, C4_BOUNCE
    plain = w.trace_plain()
    w.schedule = BATCH_SCHEDULE  # the node-record walk: the same bits for every ray
    rec = w.trace_plain()
    torch.cuda.synchronize()
    assert int(plain["h1"]["err"].item()) == 0 and int(plain["h2"]["err"].item()) == 0
    for k in ("h1", "h2"):
        assert int(rec[k]["err"].item()) == 0
        assert torch.equal(rec[k]["id"], plain[k]["id"]) and torch.equal(rec[k]["t"], plain[k]["t"]) and torch.equal(rec[k]["uv"], plain[k]["uv"])
    info = _h(w.tree.info)
    assert np.all(info[:, 7] == 0)
    N, V, R = w.face_offsets[1], w.vertex_offsets[1], w.rays_per_instance
    base_faces = np.ascontiguousarray(_h(w.faces[:N])).view(np.uint32)
    for i in (0, 37):
        verts = np.ascontiguousarray(_h(w.verts[i * V:(i + 1) * V]))
        ref = oracle.lbvh_build(verts, base_faces, oracle.hitbox(verts))
        nc = ref["info"]["node_count"]
        assert int(info[i, 0]) == nc
        F0, F1 = i * N, (i + 1) * N
        t = w.tree
        _same_tree(ref, t.mesh_nodes(i, nc), t.indices[F0:F1], t.codes[F0:F1], t.faces[F0:F1], t.tris[F0:F1], t.boxes[F0:F1])
        sl = slice(i * R, (i + 1) * R)
        o, d = np.ascontiguousarray(_h(w.orig[sl])), np.ascontiguousarray(_h(w.dir[sl]))
        po, pd, _, _ = oracle.primary_rays(w.cams[i])
        assert np.array_equal(_u32(o), _u32(po)) and np.array_equal(_u32(d), _u32(pd))
        e = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], o, d)
        _same_hits(plain["h1"]["id"][sl], plain["h1"]["t"][sl], plain["h1"]["uv"][sl], e)
        b = plain["b"]
        bo, bd, btm = (np.ascontiguousarray(_h(x[sl])) for x in b[:3])
        if i == 0:  # ray indices of instance 0 start at 0, as the oracle's generator counts them
            eo, ed, et = oracle.bounce_rays(ref["tris"], o, d, e["id"], e["t"], 1000 + w.frame_index)
            assert np.array_equal(_u32(bo), _u32(eo)) and np.array_equal(_u32(bd), _u32(ed)) and np.array_equal(_u32(btm), _u32(et))
        e2 = oracle.trace(ref["nodes"], ref["tris"], ref["indices"], bo, bd, btm)
        _same_hits(plain["h2"]["id"][sl], plain["h2"]["t"][sl], plain["h2"]["uv"][sl], e2)
        assert (e["id"] >= 0).mean() > 0.1


def test_batch_bounce_rays_match_global_positions():
    """rt_batch_bounce_rays (instance-local hit positions) makes the same rays as rt_bounce_rays given the
    global positions."""
    from cudart_b200 import core
    from cudart_b200.instances import InstancedFrames
    w = InstancedFrames(4, 1 / 256, 64, 48)
    w.displace(3)
    w.build()
    h1 = core.batch_trace(w.tree, w.orig, w.dir, w.ray_offsets)
    b = w.bounce(h1)
    gpos = torch.where(h1["id"] >= 0, h1["id"] + w.ray_face_base, h1["id"])
    b2 = core.bounce_rays(w.tree.tris, w.orig, w.dir, gpos, h1["t"], 1000 + w.frame_index)
    torch.cuda.synchronize()
    assert (h1["id"] >= 0).any() and (h1["id"] < 0).any()
    for x, y in zip(b, b2):
        assert torch.equal(x.view(torch.int32), y.view(torch.int32))


def test_batch_ray_orders_and_schedules_identical():
    """rt_batch_ray_order is a permutation with the rays grouped by mesh, then octant, inactive rays last;
    rt_image_tile_order maps each 32 slots to an 8 x 4 tile of one instance's image; and every batched
    schedule, the ordered ones included, returns the same bits for primaries and bounces."""
    from cudart_b200 import core, tune
    from cudart_b200.instances import InstancedFrames
    w = InstancedFrames(4, 1 / 256, 64, 48)
    w.displace(2)
    w.build()
    h1 = core.batch_trace(w.tree, w.orig, w.dir, w.ray_offsets)
    b = w.bounce(h1)
    h2 = core.batch_trace(w.tree, b[0], b[1], w.ray_offsets, tmax=b[2])
    torch.cuda.synchronize()
    R, W, H = w.ray_count, w.width, w.height
    tiles = core.image_tile_order(w.count, W, H).cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(tiles), np.arange(R))
    s = np.arange(R)
    img, k = s // (W * H), s % (W * H)
    x = (k // 32 % (W // 8)) * 8 + (k % 32) % 8
    y = (k // 32 // (W // 8)) * 4 + (k % 32) // 8
    assert np.array_equal(tiles, img * W * H + y * W + x)
    tm = b[2].cpu().numpy()
    dirs = b[1].cpu().numpy()
    mesh = np.repeat(np.arange(w.count), w.rays_per_instance)
    for bits in (0, 6, 21):
        order = core.batch_ray_order(b[0], b[1], b[2], w.ray_offsets, w.count, core.batch_tree_box(w.tree), bits).cpu().numpy()
        order = order.astype(np.int64)
        assert np.array_equal(np.sort(order), np.arange(R))
        act = tm[order] > 0
        n_act = int((tm > 0).sum())
        assert act[:n_act].all() and not act[n_act:].any()
        key = mesh[order[:n_act]] * 8 + ((dirs[order[:n_act], 0] < 0) | 2 * (dirs[order[:n_act], 1] < 0) | 4 * (dirs[order[:n_act], 2] < 0))
        assert np.all(np.diff(key) >= 0), bits
        if bits == 0:  # stable: equal keys keep their index order
            same = np.diff(key) == 0
            assert np.all(np.diff(order[:n_act])[same] > 0)
    for sch in tune.batch_candidates(images=(w.count, W, H)) + tune.cluster_batch_candidates(images=(w.count, W, H)):
        a = core.batch_trace(w.tree, w.orig, w.dir, w.ray_offsets, schedule=sch)
        c = core.batch_trace(w.tree, b[0], b[1], w.ray_offsets, tmax=b[2], schedule=sch)
        torch.cuda.synchronize()
        for x_, y_ in ((a, h1), (c, h2)):
            assert int(x_["err"].item()) == 0, sch
            assert torch.equal(x_["id"], y_["id"]) and torch.equal(x_["t"], y_["t"]) and torch.equal(x_["uv"], y_["uv"]), sch


def test_bounce_order_is_active_first_and_traces_the_same():
    """rt_batch_bounce_rays' order lists every ray once, the active bounces first; the bounce launch traced in
    that order returns the same bits as in ray order."""
    from cudart_b200 import core
    from cudart_b200.instances import InstancedFrames
    w = InstancedFrames(4, 1 / 256, 64, 48)
    w.displace(5)
    w.build()
    h1 = core.batch_trace(w.tree, w.orig, w.dir, w.ray_offsets)
    b = w.bounce(h1)
    base = core.batch_trace(w.tree, b[0], b[1], w.ray_offsets, tmax=b[2])
    R = w.ray_count
    order = b[3][:R].cpu().numpy().astype(np.int64)
    tm = b[2].cpu().numpy()
    assert np.array_equal(np.sort(order), np.arange(R))
    n_act = int((tm > 0).sum())
    assert 0 < n_act < R
    assert (tm[order[:n_act]] > 0).all() and not (tm[order[n_act:]] > 0).any()
    for sch in [dict(while_while=True, wide=True, persistent=True, blocks_per_sm=8, coop=coop) for coop in (False, True)] + \
            [dict(clusters=True, persistent=True, blocks_per_sm=8, coop=coop) for coop in (False, True)]:
        h = core.batch_trace(w.tree, b[0], b[1], w.ray_offsets, tmax=b[2], schedule=sch, order=b[3])
        torch.cuda.synchronize()
        assert torch.equal(h["id"], base["id"]) and torch.equal(h["t"], base["t"]) and torch.equal(h["uv"], base["uv"])
