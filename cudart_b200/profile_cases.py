"""Small, self-contained workloads for profiling one kernel at a time (the
commands recorded in profiles/*.md run these).

    python -m cudart_b200.profile_cases <case>

Each case builds its inputs, runs the operation once untimed (warm-up), then
once more; a profiler capturing the last launch of the named kernel sees a
steady-state launch. Cases (kernel of interest in brackets):

  bench_step     three steps of the main workload (build, primary, bounce)     [launch list]
  build_16m      LBVH build of a 2^24-face soup, twice                            [k_radix_scatter, k_leaves, k_boxes_morton]
  batch_build    batched build of 1024 meshes (9.9M faces), twice                 [launch list]
  trace_primary  2^20-face soup, 1920x1080 primary rays, tuned tile schedule   [k_trace_accel]
  trace_bounce   the same scene's diffuse bounces, cooperative schedule          [k_trace_coop]
  mlp_propose    proposal network inference on 2^18 rays (4096 slots)            [k_mlp_propose_tc]
  mlp_train      one training step, batch 8192                                   [k_gemm_xent_tc, k_gemm_tc]
  sah_build      SAH build of the 2^20-face soup                                 [k_sah_small, k_huge_bins, k_sah_big]
  raster         rasteriser, 2^20-face soup, 1920x1080                           [k_raster_zones, k_raster_emit]
  mlp_grouped    64 grouped networks: 3 training steps of 1024 rays each,        [k_gemm_tc, k_softmax_xent, ...]
                 then proposals for 64 x 518,400 rays
  sort_16m       2^24 random (key, value) pairs, 32-bit keys, sorted twice         [k_onesweep, k_sort_hist]
  trace_clusters 2^20-face soup with its cluster tree: packet primaries, per-lane [k_trace_clusters*]
                 bounces, twice each
  c4_frame [M]   M (default 64) deformed instances of the 1/16-size learned       [launch list, k_batch_trace_clusters*]
                 scene, three frames of the plain path: batched build, primary
                 rays, batched trace, bounce rays, batched trace
"""
from __future__ import annotations

import sys

import numpy as np
import torch


def _soup_scene():
    from . import core, scenes
    mesh, cam = scenes.soup_1m_scene()
    v = torch.from_numpy(mesh.vertices).cuda()
    f = torch.from_numpy(mesh.faces.view(np.int32)).cuda()
    return mesh, cam, v, f, core.build_lbvh(v, f)


def trace_primary():
    from . import core
    mesh, cam, v, f, tree = _soup_scene()
    c = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    o, d = core.primary_rays(c, cam.width, cam.height)
    sch = dict(image_width=cam.width, while_while=True, wide=True)  # the schedule the tuner picks for these rays
    for _ in range(2):
        core.trace(tree, o, d, schedule=sch)
    torch.cuda.synchronize()


def trace_bounce():
    from . import core
    mesh, cam, v, f, tree = _soup_scene()
    c = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    o, d = core.primary_rays(c, cam.width, cam.height)
    h = core.trace(tree, o, d)
    b = core.bounce_rays(tree.tris, o, d, h["id"], h["t"], 1234)
    for _ in range(2):
        core.trace(tree, b[0], b[1], tmax=b[2], schedule=dict(persistent=True, blocks_per_sm=16, while_while=True, sorted=True,
                                                              coop=True, wide=True))  # the tuner's pick for these rays
    torch.cuda.synchronize()


def trace_clusters():
    """The 2^20-face soup with its cluster tree: primary rays as warp packets over 8 x 4 pixel tiles, then their
    bounces as per-lane walks over 8 x 4 tiles (the c1 leg's picks), twice each."""
    from . import core
    mesh, cam, v, f, _ = _soup_scene()
    tree = core.build_lbvh(v, f, clusters=True)
    c = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    o, d = core.primary_rays(c, cam.width, cam.height)
    s1 = dict(clusters=True, image_width=cam.width, persistent=True, blocks_per_sm=16, packet=True)
    s2 = dict(clusters=True, image_width=cam.width)
    h = core.trace(tree, o, d, schedule=s1)
    b = core.bounce_rays(tree.tris, o, d, h["id"], h["t"], 1234)
    for _ in range(2):
        core.trace(tree, o, d, schedule=s1)
        core.trace(tree, b[0], b[1], tmax=b[2], schedule=s2)
    torch.cuda.synchronize()


def bench_step():
    """Three steps of the main workload with the schedules the tuner picks for
    it: build, primary rays, trace, bounce rays, trace (no tuning launches)."""
    from . import core
    mesh, cam, v, f, tree = _soup_scene()
    c = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    W, H = cam.width, cam.height
    s1 = dict(image_width=W, while_while=True, wide=True)
    s2 = dict(persistent=True, blocks_per_sm=16, while_while=True, sorted=True, coop=True, wide=True)
    for _ in range(3):
        core.build_lbvh(v, f, out=tree)
        o, d = core.primary_rays(c, W, H)
        h = core.trace(tree, o, d, schedule=s1)
        b = core.bounce_rays(tree.tris, o, d, h["id"], h["t"], 1234)
        core.trace(tree, b[0], b[1], tmax=b[2], schedule=s2)
    torch.cuda.synchronize()


def build_16m():
    from . import core, scenes
    mesh = scenes.soup(1 << 24, seed=7)
    v = torch.from_numpy(mesh.vertices).cuda()
    f = torch.from_numpy(mesh.faces.view(np.int32)).cuda()
    del mesh
    t = core.build_lbvh(v, f)
    core.build_lbvh(v, f, out=t)
    torch.cuda.synchronize()


def batch_build():
    from . import core, scenes
    meshes = scenes.batch_meshes(1024, seed=3)
    verts, faces, fo, vo = scenes.concat_batch(meshes)
    del meshes
    v = torch.from_numpy(verts).cuda()
    f = torch.from_numpy(faces.view(np.int32)).cuda()
    t = core.batch_build(v, f, fo, vo)
    core.batch_build(v, f, fo, vo, out=t)
    torch.cuda.synchronize()


def mlp_propose():
    from . import proposal, scenes
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    o, d = scenes.box_rays_torch(1 << 18, box, seed=1)
    net = proposal.ProposalNet(seed=0)
    for _ in range(2):
        net.propose(o, d, box)
    torch.cuda.synchronize()


def mlp_train():
    from . import proposal, scenes
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    B = 8192
    o, d = scenes.box_rays_torch(B, box, seed=1)
    labels = torch.randint(0, 4096, (B,), dtype=torch.int32, device="cuda", generator=torch.Generator(device="cuda").manual_seed(2))
    net = proposal.ProposalNet(seed=0)
    for _ in range(2):
        net.train_step(o, d, labels, box)
    torch.cuda.synchronize()


def sah_build():
    from . import core, scenes
    mesh = scenes.soup(1 << 20, 1)
    v = torch.from_numpy(mesh.vertices).cuda()
    f = torch.from_numpy(mesh.faces.view(np.int32)).cuda()
    t = core.build_sah(v, f)
    core.build_sah(v, f, out=t)
    torch.cuda.synchronize()


def raster():
    from . import core, scenes
    mesh, cam = scenes.soup_1m_scene()
    v = torch.from_numpy(mesh.vertices).cuda()
    f = torch.from_numpy(mesh.faces.view(np.int32)).cuda()
    c = core.make_camera((cam.center[0] + 0.05, cam.center[1] + 0.1, cam.center[2]), cam.target, fov=cam.fov, ratio=cam.ratio)
    m = core.raster_matrix(c, cam.target)
    for _ in range(2):
        core.rasterize(v, f, m, cam.width, cam.height)
    torch.cuda.synchronize()


def mlp_grouped():
    from . import proposal, scenes
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    G, B, R = 64, 1024, 518400
    o, d = scenes.box_rays_torch(G * B, box, seed=1)
    labels = torch.randint(0, 4096, (G * B,), dtype=torch.int32, device="cuda", generator=torch.Generator(device="cuda").manual_seed(2))
    net = proposal.ProposalGroup(G, seed=0)
    for _ in range(3):
        net.train_step(o, d, labels, box, B)
    po, pd = scenes.box_rays_torch(G * R, box, seed=3)
    for _ in range(2):
        net.propose(po, pd, box, R)
    torch.cuda.synchronize()


def sort_16m():
    from . import core
    g = torch.Generator(device="cuda").manual_seed(5)
    k0 = torch.randint(-(1 << 31), (1 << 31) - 1, (1 << 24,), dtype=torch.int32, device="cuda", generator=g)
    for _ in range(2):
        k = k0.clone()
        v = torch.empty_like(k)
        core.sort_pairs(k, v, 32, init_values=True)
    torch.cuda.synchronize()


def c4_frame(count: int = 64):
    """Three frames of the instanced workload's plain path (cluster trees) with the schedules the tuner picks on
    it: the primaries as warp packets over 8 x 4 pixel tiles, the bounces as per-lane walks in warps that take
    new rays once 8 lanes are idle."""
    from .instances import InstancedFrames
    w = InstancedFrames(count, 1 / 16, 960, 540)
    w.schedule_primary = dict(clusters=True, persistent=True, blocks_per_sm=16, packet=True, tiles=[count, 960, 540])
    w.schedule_bounce = dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, lane_threshold=8)
    plain = None
    for f in range(3):
        w.displace(f)
        w.build()
        w.primary_rays()
        plain = w.trace_plain(out=plain)
    torch.cuda.synchronize()


CASES = {"bench_step": bench_step, "trace_clusters": trace_clusters, "build_16m": build_16m, "batch_build": batch_build, "trace_primary": trace_primary, "trace_bounce": trace_bounce, "mlp_propose": mlp_propose, "mlp_train": mlp_train,
         "sah_build": sah_build, "raster": raster, "mlp_grouped": mlp_grouped, "c4_frame": c4_frame, "sort_16m": sort_16m}

if __name__ == "__main__":
    if len(sys.argv) not in (2, 3) or sys.argv[1] not in CASES:
        raise SystemExit("usage: python -m cudart_b200.profile_cases {" + ",".join(CASES) + "} [size]")
    torch.cuda.set_device(0)
    CASES[sys.argv[1]](*(int(a) for a in sys.argv[2:]))
    print("ok", sys.argv[1])
