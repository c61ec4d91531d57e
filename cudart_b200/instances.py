"""Many deformed instances of one scene, rebuilt and traced every frame, each
with its own proposal network fine-tuned on the previous frame's hits.

Per frame: every instance's vertices move by fresh N(0, sigma^2) noise; one
batched LBVH build makes all instance trees (rt_batch_build); each instance's
primary rays (one pinhole camera per instance) and one diffuse bounce per hit
are traced two ways over all instances at once:

  plain   rt_batch_trace for the primaries, rt_bounce_rays, rt_batch_trace
          for the bounces;
  learned the grouped MLP (one network per instance, the same launches for
          all) proposes a depth-12 slot of the instance's tree per ray, and
          rt_batch_trace_seeded walks it first. Hits are bit-identical to the
          plain ones, so the bounces are the same rays.

The plain hits label the frame's rays (the slot holding the hit, per
instance); the next frame fine-tunes every instance's network on them with
`steps` grouped Adam steps of `batch` rays per instance, alternating between
primary and bounce rays.
"""
from __future__ import annotations

import numpy as np
import torch

from . import core, proposal, scenes


HOP = 7919  # a prime: consecutive samples of a batch lie far apart in the list of hits


class InstancedFrames:
    def __init__(self, count: int, scale: float, width: int, height: int, device="cuda", seed: int = 7, depth: int = proposal.DEPTH,
                 batch: int = 1024, steps: int = 200, lr: float = 1e-3, sigma: float = 0.002, net_seed: int = 0,
                 clusters: bool = True):
        if (width * height) % 128:
            raise ValueError("width * height must be a multiple of 128 (one grouped GEMM tile of rays)")
        self.count, self.width, self.height = count, width, height
        self.dev = torch.device(device)
        self.seed, self.depth, self.batch, self.steps, self.lr, self.sigma = seed, depth, batch, steps, lr, sigma
        base = scenes.learned_scene(scale)
        self.base_faces = base.face_count
        self.base_v = torch.from_numpy(base.vertices).to(self.dev)
        f = torch.from_numpy(base.faces.view(np.int32)).to(self.dev)
        self.faces = f.repeat(count, 1).contiguous()
        N, V = base.face_count, base.vertex_count
        self.face_offsets = [i * N for i in range(count + 1)]
        self.vertex_offsets = [i * V for i in range(count + 1)]
        self.cams = scenes.instance_cameras(count, width, height)
        R = width * height
        self.rays_per_instance = R
        self.orig = torch.empty((count * R, 4), dtype=torch.float32, device=self.dev)
        self.dir = torch.empty((count * R, 4), dtype=torch.float32, device=self.dev)
        self.rt_cams = [core.make_camera(c.center, c.target, fov=c.fov, ratio=c.ratio) for c in self.cams]
        self.cam_bases = core.camera_bases(self.rt_cams, width, height, device=self.dev)  # the cameras stay put
        self.primary_rays()
        self.ray_offsets = torch.tensor([i * R for i in range(count + 1)], dtype=torch.int32, device=self.dev)
        self.ray_face_base = torch.repeat_interleave(torch.tensor(self.face_offsets[:-1], dtype=torch.int32, device=self.dev),
                                                     torch.full((count,), R, dtype=torch.int64, device=self.dev))
        pts = np.concatenate([base.vertices[:, :3], np.array([c.center for c in self.cams], np.float32)])
        lo, hi = pts.min(0).astype(np.float64), pts.max(0).astype(np.float64)
        mid, half = 0.5 * (lo + hi), 0.55 * (hi - lo)
        self.box = tuple(float(x) for x in np.concatenate([mid - half, mid + half]))
        self.nets = proposal.ProposalGroup(count, 1 << depth, device=self.dev, seed=net_seed)
        self.verts = None
        self.tree = None
        self.slots = None
        self.frame_index = -1
        # batched traversal schedules of the primary and bounce launches (tune() picks them); results never depend on them
        self.schedule_primary = self.schedule_bounce = None
        self.prev = None  # (bounce orig, bounce dir, primary labels, bounce labels) of the previous frame
        self.clusters = clusters  # every build also makes the cluster trees (the tuner then tries their walks)

    @property
    def schedule(self):
        return self.schedule_primary

    @schedule.setter
    def schedule(self, sch):
        """One schedule for both launches."""
        self.schedule_primary = self.schedule_bounce = sch

    @property
    def face_count(self) -> int:
        return self.faces.shape[0]

    @property
    def ray_count(self) -> int:
        return self.orig.shape[0]

    # ------------------------------------------------------------ frame steps
    def displace(self, frame: int):
        self.frame_index = frame
        self.verts = scenes.displace_instances(self.base_v, self.count, frame, self.seed, self.sigma, out=self.verts)

    def primary_rays(self, stream=None):
        """Every instance's pinhole rays (one rt_batch_primary_rays launch for all cameras) into orig / dir."""
        core.batch_primary_rays(self.cam_bases, self.width, self.height, out=(self.orig, self.dir), stream=stream)

    def build(self, verts=None):
        """One batched LBVH build of all instances, from `verts` (default: the displaced frame)."""
        v = self.verts if verts is None else verts
        self.tree = core.batch_build(v, self.faces, self.face_offsets, self.vertex_offsets, out=self.tree, clusters=self.clusters)
        return self.tree

    def build_and_rays(self, verts=None, aux=None):
        """The frame's build and its primary rays side by side: the rays do not depend on the build, so they are
        made on stream `aux` (forked from and joined back into the current stream; inside a graph capture this
        becomes two parallel branches)."""
        if aux is None:
            self.primary_rays()
            return self.build(verts)
        cur = torch.cuda.current_stream()
        aux.wait_stream(cur)
        with torch.cuda.stream(aux):
            self.primary_rays()
        tree = self.build(verts)
        cur.wait_stream(aux)
        return tree

    def make_slots(self):
        self.slots = proposal.batch_subtree_slots(self.tree, self.depth)
        return self.slots

    def bounce_seed(self) -> int:
        return 1000 + self.frame_index

    def bounce_needs_order(self) -> bool:
        """Whether a traced schedule reads the bounce generator's active-first order (or no schedule is picked yet)."""
        return self.schedule_bounce is None or bool(self.schedule_bounce.get("given_order")) or \
            bool((self.seeded_schedules()[1] or {}).get("given_order"))

    def bounce(self, hits, out=None, order=None):
        """One diffuse bounce per primary hit (rt_batch_bounce_rays: hit ids are instance-local positions):
        (orig, dir, tmax, order), the order listing the active bounces first. The order is made when `order` is
        true, by default only when a traced schedule reads it (or before tune() has picked the schedules)."""
        if order is None:
            order = self.bounce_needs_order()
        return core.batch_bounce_rays(self.tree, self.ray_offsets, self.orig, self.dir, hits["id"], hits["t"], self.bounce_seed(),
                                      out=out, order=order)

    def primary(self, out_h1=None, out_b=None):
        """The primary hits and their bounces (h1, b): in one rt_batch_trace call that writes the bounces too (the
        packet schedule as each ray finishes) unless a schedule needs the generator's order; then the trace and
        bounce(). The bounces are the same rays either way."""
        if self.bounce_needs_order():
            h1 = core.batch_trace(self.tree, self.orig, self.dir, self.ray_offsets, out=out_h1, schedule=self.schedule_primary)
            return h1, self.bounce(h1, out=out_b)
        h1 = core.batch_trace(self.tree, self.orig, self.dir, self.ray_offsets, out=out_h1, schedule=self.schedule_primary,
                              bounce=(self.bounce_seed(), out_b))
        return h1, h1["b"]

    def bounce_order(self, b):
        """The tracing order of the bounce launch: the generator's active-first order when the bounce schedule asks
        for it, else None (the schedule's own)."""
        return b[3] if (self.schedule_bounce or {}).get("given_order") else None

    def tune(self):
        """Pick the batched traversal schedules on this frame's rays (untimed): the primary launch's on the
        primary rays (8 x 4 pixel tiles of each instance's image are a candidate), the bounce launch's on their
        bounces (ray orders by instance, octant and origin, and the pixel tiles of the primaries they leave, are
        candidates). Returns both and their timings."""
        from . import tune
        self.schedule_primary, t1 = tune.tune_batch_trace(self.tree, self.orig, self.dir, self.ray_offsets, use_cache=False,
                                                          images=(self.count, self.width, self.height))
        h1 = core.batch_trace(self.tree, self.orig, self.dir, self.ray_offsets, schedule=self.schedule_primary)
        b = self.bounce(h1, order=True)
        self.schedule_bounce, t2 = tune.tune_batch_trace(self.tree, b[0], b[1], self.ray_offsets, tmax=b[2], use_cache=False,
                                                         order=b[3], images=(self.count, self.width, self.height))
        # the seeded walks go through the node records: the fastest schedule of those for each launch
        self.seeded_primary = min((x for x in t1 if not x[0].get("clusters")), key=lambda x: x[1])[0]
        self.seeded_bounce = min((x for x in t2 if not x[0].get("clusters")), key=lambda x: x[1])[0]
        return (self.schedule_primary, self.schedule_bounce), (t1, t2)

    def seeded_schedules(self):
        """Schedules of the seeded (learned) launches: tune()'s fastest node-record schedules, else the plain ones
        (which then must not walk the cluster tree: seeded walks start inside the node tree)."""
        sp = getattr(self, "seeded_primary", None) or self.schedule_primary
        sb = getattr(self, "seeded_bounce", None) or self.schedule_bounce
        return sp, sb

    def seeded_order(self, b):
        """The bounce tracing order of the seeded launch (see bounce_order)."""
        return b[3] if (self.seeded_schedules()[1] or {}).get("given_order") else None

    def trace_plain(self, out=None):
        """Primary hits, bounce rays and bounce hits through rt_batch_trace (the bounces made by the primary call
        where the schedules allow, see primary())."""
        out = out or {}
        h1, b = self.primary(out.get("h1"), out.get("b"))
        h2 = core.batch_trace(self.tree, b[0], b[1], self.ray_offsets, tmax=b[2], out=out.get("h2"), schedule=self.schedule_bounce,
                              order=self.bounce_order(b))
        return dict(h1=h1, b=b, h2=h2)

    def trace_learned(self, out=None, in_proposal: bool = False):
        """The same through the grouped proposal and rt_batch_trace_seeded."""
        out = out or {}
        R = self.rays_per_instance
        p1 = self.nets.propose(self.orig, self.dir, self.box, R, out=out.get("p1"))
        sp, sb = self.seeded_schedules()
        h1 = proposal.batch_trace_seeded(self.tree, self.orig, self.dir, self.ray_offsets, p1, self.slots, in_proposal=in_proposal,
                                         out=out.get("h1"), schedule=sp)
        b = self.bounce(h1, out=out.get("b"))
        p2 = self.nets.propose(b[0], b[1], self.box, R, out=out.get("p2"), tmax=b[2])  # bounces of misses are inactive
        h2 = proposal.batch_trace_seeded(self.tree, b[0], b[1], self.ray_offsets, p2, self.slots, tmax=b[2], in_proposal=in_proposal,
                                         out=out.get("h2"), schedule=sb, order=self.seeded_order(b))
        return dict(p1=p1, h1=h1, b=b, p2=p2, h2=h2)

    def labels(self, plain):
        """Per-instance slot labels of the frame's primary and bounce rays (-1 for misses)."""
        l1 = proposal.batch_hit_labels(self.tree, plain["h1"]["id"], self.ray_offsets, self.slots["pos_label"])
        l2 = proposal.batch_hit_labels(self.tree, plain["h2"]["id"], self.ray_offsets, self.slots["pos_label"])
        return l1, l2

    def remember(self, plain):
        """Keep this frame's rays, labels and per-instance lists of the rays
        that hit, for the next frame's fine-tuning."""
        l1, l2 = self.labels(plain)
        b = plain["b"]
        s1 = proposal.group_select(l1, self.count, self.rays_per_instance)
        s2 = proposal.group_select(l2, self.count, self.rays_per_instance)
        self.prev = (b[0].clone(), b[1].clone(), l1, l2, s1, s2)

    def fine_tune(self, steps: int | None = None):
        """Grouped Adam steps on the previous frame's rays that hit: even steps
        take primary rays, odd steps bounce rays; each instance walks its list
        of hits with a stride of HOP entries, so that a batch spreads over the
        whole image."""
        if self.prev is None:
            return None
        steps = self.steps if steps is None else steps
        bo, bd, l1, l2, s1, s2 = self.prev
        net, B, R = self.nets, self.batch, self.rays_per_instance
        ws = net._workspace(B, True)
        gb = (ws["bo"], ws["bd"], ws["bl"])
        loss = None
        for j in range(steps):
            o, d, lab, sel = (self.orig, self.dir, l1, s1) if j % 2 == 0 else (bo, bd, l2, s2)
            proposal.gather_batch(o, d, lab, self.count, R, (j // 2) * B, B, gb, index=sel[0], count=sel[1], hop=HOP)
            loss = net.train_step(gb[0], gb[1], gb[2], self.box, B, lr=self.lr)
        return loss
