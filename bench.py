"""Benchmark: LBVH build + closest-hit traversal, headline on the instanced-frame workload.

Headline workload (one "step" = one frame of the plain path): 64 deformed
instances of the 4,022,242-triangle terrain + soup scene at 1/16 size
(251,518 triangles each, 16,097,152 per frame). Every frame each instance's
vertices move by fresh N(0, 0.002^2) noise (input generation, outside the
timed events), then the timed frame runs: one batched LBVH build of all 64
instances, 64 pinhole cameras' primary rays (a 3840 x 2160 frame at 4 samples
per pixel, 480 x 270 tiles rendered at 960 x 540 each), the batched
closest-hit trace, one cosine-weighted diffuse bounce per hit and the batched
trace of the bounces. `value` = closest-hit rays (primaries + active bounces)
per frame / frame time, in Mrays/s; `build` = the frame's LBVH build in Mtri/s;
`nn_over_plain` = the learned proposal path (grouped per-instance networks +
seeded traversal) against the plain traversal on the same rays, hits compared
bit for bit.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Output: one JSON line per secondary workload ({"leg": ...}: the 128^2 terrain,
the 2^20-face soup, the 16M-face build, the 1024-mesh batch, the 4M-triangle
learned scene, SAH / Hybrid trees, the rasteriser), then the headline line last.
With N > 1 (torchrun, one rank per GPU) every rank runs its own replica of the
workload (weak scaling); times are the max over ranks.
`--impl reference` times the reference algorithm's CPU implementation (the
oracle restatement, checked bit-exact against the reference's own code; the
reference's GPU code cannot be built with CUDA 12) on the host cores, on rank 0
only, on a bounded sample of the same frame workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "closest-hit Mrays/s (plain vs NN-proposal, bit-exact) and LBVH build Mtri/s"
WORKLOAD_SHORT = "c4 instanced frames: 64 x 251,518-tri instances rebuilt per frame, 3840x2160 at 4 spp + 1 bounce"
WORKLOAD = ("instanced frames: 64 deformed instances of the terrain + soup scene at 1/16 size (16,097,152 triangles rebuilt per "
            "frame), 3840x2160 at 4 spp over 64 cameras (33,177,600 primary rays) + 1 diffuse bounce per hit")
SEED_MESH = 1
SEED_BOUNCE = 1234
L2_FLUSH_BYTES = 512 << 20  # > 126 MB L2
C4_SCALE, C4_W, C4_H = 1 / 16, 960, 540


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-legs", action="store_true", help="only the oracle port on the host cores for c0-c3 (no GPU work)")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--nn-frames", type=int, default=3, help="frames of the learned path (fine-tuning + proposals) timed beside plain")
    ap.add_argument("--legs", default="c0,c1,build16m,c2,c3,sah,raster",
                    help="secondary workloads printed before the headline line (comma list, or 'none')")
    return ap.parse_args()


def emit(obj):
    print(json.dumps(obj, separators=(",", ":")), flush=True)


def capture_graphs(stages):
    """One CUDA graph per callable (each run once eagerly first, on a side stream).
    Returns the graphs and the number of this library's kernel launches they hold."""
    import torch

    from cudart_b200 import _abi

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    graphs = []
    with torch.cuda.stream(side):
        for fn in stages:
            fn()
        torch.cuda.synchronize()
        n0 = _abi.lib().rt_launch_count()
        for fn in stages:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                fn()
            graphs.append(g)
        kernels = _abi.lib().rt_launch_count() - n0
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    return graphs, int(kernels)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(key: str):
    """DRAM bytes (read + write) per launch of one kernel on one workload, from the committed ncu capture
    summary profiles/trace_traffic.json (a figure of an earlier capture, not of this run)."""
    p = os.path.join(ROOT, "profiles", "trace_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(key)
    return None


def max_over_ranks(values, world, dev):
    if world == 1:
        return values
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def trace_roofline(kernel, launch, model_bytes, ms, ray_slots, peak, peak_kind, traffic_key):
    """Roofline of one trace launch. The bound that applies is HBM; `frac` is the DRAM fraction: ncu's DRAM
    bytes per launch (a committed capture of this kernel on this workload) over the live launch time. The
    per-ray model bytes (32 B ray + 16 B hit per slot, 32 B per box record read, 48 B per triangle tested)
    include every node and triangle read that L1 / L2 serve; they are reported as `model_frac`, not as HBM."""
    t = load_traffic(traffic_key)
    traffic = None if t is None else int(t["dram_bytes_per_launch"])
    model_gbs = model_bytes / (ms * 1e-3) / 1e9
    out = {"bound": "hbm", "kernel": kernel, "launch": launch, "ray_slots": ray_slots, "launch_ms": round(ms, 3), "unit": "GB/s",
           "peak": peak, "peak_kind": peak_kind, "traffic": traffic,
           "model_bytes": int(model_bytes), "model_gbs": round(model_gbs, 1), "model_frac": round(model_gbs / peak, 4),
           "model_note": "per-ray bytes incl. L1/L2-served node and triangle reads (not DRAM)"}
    if traffic is not None:
        a = traffic / (ms * 1e-3) / 1e9
        out.update(achieved=round(a, 1), frac=round(a / peak, 4), traffic_source=t.get("source", ""), l1_frac=t.get("l1tex_frac"),
                   limiter=t.get("limiter"))
    else:
        out.update(achieved=None, frac=None, traffic_source="no capture of this kernel on this workload")
    return out


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons (every 20 ms, from
    before the timed region until after it); the summary keeps the samples
    taken inside the timed window (or the nearest one when the window is short)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.samples = []  # (monotonic time, sm_mhz, max_mhz, reason flags)
        self.t0 = self.t1 = None

    def _reader(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                self.samples.append((time.monotonic(), float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue

    def start(self):
        import threading
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self
        self.thread = threading.Thread(target=self._reader, daemon=True)
        self.thread.start()
        deadline = time.monotonic() + 10.0
        while not self.samples and time.monotonic() < deadline:
            time.sleep(0.01)
        return self

    def __enter__(self):
        self.t0 = time.monotonic()
        return self

    def __exit__(self, *a):
        self.t1 = time.monotonic()
        time.sleep(0.05)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples or self.t0 is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        rows = [r for r in self.samples if self.t0 <= r[0] <= self.t1]
        if not rows:
            rows = [min(self.samples, key=lambda r: abs(r[0] - self.t1))]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for _, _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": max(r[2] for r in rows), "reasons": reasons,
                "samples": len(rows)}


# ----------------------------------------------------------------------------
# headline: instanced frames (plain path timed per frame; learned path beside it)
# ----------------------------------------------------------------------------
def batch_kernel(sched):
    base = "k_batch_trace_clusters" if sched.get("clusters") else "k_batch_trace"
    if sched.get("clusters") and sched.get("persistent"):
        if sched.get("packet"):
            return base + "_packet"
        if sched.get("refill"):
            return base + "_refill"
    if sched.get("coop"):
        return base + "_coop"
    return base + "_persistent" if sched.get("persistent") else base


def run_headline(args, rank, world, local_rank):
    import torch

    from cudart_b200 import _abi, core
    from cudart_b200.instances import InstancedFrames

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if not core.device_check():
        raise RuntimeError("no CUDA device: the CUDA path has no CPU fallback")
    w = InstancedFrames(args.instances, C4_SCALE, C4_W, C4_H, device=dev)
    w.displace(0)
    w.build()
    w.make_slots()
    (s1, s2), (tim1, tim2) = w.tune()  # untimed; results never depend on the schedules
    plain = w.trace_plain()
    torch.cuda.synchronize()
    R = w.ray_count
    F = w.face_count
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    # the primary call also writes the bounce rays (the packet walk, as each ray finishes) unless the bounce
    # schedule reads the generator's order; then the bounces are a stage of their own
    fused = not w.bounce_needs_order()

    def trace1():
        if fused:
            w.primary(plain["h1"], plain["b"])
        else:
            core.batch_trace(w.tree, w.orig, w.dir, w.ray_offsets, out=plain["h1"], schedule=s1)

    def trace2():
        b = plain["b"]
        core.batch_trace(w.tree, b[0], b[1], w.ray_offsets, tmax=b[2], out=plain["h2"], schedule=s2, order=w.bounce_order(b))

    aux = torch.cuda.Stream()  # the primary rays run beside the build (they do not depend on it)
    stages = [lambda: w.build_and_rays(aux=aux), trace1] + ([] if fused else [lambda: w.bounce(plain["h1"], out=plain["b"])]) + [trace2]
    graphs, kernels_per_step = capture_graphs(stages)
    active = torch.zeros(1, dtype=torch.int64, device=dev)

    def step(frame, timed_list=None):
        w.displace(frame)  # the frame's input (outside the events)
        flush.zero_()  # L2 flush between frames (outside the events)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(graphs) + 1)]
        ev[0].record(stream)
        for i, g in enumerate(graphs):
            g.replay()
            ev[i + 1].record(stream)
        if timed_list is not None:
            timed_list.append(ev)
            active.add_((plain["b"][2] > 0).sum())  # rays of the frame (counted after its last event)

    for k in range(args.warmup):
        step(1 + k)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    evs = []
    sampler = ClockSampler(local_rank).start()
    with sampler as clk:
        for k in range(args.steps):
            step(1 + args.warmup + k, evs)
        torch.cuda.synchronize()
    sampler.stop()
    K = args.steps
    frame_ms = sum(e[0].elapsed_time(e[-1]) for e in evs)
    build_ms = sum(e[0].elapsed_time(e[1]) for e in evs)  # the build, with the primary rays made beside it
    t1_ms = sum(e[1].elapsed_time(e[2]) for e in evs)  # the primary trace (with the bounce rays when fused)
    bounce_gen_ms = 0.0 if fused else sum(e[2].elapsed_time(e[3]) for e in evs)
    t2_ms = sum(e[-2].elapsed_time(e[-1]) for e in evs)
    frame_ms, build_ms, t1_ms, bounce_gen_ms, t2_ms = max_over_ranks([frame_ms, build_ms, t1_ms, bounce_gen_ms, t2_ms], world, dev)
    rays_total = K * R + int(active.item())
    value = world * rays_total / (frame_ms * 1e-3) / 1e6
    info = w.tree.info.cpu().numpy()
    nodes_total = int(info[:, 0].astype(np.int64).sum())
    dev_errors = int((info[:, 7] != 0).sum())
    hits1 = int((plain["h1"]["id"] >= 0).sum().item())
    active_last = int((plain["b"][2] > 0).sum().item())

    # counted launches (untimed) of the last frame's rays: box records read and triangles tested per ray
    b = plain["b"]
    c1 = core.batch_trace(w.tree, w.orig, w.dir, w.ray_offsets, counters=True, schedule=s1)
    c2 = core.batch_trace(w.tree, b[0], b[1], w.ray_offsets, tmax=b[2], counters=True, schedule=s2, order=w.bounce_order(b))
    torch.cuda.synchronize()
    same = torch.equal(c1["id"], plain["h1"]["id"]) and torch.equal(c2["id"], plain["h2"]["id"])
    m1 = 48 * R + 32 * int(c1["visits"].sum().item()) + 48 * int(c1["tests"].sum().item())
    m2 = 48 * R + 32 * int(c2["visits"].sum().item()) + 48 * int(c2["tests"].sum().item())
    del c1, c2
    peak, peak_kind = load_peaks()
    if t1_ms >= t2_ms:
        kname = batch_kernel(s1)
        roof = trace_roofline(kname, "primary", m1, t1_ms / K, R, peak, peak_kind, f"c4:{kname}:primary")
    else:
        kname = batch_kernel(s2)
        roof = trace_roofline(kname, "bounce", m2, t2_ms / K, R, peak, peak_kind, f"c4:{kname}:bounce")
    # build: algorithmic bytes per face = 16 face + 48 vertices + 32 box + 8 code/index + 64 sort + 4 split scan
    # + 32 leaf gather + 36 reorder + 48 triangle stream, + 64 per node (write + child read)
    build_bytes = F * (16 + 48 + 32 + 8 + 64 + 4 + 32 + 36 + 48) + 64 * nodes_total
    if w.clusters:  # cluster trees: codes + triangles read, position and node boxes, child pairs, arrival words
        build_bytes += F * (4 + 48 + 32 + 32 + 8 + 4)
    bgbs = build_bytes / (build_ms / K * 1e-3) / 1e9
    result = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": round(frame_ms / K, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic, seeded",
        "config": {"workload": WORKLOAD_SHORT, "faces": F, "primary_rays": R, "rays_per_step": round(rays_total / K),
                   "l2": "flushed between frames; inputs > L2"},
        "build": {"value": round(world * F * K / (build_ms * 1e-3) / 1e6, 1), "unit": "Mtri/s", "ms": round(build_ms / K, 3),
                  "roofline": {"bound": "hbm", "achieved": round(bgbs, 1), "peak": peak, "unit": "GB/s", "frac": round(bgbs / peak, 4)}},
        "trace": {"mrays_s": round(world * rays_total / ((t1_ms + t2_ms) * 1e-3) / 1e6, 1), "primary_ms": round(t1_ms / K, 3),
                  "bounce_ms": round(t2_ms / K, 3)},
        "roofline": {k: roof.get(k) for k in ("bound", "kernel", "launch", "launch_ms", "achieved", "peak", "unit", "frac", "traffic",
                                              "model_frac", "l1_frac", "limiter")},
        "gpu_launches": int(kernels_per_step * K),
    }
    clocks = clk.summary()
    result["clocks"] = {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"], "reasons": clocks["reasons"],
                        "samples": clocks["samples"]}
    legs = {"c4_tuning": {"primary_ms": {json.dumps(k, sort_keys=True): round(v, 3) for k, v in tim1},
                          "bounce_ms": {json.dumps(k, sort_keys=True): round(v, 3) for k, v in tim2}},
            "c4_detail": {"workload": WORKLOAD, "schedule_primary": s1, "schedule_bounce": s2, "counted_identical": bool(same), "device_errors": dev_errors,
                          "nodes": nodes_total, "build_bytes": int(build_bytes),
                          "bounce_rays_ms": "in the primary trace" if fused else round(bounce_gen_ms / K, 3),
                          "primary_hits_last": hits1, "active_bounces_last": active_last, "kernels_per_frame": kernels_per_step,
                          "graphs": (f"{len(stages)} CUDA graph replays per frame: build with the primary rays made beside it (one "
                                     "rt_batch_primary_rays launch on a second stream), trace"
                                     + (" writing the bounce rays, trace" if fused else ", bounce rays, trace")),
                          "roofline": roof}}
    del graphs
    # learned proposal on the same frames (fine-tuning, grouped proposals + seeded traversal), hits bit for bit
    if args.nn_frames > 0:
        legs["c4_learned"] = learned_frames(w, args, dev, world, plain, first_frame=1 + args.warmup + K)
        nn = legs["c4_learned"]
        result["nn_over_plain"] = nn["nn_over_plain"]
        result["nn"] = {k: nn[k] for k in ("bit_exact", "proposal_accuracy", "oracle_seeded_over_plain")}
    if not args.no_e2e:
        e2e = run_e2e(w, args, dev, world, s1, s2)
        legs["c4_e2e"] = e2e
        result["e2e"] = {k: e2e[k] for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step", "ms_per_step")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_c4(w.count, frame=0, steps=1, one_thread=True)
        legs["c4_cpu_baseline"] = cb
        result["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "value_1_thread")}
        result["cpu_baseline"]["sample"] = f"1/{w.count} frame (1 instance built + all its rays), oracle port"
    del flush
    return result, legs


def learned_frames(w, args, dev, world, plain, first_frame):
    """`nn_frames` frames of the learned path beside the plain one: each frame rebuilds, fine-tunes every
    instance's network (200 grouped Adam steps of 1024 rays) on the previous frame's plain hits, then traces
    the frame plain and through the grouped proposals + seeded traversal; all hits compared bit for bit. The
    `oracle` figure seeds every ray with the slot its plain hit lies in: what a perfect proposal gives."""
    import torch

    from cudart_b200 import proposal

    w.remember(plain)
    learned = w.trace_learned()
    sp, sb = w.seeded_schedules()
    torch.cuda.synchronize()
    ev = []
    mism = torch.zeros(1, dtype=torch.int64, device=dev)
    inprop = torch.zeros(2, dtype=torch.int64, device=dev)
    for f in range(args.nn_frames):
        w.displace(first_frame + f)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(7)]
        w.build()
        w.make_slots()
        e[0].record()
        w.fine_tune()
        e[1].record()
        w.trace_plain(out=plain)
        e[2].record()
        R = w.rays_per_instance
        learned["p1"] = w.nets.propose(w.orig, w.dir, w.box, R, out=learned["p1"])
        e[3].record()
        proposal.batch_trace_seeded(w.tree, w.orig, w.dir, w.ray_offsets, learned["p1"], w.slots, in_proposal=True,
                                    out=learned["h1"], schedule=sp)
        e[4].record()
        b = plain["b"]  # the seeded hits equal the plain ones, so the bounces are the same rays
        learned["p2"] = w.nets.propose(b[0], b[1], w.box, R, out=learned["p2"], tmax=b[2])
        e[5].record()
        proposal.batch_trace_seeded(w.tree, b[0], b[1], w.ray_offsets, learned["p2"], w.slots, tmax=b[2], in_proposal=True,
                                    out=learned["h2"], schedule=sb, order=w.seeded_order(b))
        e[6].record()
        for k in ("h1", "h2"):
            mism += (plain[k]["id"] != learned[k]["id"]).sum() + (plain[k]["t"].view(torch.int32) != learned[k]["t"].view(torch.int32)).sum()
            mism += (plain[k]["uv"].view(torch.int32) != learned[k]["uv"].view(torch.int32)).sum()
            hit = plain[k]["id"] >= 0
            inprop[0] += (learned[k]["in_proposal"].bool() & hit).sum()
            inprop[1] += hit.sum()
        w.remember(plain)
        ev.append(e)
    torch.cuda.synchronize()
    n = args.nn_frames
    tune_ms = sum(e[0].elapsed_time(e[1]) for e in ev) / n
    plain_ms = sum(e[1].elapsed_time(e[2]) for e in ev) / n
    mlp_ms = sum(e[2].elapsed_time(e[3]) + e[4].elapsed_time(e[5]) for e in ev) / n
    seeded_ms = sum(e[3].elapsed_time(e[4]) + e[5].elapsed_time(e[6]) for e in ev) / n
    # a perfect proposal (the slot of each ray's plain hit), seeded traversal only
    l1, l2 = w.labels(plain)
    torch.cuda.synchronize()
    o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    o0.record()
    proposal.batch_trace_seeded(w.tree, w.orig, w.dir, w.ray_offsets, l1, w.slots, out=learned["h1"], schedule=sp)
    b = plain["b"]
    proposal.batch_trace_seeded(w.tree, b[0], b[1], w.ray_offsets, l2, w.slots, tmax=b[2], out=learned["h2"], schedule=sb,
                                order=w.seeded_order(b))
    o1.record()
    torch.cuda.synchronize()
    oracle_ms = o0.elapsed_time(o1)
    plain_ms, mlp_ms, seeded_ms, tune_ms, oracle_ms = max_over_ranks([plain_ms, mlp_ms, seeded_ms, tune_ms, oracle_ms], world, dev)
    return {"frames": n, "bit_exact": int(mism.item()) == 0,
            "proposal_accuracy": round(int(inprop[0].item()) / max(1, int(inprop[1].item())), 4),
            "finetune_ms": round(tune_ms, 2), "plain_ms": round(plain_ms, 3), "mlp_ms": round(mlp_ms, 3), "seeded_ms": round(seeded_ms, 3),
            "nn_over_plain": round(plain_ms / (mlp_ms + seeded_ms), 4), "seeded_only_over_plain": round(plain_ms / seeded_ms, 4),
            "oracle_seeded_over_plain": round(plain_ms / oracle_ms, 4),
            "note": "nn = grouped MLP proposals + seeded traversal of primaries and bounces; fine-tuning reported apart"}


def run_e2e(w, args, dev, world, s1, s2):
    """The headline metric through the public API with host buffers, as a frame pipeline: every frame copies
    the 64 instances' displaced vertices from pinned host memory, builds, makes the primary rays, traces them
    and their bounces, and brings every hit of both launches back to pinned host memory: the ids of all rays,
    then the (t, u, v) of the rays that hit, packed on the device by rt_pack_hits (a miss is t = its tmax,
    uv = 0, so the host has every hit exactly; the last frame's are rebuilt and checked). The copies run on two
    copy streams (one per direction) with the device vertices and hits double-buffered, so that frame k+1's
    upload and frame k-1's download overlap frame k's kernels (one CUDA graph per buffer set); the host reads a
    frame's hit counts before it sizes that frame's packed copies, one frame behind. The timed region holds
    every frame's copies and kernels. The faces (the instances' fixed topology) stay resident."""
    import torch

    from cudart_b200 import core

    vh = w.verts.cpu().pin_memory()
    R = w.ray_count
    comp = torch.cuda.current_stream()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    v = [torch.empty_like(w.verts) for _ in range(2)]
    for s in range(2):
        v[s].copy_(vh)
    outs = [w.trace_plain() for _ in range(2)]
    packs = [[core.pack_hits(outs[s][h]) for h in ("h1", "h2")] for s in range(2)]
    out_id = torch.empty((2, 2, R), dtype=torch.int32).pin_memory()
    out_cnt = torch.zeros((2, 2), dtype=torch.int32).pin_memory()
    out_pk = torch.empty((2, 2, 3 * R), dtype=torch.float32).pin_memory()
    ev = {k: [torch.cuda.Event(), torch.cuda.Event()] for k in ("uploaded", "traced", "ids_down", "downloaded")}

    aux = torch.cuda.Stream()

    def compute(s):
        w.build_and_rays(v[s], aux=aux)
        o = outs[s]
        w.primary(o["h1"], o["b"])
        core.batch_trace(w.tree, o["b"][0], o["b"][1], w.ray_offsets, tmax=o["b"][2], out=o["h2"], schedule=s2,
                         order=w.bounce_order(o["b"]))
        for i, h in enumerate(("h1", "h2")):
            core.pack_hits(o[h], out=packs[s][i])

    graphs, _ = capture_graphs([lambda: compute(0), lambda: compute(1)])
    packed_bytes = [0]

    def finish(j):
        # frame j's hit counts are on the host once its id copies are: size and queue its packed copies
        s = j % 2
        ev["ids_down"][s].synchronize()
        with torch.cuda.stream(down):
            for i in range(2):
                n = int(out_cnt[s, i])
                out_pk[s, i, :3 * n].copy_(packs[s][i]["packed"][:3 * n], non_blocking=True)
                packed_bytes[0] += 12 * n
        ev["downloaded"][s].record(down)

    def step(k):
        s = k % 2
        if k >= 2:
            up.wait_event(ev["traced"][s])  # frame k-2's kernels are done with this vertex buffer
        with torch.cuda.stream(up):
            v[s].copy_(vh, non_blocking=True)
        ev["uploaded"][s].record(up)
        comp.wait_event(ev["uploaded"][s])
        if k >= 2:
            comp.wait_event(ev["downloaded"][s])  # frame k-2's hits have reached the host
        graphs[s].replay()
        ev["traced"][s].record(comp)
        if k >= 1:
            finish(k - 1)
        down.wait_event(ev["traced"][s])
        with torch.cuda.stream(down):
            for i, h in enumerate(("h1", "h2")):
                out_id[s, i].copy_(outs[s][h]["id"], non_blocking=True)
                out_cnt[s, i].copy_(packs[s][i]["count"][0], non_blocking=True)
        ev["ids_down"][s].record(down)

    for k in range(args.warmup):
        step(k)
    finish(args.warmup - 1)
    torch.cuda.synchronize()
    active = sum(int((outs[s]["b"][2] > 0).sum().item()) for s in range(2)) / 2.0
    packed_bytes[0] = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(comp)
    up.wait_event(e0)
    down.wait_event(e0)
    for k in range(args.steps):
        step(k)
    finish(args.steps - 1)
    comp.wait_event(ev["downloaded"][(args.steps - 1) % 2])
    e1.record(comp)
    torch.cuda.synchronize()
    ms, = max_over_ranks([e0.elapsed_time(e1)], world, dev)
    # the last frame's hits rebuilt on the host from its ids and packed hits equal the device's, bit for bit
    s = (args.steps - 1) % 2
    ok = True
    for i, h in enumerate(("h1", "h2")):
        tm = None if h == "h1" else outs[s]["b"][2].cpu()
        t, uv = core.unpack_hits(out_id[s, i], out_pk[s, i], int(out_cnt[s, i]), tmax=tm)
        d = outs[s][h]
        ok = ok and torch.equal(out_id[s, i], d["id"].cpu()) and torch.equal(t.view(torch.int32), d["t"].cpu().view(torch.int32)) \
            and torch.equal(uv.view(torch.int32), d["uv"].cpu().view(torch.int32))
    h2d = vh.numel() * 4
    d2h = out_id[0].numel() * 4 + out_cnt[0].numel() * 4 + packed_bytes[0] / args.steps
    del graphs
    return {"value": round(world * (R + active) * args.steps / (ms * 1e-3) / 1e6, 2), "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": round(ms / args.steps, 3), "download_checked": bool(ok),
            "pipeline": "vertices up / ids, hit counts and packed hits down on two copy streams, double-buffered around one CUDA "
                        "graph per frame"}


# ----------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle (the reference algorithm restated in
# C++, checked against the reference's own code) on the host cores
# ----------------------------------------------------------------------------
_C4_HOST = {}


def c4_host_scene(count):
    """Host copy of the instanced scene: base mesh and the instances' cameras (the same generators as the GPU arm)."""
    if count not in _C4_HOST:
        from cudart_b200 import scenes
        _C4_HOST[count] = (scenes.learned_scene(C4_SCALE), scenes.instance_cameras(count, C4_W, C4_H))
    return _C4_HOST[count]


def c4_instance_sample(count, frame, threads, ray_stride=1):
    """One instance of one frame on the host cores: its displaced vertices (numpy N(0, 0.002^2), seeded by the
    frame and instance), its LBVH build, its camera's primary rays (every `ray_stride`-th) traced, their
    diffuse bounces traced. Returns (seconds, rays traced, faces built, seconds of the build)."""
    from oracle import api as O

    base, cams = c4_host_scene(count)
    i = frame % count
    rng = np.random.default_rng(7_000_003 + 64 * frame + i)
    verts = base.vertices.copy()
    verts[:, :3] += rng.normal(0.0, 0.002, size=(len(verts), 3)).astype(np.float32)
    o, d, _, _ = O.primary_rays(cams[i])
    if ray_stride > 1:
        o, d = np.ascontiguousarray(o[::ray_stride]), np.ascontiguousarray(d[::ray_stride])
    O.set_threads(threads)
    t0 = time.perf_counter()
    ref = O.lbvh_build(verts, base.faces)
    t_build = time.perf_counter() - t0
    e = O.trace(ref["nodes"], ref["tris"], ref["indices"], o, d, threads=threads)
    bo, bd, bt = O.bounce_rays(ref["tris"], o, d, e["id"], e["t"], 1000 + frame)
    O.trace(ref["nodes"], ref["tris"], ref["indices"], bo, bd, bt, threads=threads)
    total = time.perf_counter() - t0
    O.set_threads(0)
    return total, len(o) + int((bt > 0).sum()), base.face_count, t_build


def cpu_baseline_c4(count, frame=0, steps=1, one_thread=True):
    """The frame workload's rate on the host cores: instance (frame mod count) of a frame, built and traced
    whole (1/count of the frame) with all threads; the 1-thread figure on every 16th of its primary rays."""
    from oracle import api as O

    cores = O.max_threads()
    c4_instance_sample(count, frame, cores, ray_stride=64)  # load the library, page the scene in
    vals, builds = [], []
    for k in range(steps):
        sec, rays, faces, tb = c4_instance_sample(count, frame + k, cores)
        vals.append(rays / sec / 1e6)
        builds.append(faces / tb / 1e6)
    out = {"value": round(statistics.median(vals), 4), "unit": "Mrays/s", "cores": cores, "kind": "port",
           "sample": f"1/{count} of a frame per step: one instance's build ({faces} faces) + its {C4_W * C4_H} primary rays "
                     f"and their bounces ({rays} rays), oracle port, all {cores} threads",
           "build_mtri_s": round(statistics.median(builds), 3)}
    if one_thread:
        sec, rays, faces, tb = c4_instance_sample(count, frame, 1, ray_stride=16)
        out["value_1_thread"] = round(rays / sec / 1e6, 4)
        out["build_mtri_s_1_thread"] = round(faces / tb / 1e6, 3)
    return out


def cpu_legs():
    """--cpu-legs: the oracle port (the reference algorithm) on the host cores for the secondary configs, each
    with all threads and with one: LBVH build Mtri/s and closest-hit Mrays/s on a bounded sample of the leg's
    rays (primaries and their bounces where the GPU leg traces bounces). c0 terrain (512 x 512 rays), c1 2^20-face
    soup (1920 x 1080 rays), c2 every 32nd mesh of the 1024-mesh batch (32 x 32 sphere rays each), c3 the
    4,022,242-face scene (rays uniform in its box, as the GPU leg's evaluation rays). One JSON line per leg."""
    import torch

    from cudart_b200 import scenes
    from oracle import api as O

    cores = O.max_threads()

    def run(mesh, o, d, bounce, threads, stride):
        o, d = np.ascontiguousarray(o[::stride]), np.ascontiguousarray(d[::stride])
        O.set_threads(threads)
        t0 = time.perf_counter()
        ref = O.lbvh_build(mesh.vertices, mesh.faces)
        t1 = time.perf_counter()
        e = O.trace(ref["nodes"], ref["tris"], ref["indices"], o, d, threads=threads)
        rays = len(o)
        if bounce:
            bo, bd, bt = O.bounce_rays(ref["tris"], o, d, e["id"], e["t"], SEED_BOUNCE)
            O.trace(ref["nodes"], ref["tris"], ref["indices"], bo, bd, bt, threads=threads)
            rays += int((bt > 0).sum())
        t2 = time.perf_counter()
        O.set_threads(0)
        return mesh.face_count / (t1 - t0) / 1e6, rays / (t2 - t1) / 1e6

    def leg(name, meshes_rays, bounce, stride_all, stride_one, note):
        res = {"leg": f"cpu_{name}", "kind": "port", "cores": cores}
        for label, threads, stride in (("all", cores, stride_all), ("1_thread", 1, stride_one)):
            builds, rates = [], []
            for mesh, o, d in meshes_rays:
                b, r = run(mesh, o, d, bounce, threads, stride)
                builds.append(b)
                rates.append(r)
            res[f"build_mtri_s_{label}"] = round(statistics.median(builds), 3)
            res[f"mrays_s_{label}"] = round(statistics.median(rates), 4)
        res["sample"] = note
        emit(res)

    m, cam = scenes.terrain_small_scene()
    o, d, _, _ = O.primary_rays(cam)
    leg("c0", [(m, o, d)], True, 1, 4, "terrain 32,258 faces; all 262,144 primaries + bounces (1 thread: every 4th)")
    m, cam = scenes.soup_1m_scene()
    o, d, _, _ = O.primary_rays(cam)
    leg("c1", [(m, o, d)], True, 8, 64, "soup 2^20 faces; every 8th of 2,073,600 primaries + bounces (1 thread: every 64th)")
    ms = scenes.batch_meshes(1024, seed=3)[::32]
    leg("c2", [(x, *scenes.sphere_rays(x, 32, seed=i)) for i, x in enumerate(ms)], False, 1, 1,
        "32 of the 1024 meshes (every 32nd), each built and traced with 32 x 32 sphere rays; medians over the meshes")
    m = scenes.learned_scene(1.0)
    eo, ed = scenes.box_rays_torch(1 << 18, scenes.scene_box(m, 1.5), seed=2, device="cpu")
    leg("c3", [(m, eo.numpy(), ed.numpy())], False, 1, 16, "4,022,242 faces; 262,144 rays uniform in the scene box (1 thread: every 16th)")


def run_reference(args, rank, world):
    if rank != 0:
        return None
    from oracle import api as O

    cores = O.max_threads()
    c4_instance_sample(args.instances, 0, cores, ray_stride=64)  # load the library, page the scene in
    vals, builds, secs = [], [], []
    for k in range(args.warmup + args.steps):
        sec, rays, faces, tb = c4_instance_sample(args.instances, k, cores)
        if k >= args.warmup:
            vals.append(rays / sec / 1e6)
            builds.append(faces / tb / 1e6)
            secs.append(sec)
    value = round(statistics.median(vals), 4)
    sample = (f"1/{args.instances} of a frame per step: instance (step mod {args.instances})'s build ({faces} faces) + its "
              f"{C4_W * C4_H} primary rays and their bounces, all {cores} threads")
    return {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(statistics.median(secs) * 1e3, 2), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded PCG64 scene, numpy N(0,0.002^2) displacement per frame and instance)",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "instances": args.instances, "tree_depth": 12, "parallelism": f"host cores ({cores} threads)"},
        "build": {"value": round(statistics.median(builds), 3), "unit": "Mtri/s"},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's GPU kernels use texture references and string-named symbol copies that CUDA 12 removed; "
                "its algorithm runs here as the oracle port (checked bit-exact against the reference's own code)",
    }


# ----------------------------------------------------------------------------
# secondary workloads (one JSON line each, before the headline)
# ----------------------------------------------------------------------------
def timed_ms(fn, flush, reps=5, agg=statistics.median):
    import torch
    fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return agg(ms)


def leg_single_scene(args, dev, world, mesh, cam, key, with_roofline=False):
    """One scene: LBVH build and the primary + bounce traces, each stage replayed from a CUDA graph, CUDA
    events between the replays, L2 flushed between steps, tuned schedules."""
    import torch

    from cudart_b200 import core, tune

    v = torch.from_numpy(mesh.vertices).to(dev)
    f = torch.from_numpy(mesh.faces.view(np.int32)).to(dev)
    N, W, H = mesh.face_count, cam.width, cam.height
    R = W * H
    camera = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    tree = core.build_lbvh(v, f, clusters=True)  # with the cluster tree: the tuner tries both trees' walks
    rays = core.primary_rays(camera, W, H)
    h1 = core.trace(tree, rays[0], rays[1])
    bounce = core.bounce_rays(tree.tris, rays[0], rays[1], h1["id"], h1["t"], SEED_BOUNCE)
    h2 = core.trace(tree, bounce[0], bounce[1], tmax=bounce[2])
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    s1, _ = tune.tune_trace(tree, rays[0], rays[1], image_width=W, key=f"{key}-primary", use_cache=False)
    s2, _ = tune.tune_trace(tree, bounce[0], bounce[1], tmax=bounce[2], image_width=W, key=f"{key}-bounce", use_cache=False)
    stages = [lambda: core.build_lbvh(v, f, out=tree, clusters=True), lambda: core.primary_rays(camera, W, H, out=rays),
              lambda: core.trace(tree, rays[0], rays[1], out=h1, schedule=s1),
              lambda: core.bounce_rays(tree.tris, rays[0], rays[1], h1["id"], h1["t"], SEED_BOUNCE, out=bounce),
              lambda: core.trace(tree, bounce[0], bounce[1], tmax=bounce[2], out=h2, schedule=s2)]
    graphs, kernels = capture_graphs(stages)
    steps = max(3, min(args.steps, 10))
    evs = []
    for k in range(args.warmup + steps):
        flush.zero_()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        ev[0].record()
        for i, g in enumerate(graphs):
            g.replay()
            ev[i + 1].record()
        if k >= args.warmup:
            evs.append(ev)
    torch.cuda.synchronize()
    build_ms = sum(e[0].elapsed_time(e[1]) for e in evs) / steps
    t1 = sum(e[2].elapsed_time(e[3]) for e in evs) / steps
    t2 = sum(e[4].elapsed_time(e[5]) for e in evs) / steps
    build_ms, t1, t2 = max_over_ranks([build_ms, t1, t2], world, dev)
    active = int((bounce[2] > 0).sum().item())
    info = tree.info_host()
    out = {"faces": N, "primary_rays": R, "active_bounces": active, "build_ms": round(build_ms, 4),
           "build_mtri_s": round(world * N / (build_ms * 1e-3) / 1e6, 1), "primary_ms": round(t1, 4), "bounce_ms": round(t2, 4),
           "mrays_s": round(world * (R + active) / ((t1 + t2) * 1e-3) / 1e6, 1), "nodes": info["node_count"],
           "schedule_primary": s1, "schedule_bounce": s2, "kernels_per_step": kernels}
    if with_roofline:
        c1 = core.trace(tree, rays[0], rays[1], counters=True, schedule=s1)
        c2 = core.trace(tree, bounce[0], bounce[1], tmax=bounce[2], counters=True, schedule=s2)
        torch.cuda.synchronize()
        m1 = 48 * R + 32 * int(c1["visits"].sum().item()) + 48 * int(c1["tests"].sum().item())
        m2 = 48 * R + 32 * int(c2["visits"].sum().item()) + 48 * int(c2["tests"].sum().item())
        peak, kind = load_peaks()

        def kname(sch):
            if sch.get("clusters"):
                if sch.get("persistent"):
                    for k in ("packet", "refill", "coop"):
                        if sch.get(k):
                            return "k_trace_clusters_" + k
                    return "k_trace_clusters_persistent"
                return "k_trace_clusters"
            if sch.get("coop"):
                return "k_trace_coop_persistent" if sch.get("persistent") else "k_trace_coop"
            return "k_trace_accel_persistent" if sch.get("persistent") else "k_trace_accel"
        out["roofline_primary"] = trace_roofline(kname(s1), "primary", m1, t1, R, peak, kind, kname(s1))
        out["roofline_bounce"] = trace_roofline(kname(s2), "bounce", m2, t2, R, peak, kind, kname(s2))
        bb = N * (16 + 48 + 32 + 8 + 64 + 4 + 32 + 36 + 48) + 64 * info["node_count"] + N * (4 + 48 + 32 + 32 + 8 + 4)
        a = bb / (build_ms * 1e-3) / 1e9
        out["build_roofline"] = {"bound": "hbm", "achieved": round(a, 1), "peak": peak, "unit": "GB/s", "frac": round(a / peak, 4)}
    del graphs, flush
    return out


def leg_build_16m(args, dev, world):
    """LBVH build alone on a 2^24-face soup, replayed from a CUDA graph, CUDA events, L2 flushed."""
    import torch

    from cudart_b200 import core, scenes

    mesh = scenes.soup(1 << 24, seed=7)
    v = torch.from_numpy(mesh.vertices).to(dev)
    f = torch.from_numpy(mesh.faces.view(np.int32)).to(dev)
    del mesh
    tree = core.build_lbvh(v, f)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    (graph,), kernels = capture_graphs([lambda: core.build_lbvh(v, f, out=tree)])
    ms = timed_ms(graph.replay, flush, reps=max(3, min(args.steps, 10)))
    ms, = max_over_ranks([ms], world, dev)
    info = tree.info_host()
    n = 1 << 24
    peak, _ = load_peaks()
    bb = n * (16 + 48 + 32 + 8 + 64 + 4 + 32 + 36 + 48) + 64 * info["node_count"]
    a = bb / (ms * 1e-3) / 1e9
    del graph, flush
    return {"faces": n, "mtri_s": round(world * n / (ms * 1e-3) / 1e6, 1), "ms": round(ms, 4), "nodes": info["node_count"],
            "kernels": kernels, "roofline": {"bound": "hbm", "achieved": round(a, 1), "peak": peak, "unit": "GB/s", "frac": round(a / peak, 4)}}


def leg_batch(args, dev, world, count=1024):
    """1024 independent meshes (face counts log-uniform in [64, 65536], terrain or soup by coin flip), each
    with side x side rays (side log-uniform in [64, 512]) from its bounding sphere aimed uniformly inward.
    One batched build and one batched trace, captured together in a CUDA graph and replayed."""
    import torch

    from cudart_b200 import core, scenes, tune

    meshes = scenes.batch_meshes(count, seed=3)
    verts, faces, fo, vo = scenes.concat_batch(meshes)
    orig, dirs, ro = scenes.batch_sphere_rays_torch(meshes, device=dev)
    R = int(ro[-1])
    del meshes
    V = torch.from_numpy(verts).to(dev)
    Fc = torch.from_numpy(faces.view(np.int32)).to(dev)
    roff = torch.tensor(ro.astype(np.int32), device=dev)
    tree = core.batch_build(V, Fc, fo, vo, clusters=True)
    sched, _ = tune.tune_batch_trace(tree, orig, dirs, roff, key=f"batch{count}", use_cache=False)  # untimed
    hits = core.batch_trace(tree, orig, dirs, roff, schedule=sched)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    (gb, gt), kernels = capture_graphs([lambda: core.batch_build(V, Fc, fo, vo, out=tree, clusters=True),
                                        lambda: core.batch_trace(tree, orig, dirs, roff, out=hits, schedule=sched)])
    bms = timed_ms(gb.replay, flush, reps=3)
    tms = timed_ms(gt.replay, flush, reps=3)
    bms, tms = max_over_ranks([bms, tms], world, dev)
    info = tree.info.cpu().numpy()
    N = int(fo[-1])
    del gb, gt, flush
    return {"meshes": count, "faces": N, "rays": R, "schedule": sched, "build_ms": round(bms, 4),
            "build_mtri_s": round(world * N / (bms * 1e-3) / 1e6, 1), "trace_ms": round(tms, 4),
            "trace_mrays_s": round(world * R / (tms * 1e-3) / 1e6, 1), "graph_mrays_s": round(world * R / ((bms + tms) * 1e-3) / 1e6, 1),
            "kernels": kernels, "hit_fraction": round(float((hits["id"] >= 0).float().mean().item()), 4),
            "device_errors": int((info[:, 7] != 0).sum())}


def leg_learned(args, dev, world, train_rays=16 << 20, eval_rays=8 << 20, batch=8192, lr=2e-3):
    """Learned subtree proposal on the 4,022,242-triangle terrain + soup scene, tree cut at depth 12 (4096
    slots): one epoch of Adam on 16M rays labelled by the plain traversal, then 8M fresh rays traced plain
    and with the proposal (MLP inference + seeded traversal); hits compared bit for bit."""
    import math

    import torch

    from cudart_b200 import core, proposal, scenes, tune

    mesh = scenes.learned_scene(1.0)
    box = scenes.scene_box(mesh, 1.5)
    V = torch.from_numpy(mesh.vertices).to(dev)
    Fc = torch.from_numpy(mesh.faces.view(np.int32)).to(dev)
    N = mesh.face_count
    del mesh
    tree = core.build_lbvh(V, Fc)
    slots = proposal.subtree_slots(tree, proposal.DEPTH)
    to, td = scenes.box_rays_torch(train_rays, box, seed=1, device=dev)
    eo, ed = scenes.box_rays_torch(eval_rays, box, seed=2, device=dev)
    sched, _ = tune.tune_trace(tree, eo, ed, key=f"learned{N}", use_cache=False)
    lab_hits = core.trace(tree, to, td, schedule=sched)
    labels = proposal.hit_labels(lab_hits["id"], slots["pos_label"])
    keep = labels >= 0
    to, td, tl = to[keep].contiguous(), td[keep].contiguous(), labels[keep].contiguous()
    del lab_hits, labels, keep
    n_train = (to.shape[0] // batch) * batch
    steps = n_train // batch
    net = proposal.ProposalNet(seed=0, device=dev)
    g = torch.Generator(device=dev).manual_seed(3)
    perm = torch.randperm(to.shape[0], device=dev, generator=g)[:n_train]
    to, td, tl = to[perm].contiguous(), td[perm].contiguous(), tl[perm].contiguous()
    del perm
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    for st in range(steps):
        sl = slice(st * batch, (st + 1) * batch)
        loss = net.train_step(to[sl], td[sl], tl[sl], box, lr=lr * 0.5 * (1.0 + math.cos(math.pi * st / steps)))
    ev1.record()
    torch.cuda.synchronize()
    train_ms = ev0.elapsed_time(ev1)
    flop_fwd = 2.0 * (144 * 128 + 2 * 128 * 128 + 128 * 4096)
    del to, td, tl
    R = eo.shape[0]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    plain = core.trace(tree, eo, ed, schedule=sched)
    prop = net.propose(eo, ed, box)
    seeded = proposal.trace_seeded(tree, eo, ed, prop, slots, in_proposal=True, schedule=sched)
    oracle_prop = proposal.hit_labels(plain["id"], slots["pos_label"])
    torch.cuda.synchronize()
    exact = (torch.equal(plain["id"], seeded["id"]) and torch.equal(plain["t"].view(torch.int32), seeded["t"].view(torch.int32))
             and torch.equal(plain["uv"].view(torch.int32), seeded["uv"].view(torch.int32)))
    hit = plain["id"] >= 0
    acc = float(seeded["in_proposal"][hit].float().mean().item())
    hs = proposal.trace_seeded(tree, eo, ed, prop, slots, schedule=sched)
    ms_plain = timed_ms(lambda: core.trace(tree, eo, ed, schedule=sched, out=plain), flush, reps=3, agg=min)
    ms_mlp = timed_ms(lambda: net.propose(eo, ed, box, out=prop), flush, reps=3, agg=min)
    ms_seeded = timed_ms(lambda: proposal.trace_seeded(tree, eo, ed, prop, slots, schedule=sched, out=hs), flush, reps=3, agg=min)
    ms_oracle = timed_ms(lambda: proposal.trace_seeded(tree, eo, ed, oracle_prop, slots, schedule=sched, out=hs), flush, reps=3, agg=min)
    ms_plain, ms_mlp, ms_seeded, ms_oracle = max_over_ranks([ms_plain, ms_mlp, ms_seeded, ms_oracle], world, dev)
    del flush
    return {"faces": N, "train_steps": steps, "batch": batch, "train_ms": round(train_ms, 1),
            "train_tflops": round(3 * flop_fwd * n_train / (train_ms * 1e-3) / 1e12, 1), "loss_last": round(float(loss.item()), 4),
            "eval_rays": R, "bit_exact": bool(exact), "proposal_accuracy": round(acc, 4), "plain_ms": round(ms_plain, 3),
            "plain_mrays_s": round(world * R / (ms_plain * 1e-3) / 1e6, 1), "mlp_ms": round(ms_mlp, 3),
            "mlp_tflops": round(flop_fwd * R / (ms_mlp * 1e-3) / 1e12, 1), "seeded_ms": round(ms_seeded, 3),
            "nn_over_plain": round(ms_plain / (ms_mlp + ms_seeded), 4), "oracle_seeded_over_plain": round(ms_plain / ms_oracle, 4)}


def leg_sah(args, dev, world):
    """SAH and Hybrid (LBVH depth 12, then SAH) builds of the 2^20-face soup, and the primary + bounce trace
    through each tree with its own tuned schedule, beside the LBVH tree's."""
    import torch

    from cudart_b200 import core, scenes, tune

    mesh, cam = scenes.soup_1m_scene(seed=SEED_MESH)
    v = torch.from_numpy(mesh.vertices).to(dev)
    f = torch.from_numpy(mesh.faces.view(np.int32)).to(dev)
    camera = core.make_camera(cam.center, cam.target, fov=cam.fov, ratio=cam.ratio)
    W, H = cam.width, cam.height
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    trees = {"lbvh": core.build_lbvh(v, f), "sah": core.build_sah(v, f), "hybrid12": core.build_sah(v, f, lbvh_depth=12)}
    o, d = core.primary_rays(camera, W, H)
    base = core.trace(trees["lbvh"], o, d)
    b = core.bounce_rays(trees["lbvh"].tris, o, d, base["id"], base["t"], SEED_BOUNCE)
    R = o.shape[0]
    out = {"faces": int(f.shape[0]),
           "sah_build_ms": round(timed_ms(lambda: core.build_sah(v, f, out=trees["sah"]), flush), 4),
           "hybrid12_build_ms": round(timed_ms(lambda: core.build_sah(v, f, lbvh_depth=12, out=trees["hybrid12"]), flush), 4),
           "lbvh_build_ms": round(timed_ms(lambda: core.build_lbvh(v, f, out=trees["lbvh"]), flush), 4)}
    for name, tr in trees.items():
        s1, _ = tune.tune_trace(tr, o, d, image_width=W, key=f"sah-{name}-p", use_cache=False)
        s2, _ = tune.tune_trace(tr, b[0], b[1], tmax=b[2], key=f"sah-{name}-b", use_cache=False)
        tp = timed_ms(lambda: core.trace(tr, o, d, schedule=s1), flush)
        tb = timed_ms(lambda: core.trace(tr, b[0], b[1], tmax=b[2], schedule=s2), flush)
        out[name] = {"nodes": tr.node_count, "primary_ms": round(tp, 4), "bounce_ms": round(tb, 4),
                     "mrays_s": round(world * 2 * R / ((tp + tb) * 1e-3) / 1e6, 1)}
    del flush
    return out


def leg_raster(args, dev, world):
    """The rasteriser on the 2^20-face soup (faces in the build's position order) at 1920 x 1080, beside the
    primary-ray trace of the same view; camera moved off the z axis (the reference's view matrix is NaN for
    a camera looking exactly along z)."""
    import torch

    from cudart_b200 import core, scenes

    mesh, cam = scenes.soup_1m_scene(seed=SEED_MESH)
    v = torch.from_numpy(mesh.vertices).to(dev)
    f = torch.from_numpy(mesh.faces.view(np.int32)).to(dev)
    tree = core.build_lbvh(v, f)
    W, H = cam.width, cam.height
    center = (cam.center[0] + 0.05, cam.center[1] + 0.1, cam.center[2])
    camera = core.make_camera(center, cam.target, fov=cam.fov, ratio=cam.ratio)
    m = core.raster_matrix(camera, cam.target)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    P = W * H
    out = dict(id=torch.zeros(P, dtype=torch.int32, device=dev), uv=torch.zeros((P, 2), dtype=torch.float32, device=dev),
               depth=torch.full((P,), 3.402823466e38, dtype=torch.float32, device=dev), err=torch.zeros(1, dtype=torch.int32, device=dev))

    def draw():
        out["depth"].fill_(3.402823466e38)  # CUDABuffer::clearOutputSurfaces
        core.rasterize(v, tree.faces, m, W, H, out=out)

    r = timed_ms(draw, flush)
    o, d = core.primary_rays(camera, W, H)
    t = timed_ms(lambda: core.trace(tree, o, d), flush)
    del flush
    return {"width": W, "height": H, "faces": int(f.shape[0]), "raster_ms": round(r, 4), "raster_mpix_s": round(world * P / (r * 1e-3) / 1e6, 1),
            "covered_fraction": round(float((out["depth"] < 3.4e38).float().mean().item()), 4), "trace_primary_ms_same_view": round(t, 4),
            "device_errors": int(out["err"].item())}


def run_legs(args, rank, world, local_rank):
    import torch

    from cudart_b200 import scenes

    dev = torch.device("cuda", local_rank)
    names = [] if args.legs in ("", "none") else args.legs.split(",")
    for name in names:
        if name == "c0":
            mesh, cam = scenes.terrain_small_scene()
            d = leg_single_scene(args, dev, world, mesh, cam, "terrain128")
            d["workload"] = "terrain 128^2 vertices (32,258 triangles), 512x512 primary rays + 1 bounce per hit"
        elif name == "c1":
            mesh, cam = scenes.soup_1m_scene(seed=SEED_MESH)
            d = leg_single_scene(args, dev, world, mesh, cam, "soup1m", with_roofline=True)
            d["workload"] = "soup 2^20 triangles, 1920x1080 primary rays + 1 diffuse bounce per hit"
        elif name == "build16m":
            d = leg_build_16m(args, dev, world)
        elif name == "c2":
            d = leg_batch(args, dev, world)
        elif name == "c3":
            d = leg_learned(args, dev, world)
        elif name == "sah":
            d = leg_sah(args, dev, world)
        elif name == "raster":
            d = leg_raster(args, dev, world)
        else:
            raise SystemExit(f"unknown leg {name}")
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        if rank == 0:
            emit({"leg": name, **d})


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            emit(res)
        return
    if args.cpu_legs:
        if rank == 0:
            cpu_legs()
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import torch
    torch.cuda.set_device(local_rank)
    run_legs(args, rank, world, local_rank)
    res, legs = run_headline(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        for k, d in legs.items():
            emit({"leg": k, **d})
        emit(res)


if __name__ == "__main__":
    main()
