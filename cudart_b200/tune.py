"""Autotuner for the traversal schedule.

The blob traversal has knobs that change its speed and never its results
(including how many top levels of 4-wide records a persistent CTA stages in
shared memory):
the ray-to-thread mapping (linear, 8x4 pixel tiles of a row-major image, or
an order sorted by direction octant and origin Morton code, whose cost is
part of the timed trace),
warp-cooperative leaf tests (the warp's lanes share the triangle tests of all
its rays' leaves), static one-ray-per-thread launches or persistent warps that fetch rays from a
counter (and how many 128-thread CTAs per SM), and the if-if or while-while
leaf schedule. ``tune_trace`` times every combination on the caller's own
rays with CUDA events and returns the fastest; the choice is cached per GPU
name and workload key in a JSON file (``CUDART_B200_TUNE_CACHE``, default
``~/.cache/cudart_b200/tune.json``).
"""
from __future__ import annotations

import itertools
import json
import os

import torch

from . import core

CACHE = os.environ.get("CUDART_B200_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cudart_b200", "tune.json"))


def candidates(image_width: int):
    widths = [0, image_width] if image_width else [0]
    out = []
    for w, ww in itertools.product(widths, (False, True)):
        out.append({"image_width": w, "persistent": False, "blocks_per_sm": 0, "while_while": ww, "sorted": False})
        for bps in (8, 16):
            out.append({"image_width": w, "persistent": True, "blocks_per_sm": bps, "while_while": ww, "sorted": False})
    for ww, (p, bps) in itertools.product((False, True), ((False, 0), (True, 16))):
        out.append({"image_width": 0, "persistent": p, "blocks_per_sm": bps, "while_while": ww, "sorted": True})
    # warp-cooperative leaf tests (always while-while)
    for w, srt, (p, bps) in itertools.product(widths, (False, True), ((False, 0), (True, 8), (True, 16))):
        if srt and w:
            continue
        out.append({"image_width": w, "persistent": p, "blocks_per_sm": bps, "while_while": True, "sorted": srt, "coop": True})
    # every schedule again with the 4-wide records
    out += [dict(c, wide=True) for c in out]
    # persistent while-while 4-wide walks with the top 2 or 3 levels of records staged in shared memory per CTA
    out += [dict(c, treelet=depth) for c in out if c.get("wide") and c.get("persistent") and c.get("while_while")
            and c.get("blocks_per_sm") == 8 for depth in (2, 3)]
    return out


def cluster_candidates(image_width: int):
    """Single-mesh schedules that walk the cluster tree (a build with clusters=True)."""
    widths = [0, image_width] if image_width else [0]
    out = []
    for w, ww in itertools.product(widths, (False, True)):
        out.append({"clusters": True, "image_width": w, "persistent": False, "blocks_per_sm": 0, "while_while": ww})
        for bps in (8, 16):
            out.append({"clusters": True, "image_width": w, "persistent": True, "blocks_per_sm": bps, "while_while": ww})
    for w, bps in itertools.product(widths, (8, 16)):
        out.append({"clusters": True, "image_width": w, "persistent": True, "blocks_per_sm": bps, "coop": True})
    for coop, ww in ((False, False), (False, True), (True, False)):
        out.append({"clusters": True, "image_width": 0, "persistent": True, "blocks_per_sm": 16, "coop": coop, "while_while": ww,
                    "sorted": True})
    # per-lane walks in warps that refill their idle lanes
    for ml, srt, ww in itertools.product((4, 8, 16), (False, True), (False, True)):
        out.append({"clusters": True, "image_width": 0, "persistent": True, "blocks_per_sm": 8, "refill": True, "lane_threshold": ml,
                    "sorted": srt, "while_while": ww})
    # warp packets: pixel tiles of the image, or rays sorted by octant and origin (leaving the packet below
    # lane_threshold lanes)
    for bps, ml in itertools.product((8, 16), (0, 8, 16)):
        out.append({"clusters": True, "image_width": 0, "persistent": True, "blocks_per_sm": bps, "packet": True, "lane_threshold": ml,
                    "sorted": True})
        if image_width:
            out.append({"clusters": True, "image_width": image_width, "persistent": True, "blocks_per_sm": bps, "packet": True,
                        "lane_threshold": ml})
    return out


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(d):
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        with open(CACHE, "w") as f:
            json.dump(d, f, indent=1)
    except OSError:
        pass


def tune_trace(tree, orig, dir, tmax=None, image_width: int = 0, key: str = "default", reps: int = 3, use_cache: bool = True):
    """Returns (best_schedule, timings) where timings is a list of (schedule, ms)."""
    gpu = torch.cuda.get_device_name(orig.device)
    cache = _load() if use_cache else {}
    ck = f"{gpu}|{key}"
    if ck in cache:
        return cache[ck]["best"], cache[ck]["timings"]
    out = core.trace(tree, orig, dir, tmax=tmax)
    stream = torch.cuda.current_stream()
    timings = []
    cands = candidates(image_width) + (cluster_candidates(image_width) if getattr(tree, "clusters", False) else [])
    for sch in cands:
        core.trace(tree, orig, dir, tmax=tmax, out=out, schedule=sch)  # warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            core.trace(tree, orig, dir, tmax=tmax, out=out, schedule=sch)
        e1.record(stream)
        torch.cuda.synchronize()
        timings.append((sch, e0.elapsed_time(e1) / reps))
    best = min(timings, key=lambda x: x[1])[0]
    if use_cache:
        cache[ck] = {"best": best, "timings": timings}
        _store(cache)
    return best, timings


def cluster_batch_candidates(images=None):
    """Batched schedules that walk the cluster tree (a build with clusters=True): per-lane walks (one thread per
    ray, persistent warps), the warp-cooperative walk, each with the ray orders of batch_candidates."""
    out = [{"clusters": True, "persistent": False, "blocks_per_sm": 0, "while_while": ww} for ww in (False, True)]
    for coop, ww, bps in ((False, False, 8), (False, False, 16), (False, True, 8), (False, True, 16), (True, False, 8), (True, False, 16)):
        out.append({"clusters": True, "persistent": True, "blocks_per_sm": bps, "coop": coop, "while_while": ww})
        for bits in (0, 12):
            out.append({"clusters": True, "persistent": True, "blocks_per_sm": bps, "coop": coop, "while_while": ww, "sorted_bits": bits})
        if images is not None and images[1] % 8 == 0 and images[2] % 4 == 0:
            out.append({"clusters": True, "persistent": True, "blocks_per_sm": bps, "coop": coop, "while_while": ww, "tiles": list(images)})
    # per-lane walks in warps that refill their idle lanes once lane_threshold of them are idle
    for ml, bits, ww in itertools.product((2, 4, 8, 16), (None, 12), (False, True)):
        c = {"clusters": True, "persistent": True, "blocks_per_sm": 8, "refill": True, "lane_threshold": ml, "while_while": ww}
        out.append(c if bits is None else dict(c, sorted_bits=bits))
    if images is not None and images[1] % 8 == 0 and images[2] % 4 == 0:  # a warp's 32 slots an 8 x 4 pixel tile
        for ml in (4, 8, 16):
            out.append({"clusters": True, "persistent": True, "blocks_per_sm": 8, "refill": True, "lane_threshold": ml,
                        "while_while": False, "tiles": list(images)})
    # warp packets (one node sequence per warp): pixel tiles, and rays ordered by mesh, octant and origin; a warp
    # leaves the packet for per-lane walks once fewer than lane_threshold lanes want its node (0: never)
    for bps in (8, 16):
        for ml in (0, 8, 16, 24):
            out.append({"clusters": True, "persistent": True, "blocks_per_sm": bps, "packet": True, "lane_threshold": ml,
                        "sorted_bits": 21})
        if images is not None and images[1] % 8 == 0 and images[2] % 4 == 0:
            for ml in (0, 4, 8):
                out.append({"clusters": True, "persistent": True, "blocks_per_sm": bps, "packet": True, "lane_threshold": ml,
                            "tiles": list(images)})
    return out


def batch_candidates(images=None):
    """Schedules of the batched traversal (rt_batch_trace). images = (count, width, height) when every mesh's
    rays form one row-major image of that size (8 x 4 pixel tiles per warp become a candidate)."""
    out = []
    for ww, wide in itertools.product((False, True), (False, True)):
        out.append({"while_while": ww, "wide": wide, "persistent": False, "blocks_per_sm": 0})
        for bps in (8, 16):
            out.append({"while_while": ww, "wide": wide, "persistent": True, "blocks_per_sm": bps})
    # warp-cooperative leaf tests (persistent, while-while)
    for wide, bps in itertools.product((False, True), (8, 16)):
        out.append({"while_while": True, "wide": wide, "persistent": True, "blocks_per_sm": bps, "coop": True})
    # ray orders on the 4-wide records: rays sorted by mesh, octant and 0..21 Morton bits of the origin
    for bits, coop in itertools.product((0, 6, 12, 21), (False, True)):
        out.append({"while_while": True, "wide": True, "persistent": True, "blocks_per_sm": 16 if coop else 8, "coop": coop,
                    "sorted_bits": bits})
    if images is not None and images[1] % 8 == 0 and images[2] % 4 == 0:
        for coop, bps in ((False, 8), (False, 16), (True, 16)):
            out.append({"while_while": True, "wide": True, "persistent": True, "blocks_per_sm": bps, "coop": coop,
                        "tiles": list(images)})
    return out


def tune_batch_trace(tree, orig, dir, ray_offsets, tmax=None, key: str = "batch", reps: int = 2, use_cache: bool = True, images=None,
                     order=None):
    """tune_trace for core.batch_trace: (best_schedule, [(schedule, ms), ...]); `images` as for batch_candidates.
    `order`: a tracing order the caller already has (such as the bounce generator's active-first order); the
    schedules marked given_order use it."""
    gpu = torch.cuda.get_device_name(orig.device)
    cache = _load() if use_cache else {}
    ck = f"{gpu}|{key}"
    if ck in cache:
        return cache[ck]["best"], cache[ck]["timings"]
    out = core.batch_trace(tree, orig, dir, ray_offsets, tmax=tmax)
    stream = torch.cuda.current_stream()
    timings = []
    cands = batch_candidates(images)
    if order is not None:
        cands += [{"while_while": True, "wide": True, "persistent": True, "blocks_per_sm": bps, "coop": coop, "given_order": True}
                  for coop, bps in ((True, 16), (True, 8), (False, 8))]
    if getattr(tree, "clusters", False):
        cands += cluster_batch_candidates(images)
        if order is not None:
            cands += [{"clusters": True, "persistent": True, "blocks_per_sm": bps, "coop": coop, "while_while": ww, "given_order": True}
                      for coop, ww, bps in ((True, False, 16), (False, False, 8), (False, True, 8))]
            cands += [{"clusters": True, "persistent": True, "blocks_per_sm": 8, "refill": True, "lane_threshold": ml, "given_order": True}
                      for ml in (4, 8)]
    for sch in cands:
        given = order if sch.get("given_order") else None
        core.batch_trace(tree, orig, dir, ray_offsets, tmax=tmax, out=out, schedule=sch, order=given)  # warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            core.batch_trace(tree, orig, dir, ray_offsets, tmax=tmax, out=out, schedule=sch, order=given)
        e1.record(stream)
        torch.cuda.synchronize()
        timings.append((sch, e0.elapsed_time(e1) / reps))
    best = min(timings, key=lambda x: x[1])[0]
    if use_cache:
        cache[ck] = {"best": best, "timings": timings}
        _store(cache)
    return best, timings
