"""Partitioning of the workload across ranks (one process per GPU).

The path has no exchange step: a scene's rays are independent given the tree,
and separate meshes are independent builds. So a rank either replicates the
tree and takes a contiguous range of a ray set, or takes a contiguous block of
meshes balanced by their cost (faces + rays). The only collective is an
optional gather of the per-ray outputs to one rank (an all-gather over NCCL /
NVLink on GPUs, gloo on CPU); nothing inside build or traversal communicates.
"""
from __future__ import annotations

import bisect

import torch


def ray_range(ray_count: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [begin, end) of a ray set for this rank; sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(ray_count, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def mesh_blocks(costs, world: int) -> list[tuple[int, int]]:
    """Split meshes 0..M-1 (in order) into `world` contiguous blocks of near-equal
    total cost: block r ends at the first mesh whose prefix cost reaches
    (r + 1) / world of the total."""
    if world <= 0:
        raise ValueError("bad world")
    prefix = [0]
    for c in costs:
        if c < 0:
            raise ValueError("negative cost")
        prefix.append(prefix[-1] + c)
    total = prefix[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        i = bisect.bisect_left(prefix, target)
        if i > 0 and target - prefix[i - 1] < prefix[i] - target:
            i -= 1  # the nearer of the two cut points
        bounds.append(min(max(i, bounds[-1]), len(costs)))
    bounds.append(len(costs))
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def gather_rays(local: torch.Tensor, ray_count: int, group=None) -> torch.Tensor:
    """All ranks' ray_range slices of a per-ray output, concatenated in ray order
    on every rank (all_gather of equal-size padded slices)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    chunk = -(-ray_count // world)
    pad = torch.zeros((chunk,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    out = []
    for r in range(world):
        b, e = ray_range(ray_count, r, world)
        out.append(parts[r][: e - b])
    return torch.cat(out)


def max_over_ranks(value: float, device="cpu", group=None) -> float:
    """The slowest rank's time (every multi-GPU number is timed this way)."""
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
