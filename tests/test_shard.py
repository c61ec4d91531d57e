"""Multi-rank host logic on CPU: ray ranges, cost-balanced mesh blocks, and the
output gather / max-over-ranks timing run as two gloo ranks (world size 2)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cudart_b200 import shard


def test_ray_ranges_cover_exactly():
    for R in (0, 1, 7, 1000, 2073601):
        for world in (1, 2, 3, 8):
            ranges = [shard.ray_range(R, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == R
            assert all(ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
            sizes = [e - b for b, e in ranges]
            assert max(sizes) - min(sizes) <= 1


def test_mesh_blocks_balanced():
    rng = np.random.default_rng(0)
    costs = np.exp(rng.uniform(np.log(64), np.log(65536), 1024)).astype(int).tolist()
    for world in (1, 2, 4, 8):
        blocks = shard.mesh_blocks(costs, world)
        assert blocks[0][0] == 0 and blocks[-1][1] == len(costs)
        assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
        loads = [sum(costs[b:e]) for b, e in blocks]
        assert max(loads) <= sum(costs) / world + max(costs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, R, result_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b, e = shard.ray_range(R, rank, world)
        ids = torch.arange(b, e, dtype=torch.int32) * 3  # stands in for this rank's hit ids
        t = torch.arange(b, e, dtype=torch.float32).unsqueeze(1).repeat(1, 2)
        all_ids = shard.gather_rays(ids, R)
        all_t = shard.gather_rays(t, R)
        slowest = shard.max_over_ranks(10.0 + rank)
        if rank == 0:
            torch.save({"ids": all_ids, "t": all_t, "slowest": slowest}, result_path)
    finally:
        dist.destroy_process_group()


def test_gather_and_max_over_two_gloo_ranks(tmp_path):
    R = 1001
    out = str(tmp_path / "res.pt")
    mp.spawn(_worker, args=(2, _free_port(), R, out), nprocs=2, join=True)
    res = torch.load(out)
    assert torch.equal(res["ids"], torch.arange(R, dtype=torch.int32) * 3)
    assert torch.equal(res["t"][:, 0], torch.arange(R, dtype=torch.float32))
    assert res["slowest"] == 11.0
