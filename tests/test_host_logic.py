"""Host-side logic that needs no GPU: rebuilding hits from ids and packed (t, u, v), the batched-trace descriptor
(schedule bits, the kept pixel-tile order, bounce outputs) and the tuner's candidate lists."""
import ctypes as C

import pytest
import torch

from cudart_b200 import _abi, core, tune


def test_unpack_hits_rebuilds_misses_and_hits():
    ids = torch.tensor([-1, 3, -1, 0, 7, -1], dtype=torch.int32)
    packed = torch.tensor([1.5, 0.25, 0.5, 2.0, 0.0, 1.0, 3.25, 0.125, 0.75] + [9.0] * 9, dtype=torch.float32)
    t, uv = core.unpack_hits(ids, packed, 3)
    huge = torch.tensor(3.402823466e38, dtype=torch.float32)
    assert torch.equal(t, torch.stack([huge, torch.tensor(1.5), huge, torch.tensor(2.0), torch.tensor(3.25), huge]))
    assert torch.equal(uv, torch.tensor([[0, 0], [0.25, 0.5], [0, 0], [0.0, 1.0], [0.125, 0.75], [0, 0]], dtype=torch.float32))
    tmax = torch.tensor([-1.0, 5.0, 0.5, 5.0, 5.0, 2.0])
    t2, _ = core.unpack_hits(ids, packed, 3, tmax=tmax)
    assert torch.equal(t2, torch.tensor([-1.0, 1.5, 0.5, 2.0, 3.25, 2.0]))
    assert torch.equal(tmax, torch.tensor([-1.0, 5.0, 0.5, 5.0, 5.0, 2.0]))  # the caller's tmax is not written


def _fake_tree(M=2, N=64):
    z = lambda n: torch.zeros(n, dtype=torch.int32)
    return core.BatchTree(face_offsets=z(M + 1), vertex_offsets=z(M + 1), face_offsets_host=[0] * (M + 1), nodes=z((2 * N, 8)),
                          boxes=z((N, 8)), indices=z(N), codes=z(N), faces=z((N, 4)), tris=z((3 * N, 4)), accel=z(1024),
                          info=z((M, 8)), clusters=True)


def test_batch_trace_desc_schedule_bits_and_kept_tile_order():
    tree = _fake_tree()
    R = 2 * 8 * 4
    o = torch.zeros((R, 4), dtype=torch.float32)
    d = torch.zeros((R, 4), dtype=torch.float32)
    roff = torch.tensor([0, R // 2, R], dtype=torch.int32)
    sch = dict(clusters=True, persistent=True, blocks_per_sm=12, packet=True, lane_threshold=5)
    desc, out = core.batch_trace_desc(tree, o, d, roff, schedule=sch)
    assert desc.schedule == _abi.TRACE_CLUSTERS | _abi.TRACE_PACKET
    assert desc.persistent_blocks_per_sm == 12 and desc.lane_threshold == 5 and desc.work_counter
    assert not desc.bounce_orig and not desc.bounce_dir and not desc.bounce_tmax
    sch = dict(clusters=True, persistent=True, blocks_per_sm=8, refill=True, while_while=True)
    desc, _ = core.batch_trace_desc(tree, o, d, roff, schedule=sch)
    assert desc.schedule == _abi.TRACE_CLUSTERS | _abi.TRACE_REFILL | _abi.TRACE_WHILE_WHILE
    # a pixel-tile order kept with the outputs is used again for the same image shape (no new order is made)
    kept = torch.arange(R, dtype=torch.int32)
    out = dict(out, _order=kept, _tile_key=(2, 8, 4))
    sch = dict(clusters=True, persistent=True, blocks_per_sm=8, packet=True, tiles=[2, 8, 4])
    desc, out2 = core.batch_trace_desc(tree, o, d, roff, out=out, schedule=sch)
    assert desc.ray_order == kept.data_ptr() and out2["_order"] is kept


def test_tuner_candidates():
    plain = tune.cluster_batch_candidates()
    tiled = tune.cluster_batch_candidates(images=(64, 960, 540))
    odd = tune.cluster_batch_candidates(images=(64, 962, 540))  # width not a multiple of 8: no pixel tiles
    assert all(c["clusters"] for c in plain + tiled)
    assert not any("tiles" in c for c in plain + odd)
    refill_tiles = [c for c in tiled if c.get("refill") and "tiles" in c]
    assert sorted(c["lane_threshold"] for c in refill_tiles) == [4, 8, 16]
    packet_tiles = [c for c in tiled if c.get("packet") and "tiles" in c]
    assert packet_tiles and all(c["tiles"] == [64, 960, 540] for c in packet_tiles)
    keys = [tuple(sorted((k, str(v)) for k, v in c.items())) for c in tiled]
    assert len(keys) == len(set(keys)), "a candidate appears twice"


def test_bounce_fields_are_the_descriptor_tail():
    """The bounce outputs sit at the end of rt_batch_trace_desc, after lane_threshold (an older caller that zeroes
    the whole struct asks for none)."""
    names = [f[0] for f in _abi.BatchTraceDesc._fields_]
    assert names[-5:] == ["lane_threshold", "bounce_seed", "bounce_orig", "bounce_dir", "bounce_tmax"]
    assert _abi.BatchTraceDesc.bounce_seed.size == C.sizeof(C.c_uint64)
