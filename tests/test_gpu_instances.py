"""Grouped proposal networks (one per mesh, include/rt_propose.h `groups`) and
the batched tree side (rt_batch_subtree_slots / rt_batch_hit_labels /
rt_batch_trace_seeded): every grouped result equals, bit for bit, the
ungrouped call on that group alone (whose numerics tests/test_gpu_proposal.py
checks against the oracle), and the seeded batched traversal returns the plain
batched traversal's hits exactly. Then the instanced-frames workload end to
end at a small size."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rand_bf16(shape, seed, scale=1.0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(shape, generator=g) * scale).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("n", [128, 512])
def test_grouped_gemm_matches_per_group(n):
    from cudart_b200 import proposal
    G, m, k = 3, 256, 192
    a, b = _rand_bf16((G * m, k), 1), _rand_bf16((G * n, k), 2, 0.1)
    bias = torch.randn(G * n, generator=torch.Generator().manual_seed(3)).cuda()
    mask = _rand_bf16((G * m, n), 4)
    outs = dict(f=torch.empty((G * m, n), device="cuda"), h=torch.empty((G * m, n), dtype=torch.bfloat16, device="cuda"),
                t=torch.empty((G * n, m), dtype=torch.bfloat16, device="cuda"))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    proposal.gemm(a, b, bias=bias, relu=True, mask=mask, out_f32=outs["f"], out_bf16=outs["h"], out_t=outs["t"], err=err, groups=G)
    for g in range(G):
        f = torch.empty((m, n), device="cuda")
        h = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
        t = torch.empty((n, m), dtype=torch.bfloat16, device="cuda")
        proposal.gemm(a[g * m:(g + 1) * m], b[g * n:(g + 1) * n], bias=bias[g * n:(g + 1) * n], relu=True, mask=mask[g * m:(g + 1) * m],
                      out_f32=f, out_bf16=h, out_t=t, err=err)
        torch.cuda.synchronize()
        assert torch.equal(outs["f"][g * m:(g + 1) * m].view(torch.int32), f.view(torch.int32))
        assert torch.equal(outs["h"][g * m:(g + 1) * m].view(torch.int16), h.view(torch.int16))
        assert torch.equal(outs["t"][g * n:(g + 1) * n].view(torch.int16), t.view(torch.int16))
    assert int(err.item()) == 0


def test_grouped_argmax_matches_per_group():
    from cudart_b200 import proposal
    G, m, n, k = 4, 256, 1024, 128
    a, b = _rand_bf16((G * m, k), 5), _rand_bf16((G * n, k), 6, 0.2)
    bias = torch.randn(G * n, generator=torch.Generator().manual_seed(7)).cuda() * 0.1
    idx = torch.empty(G * m, dtype=torch.int32, device="cuda")
    mar = torch.empty(G * m, dtype=torch.float32, device="cuda")
    proposal.gemm_argmax(a, b, bias=bias, out_index=idx, out_margin=mar, min_margin=0.05, groups=G)
    for g in range(G):
        i1 = torch.empty(m, dtype=torch.int32, device="cuda")
        m1 = torch.empty(m, dtype=torch.float32, device="cuda")
        proposal.gemm_argmax(a[g * m:(g + 1) * m], b[g * n:(g + 1) * n], bias=bias[g * n:(g + 1) * n], out_index=i1, out_margin=m1,
                             min_margin=0.05)
        torch.cuda.synchronize()
        assert torch.equal(idx[g * m:(g + 1) * m], i1)
        assert torch.equal(mar[g * m:(g + 1) * m].view(torch.int32), m1.view(torch.int32))
        logits = a[g * m:(g + 1) * m].float() @ b[g * n:(g + 1) * n].float().T + bias[g * n:(g + 1) * n]
        top2 = logits.topk(2, dim=1).values
        clear = (top2[:, 0] - top2[:, 1]) > 0.05 + 1e-3 * top2[:, 0].abs()
        assert clear.float().mean().item() > 0.5
        assert torch.equal(i1[clear].long(), logits.argmax(1)[clear])
    assert (idx >= 0).any() and (idx == -1).any()


def test_grouped_features_transpose_and_small_kernels():
    from cudart_b200 import proposal, scenes
    G, B = 3, 256
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    o, d = scenes.box_rays_torch(G * B, box, seed=11)
    X = torch.empty((G * B, 192), dtype=torch.bfloat16, device="cuda")
    XT = torch.empty((G * 192, B), dtype=torch.bfloat16, device="cuda")
    proposal.ray_features(o, d, box, out=X, out_t=XT, group_rows=B)
    torch.cuda.synchronize()
    for g in range(G):
        assert torch.equal(XT[g * 192:(g + 1) * 192].view(torch.int16), X[g * B:(g + 1) * B].t().contiguous().view(torch.int16))
    Y = _rand_bf16((G * 320, 96), 12)
    YT = torch.empty((G * 96, 320), dtype=torch.bfloat16, device="cuda")
    proposal.transpose_grouped(Y, G, YT)
    cs = torch.empty(G * 96, dtype=torch.float32, device="cuda")
    proposal.colsum_grouped(Y, G, cs)
    torch.cuda.synchronize()
    for g in range(G):
        blk = Y[g * 320:(g + 1) * 320]
        assert torch.equal(YT[g * 96:(g + 1) * 96].view(torch.int16), blk.t().contiguous().view(torch.int16))
        c1 = torch.empty(96, dtype=torch.float32, device="cuda")
        proposal.colsum(blk, c1)
        torch.cuda.synchronize()
        assert torch.equal(cs[g * 96:(g + 1) * 96].view(torch.int32), c1.view(torch.int32))
        assert torch.allclose(c1, blk.float().sum(0), rtol=1e-4, atol=1e-3)
    lab = torch.arange(G * 1000, dtype=torch.int32, device="cuda")
    oo, od = torch.empty((G * 300, 4), device="cuda"), torch.empty((G * 300, 4), device="cuda")
    ol = torch.empty(G * 300, dtype=torch.int32, device="cuda")
    oq, dq = torch.randn((G * 1000, 4), device="cuda"), torch.randn((G * 1000, 4), device="cuda")
    proposal.gather_batch(oq, dq, lab, G, 1000, 850, 300, (oo, od, ol))
    torch.cuda.synchronize()
    src = torch.tensor([g * 1000 + (850 + b) % 1000 for g in range(G) for b in range(300)], device="cuda")
    assert torch.equal(ol, lab[src]) and torch.equal(oo, oq[src]) and torch.equal(od, dq[src])


@pytest.mark.parametrize("G,R", [(3, 256), (5, 1280)])
def test_grouped_fused_propose_matches_layered(G, R):
    from cudart_b200 import proposal, scenes
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    grp = proposal.ProposalGroup(G, seed=2)
    to, td = scenes.box_rays_torch(G * 256, box, seed=40)
    lab = torch.randint(0, 4096, (G * 256,), dtype=torch.int32, device="cuda", generator=torch.Generator(device="cuda").manual_seed(6))
    for _ in range(2):
        grp.train_step(to, td, lab, box, 256, lr=3e-3)
    o, d = scenes.box_rays_torch(G * R, box, seed=41)
    a = grp.propose(o, d, box, R, fused=True)
    b = grp.propose(o, d, box, R, fused=False)
    torch.cuda.synchronize()
    assert int(grp.err.item()) == 0
    assert torch.equal(a, b)


def test_fused_propose_skips_inactive_rays():
    """With tmax, inactive rays (tmax <= 0) get -1 and whole inactive tiles are
    skipped; every active ray keeps the layered path's proposal."""
    from cudart_b200 import proposal, scenes
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    G, R = 3, 1024
    grp = proposal.ProposalGroup(G, seed=4)
    o, d = scenes.box_rays_torch(G * R, box, seed=43)
    g = torch.Generator(device="cuda").manual_seed(8)
    tmax = torch.where(torch.rand(G * R, device="cuda", generator=g) < 0.5, 1e30, -1.0).float()
    tmax[200:700] = -1.0             # tiles 2..4 of group 0 wholly inactive (rows 256..639)
    tmax[R + 128: R + 256] = 0.0     # one inactive tile of group 1
    tmax[2 * R:] = 1.0               # group 2 all active
    a = grp.propose(o, d, box, R, tmax=tmax, fused=True)
    b = grp.propose(o, d, box, R, fused=False)
    torch.cuda.synchronize()
    active = tmax > 0
    assert torch.equal(a[active], b[active])
    assert bool((a[~active] == -1).all())
    assert int(grp.err.item()) == 0


def test_group_select_and_index_gather():
    from cudart_b200 import proposal
    G, S = 3, 5000
    g = torch.Generator(device="cuda").manual_seed(4)
    lab = torch.randint(-3, 50, (G * S,), dtype=torch.int32, device="cuda", generator=g)
    lab[S:2 * S] = -1  # a group without any hit
    idx, cnt = proposal.group_select(lab, G, S)
    o, d = torch.randn((G * S, 4), device="cuda"), torch.randn((G * S, 4), device="cuda")
    B, off, hop = 700, 1400, 7919
    out = (torch.empty((G * B, 4), device="cuda"), torch.empty((G * B, 4), device="cuda"), torch.empty(G * B, dtype=torch.int32, device="cuda"))
    proposal.gather_batch(o, d, lab, G, S, off, B, out, index=idx, count=cnt, hop=hop)
    torch.cuda.synchronize()
    lab_h = lab.cpu().numpy()
    for q in range(G):
        want = np.nonzero(lab_h[q * S:(q + 1) * S] >= 0)[0]
        assert int(cnt[q]) == want.size
        assert np.array_equal(idx[q * S: q * S + want.size].cpu().numpy(), want)
        for b in (0, 1, B - 1):
            row = q * B + b
            if want.size == 0:
                assert int(out[2][row]) == -1
                continue
            src = q * S + int(want[((off + b) * hop) % want.size])
            assert torch.equal(out[0][row], o[src]) and torch.equal(out[1][row], d[src]) and int(out[2][row]) == int(lab_h[src])
    assert bool((out[2][:B] >= 0).all()) and bool((out[2][B:2 * B] == -1).all())


def test_grouped_training_matches_single_networks():
    """Two Adam steps of a 3-group network on different rays and labels per
    group leave group g's weights equal, bit for bit, to a ProposalNet trained
    alone on group g's rays."""
    from cudart_b200 import proposal, scenes
    G, B, K = 3, 256, 1024
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    base = proposal.ProposalNet(K, seed=5)
    grp = proposal.ProposalGroup(G, K, init=base)
    singles = [proposal.ProposalNet(K, seed=5) for _ in range(G)]
    gen = torch.Generator(device="cuda").manual_seed(9)
    for step in range(2):
        o, d = scenes.box_rays_torch(G * B, box, seed=20 + step)
        lab = torch.randint(-1, K, (G * B,), dtype=torch.int32, device="cuda", generator=gen)
        grp.train_step(o, d, lab, box, B, lr=3e-3)
        for g in range(G):
            sl = slice(g * B, (g + 1) * B)
            singles[g].train_step(o[sl].contiguous(), d[sl].contiguous(), lab[sl].contiguous(), box, lr=3e-3)
    torch.cuda.synchronize()
    for g in range(G):
        ng = grp.net(g)
        for i in range(4):
            assert torch.equal(ng.W[i].view(torch.int32), singles[g].W[i].view(torch.int32)), (g, i)
            assert torch.equal(ng.b[i].view(torch.int32), singles[g].b[i].view(torch.int32)), (g, i)
            assert torch.equal(ng.W16t[i].view(torch.int16), singles[g].W16t[i].view(torch.int16)), (g, i)
    assert not torch.equal(grp.net(0).W[3], grp.net(1).W[3])  # the groups did train apart
    assert int(grp.err.item()) == 0


def _batch(seed=3, count=5):
    from cudart_b200 import core, scenes
    meshes = scenes.batch_meshes(count, seed=seed, min_faces=64, max_faces=20000)
    v, f, fo, vo = scenes.concat_batch(meshes)
    V = torch.from_numpy(v).cuda()
    F = torch.from_numpy(f.view(np.int32)).cuda()
    return meshes, V, F, fo, vo, core.batch_build(V, F, fo, vo)


def test_batch_slots_match_single_builds():
    from cudart_b200 import core, proposal
    meshes, V, F, fo, vo, bt = _batch()
    bs = proposal.batch_subtree_slots(bt, 10)
    torch.cuda.synchronize()
    for m, mesh in enumerate(meshes):
        t = core.build_lbvh(torch.from_numpy(mesh.vertices).cuda(), torch.from_numpy(mesh.faces.view(np.int32)).cuda())
        s = proposal.subtree_slots(t, 10)
        torch.cuda.synchronize()
        assert torch.equal(bs["slot_ref"][m], s["slot_ref"]), m
        assert torch.equal(bs["slot_box"][m].view(torch.int32), s["slot_box"].view(torch.int32)), m
        assert torch.equal(bs["pos_label"][fo[m]:fo[m + 1]], s["pos_label"]), m


def test_batch_seeded_trace_is_bit_exact():
    from cudart_b200 import core, proposal, scenes
    meshes, V, F, fo, vo, bt = _batch(5, 6)
    rays = [scenes.sphere_rays(mesh, 48, seed=30 + i) for i, mesh in enumerate(meshes)]
    o = torch.from_numpy(np.concatenate([r[0] for r in rays])).cuda()
    d = torch.from_numpy(np.concatenate([r[1] for r in rays])).cuda()
    roff = torch.tensor(np.cumsum([0] + [r[0].shape[0] for r in rays]), dtype=torch.int32, device="cuda")
    slots = proposal.batch_subtree_slots(bt, 12)
    plain = core.batch_trace(bt, o, d, roff, counters=True)
    labels = proposal.batch_hit_labels(bt, plain["id"], roff, slots["pos_label"])
    g = torch.Generator(device="cuda").manual_seed(1)
    R = o.shape[0]
    rnd = torch.randint(-2, 4200, (R,), dtype=torch.int32, device="cuda", generator=g)  # includes none and out of range
    sch_wide = dict(while_while=True, wide=True, persistent=True, blocks_per_sm=4)
    sch_coop = dict(while_while=True, wide=True, persistent=True, blocks_per_sm=4, coop=True)
    for prop in (labels, rnd):
        for box_test, sch in ((True, None), (False, None), (True, sch_wide), (True, sch_coop)):
            s = proposal.batch_trace_seeded(bt, o, d, roff, prop, slots, counters=True, in_proposal=True, box_test=box_test,
                                            schedule=sch)
            torch.cuda.synchronize()
            assert int(s["err"].item()) == 0
            assert torch.equal(s["id"], plain["id"])
            assert torch.equal(s["t"].view(torch.int32), plain["t"].view(torch.int32))
            assert torch.equal(s["uv"].view(torch.int32), plain["uv"].view(torch.int32))
    best = proposal.batch_trace_seeded(bt, o, d, roff, labels, slots, counters=True, in_proposal=True)
    hit = plain["id"] >= 0
    assert bool(best["in_proposal"][hit].all())  # the true slot always holds the hit


def test_instanced_frames_small():
    """Four instances of the instanced learned scene (1/256 size), 3 frames:
    plain and learned traversal agree bit for bit every frame, and the
    networks' loss falls as they fine-tune."""
    from cudart_b200.instances import InstancedFrames
    w = InstancedFrames(4, 1 / 256, 64, 48, batch=256, steps=40, lr=3e-3)
    losses = []
    for f in range(3):
        w.displace(f)
        w.build()
        w.make_slots()
        if f > 0:
            losses.append(float(w.fine_tune().item()) / w.count)
        plain = w.trace_plain()
        learned = w.trace_learned(in_proposal=True)
        torch.cuda.synchronize()
        for k in ("h1", "h2"):
            assert torch.equal(plain[k]["id"], learned[k]["id"])
            assert torch.equal(plain[k]["t"].view(torch.int32), learned[k]["t"].view(torch.int32))
            assert torch.equal(plain[k]["uv"].view(torch.int32), learned[k]["uv"].view(torch.int32))
        assert (plain["h1"]["id"] >= 0).float().mean().item() > 0.2
        w.remember(plain)
    assert int(w.nets.err.item()) == 0
    assert losses[-1] < 7.0, losses  # from ln(4096) = 8.32: every training row is a hit
    info = w.tree.info.cpu()
    assert int(info[:, 7].abs().sum()) == 0  # rt_build_info.error of every instance
