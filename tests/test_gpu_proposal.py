"""GPU checks of the learned subtree proposal (include/rt_propose.h).

* tcgen05 GEMM against torch (FP32 accumulation of BF16 products: relative
  error <= 1e-3 of the output scale), fused-argmax GEMM against torch's argmax;
* ray features against the oracle (|diff| <= 2^-7, one BF16 step near 1);
* one training step's gradients against the oracle (relative Frobenius error
  <= 2e-2 per tensor: BF16 intermediates may round differently when the FP32
  accumulation order differs);
* slot tables against a CPU walk of the node array;
* the seeded traversal: hits bit-identical to the plain traversal for random,
  invalid and trained proposals, all schedules;
* training gains: after a short training on plain-traversal labels the
  proposal lands in the hit's subtree far more often than an untrained one,
  and the seeded traversal reads fewer boxes than the plain one.
"""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bf16(x):
    return x.to(torch.bfloat16).contiguous()


@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (256, 256, 192), (384, 144, 128), (128, 192, 256), (256, 4096, 128)])
def test_gemm_matches_torch(m, n, k):
    from cudart_b200 import proposal as P
    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    a = _bf16(torch.randn(m, k, device="cuda", generator=g))
    b = _bf16(torch.randn(n, k, device="cuda", generator=g))
    bias = torch.randn(n, device="cuda", generator=g)
    ref = a.float() @ b.float().T
    c = torch.empty(m, n, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    P.gemm(a, b, out_f32=c, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    scale = ref.abs().max().item()
    assert (c - ref).abs().max().item() <= 1e-3 * scale
    # bias + ReLU, BF16 and transposed outputs, ReLU mask
    c16 = torch.empty(m, n, dtype=torch.bfloat16, device="cuda")
    ct = torch.empty(n, m, dtype=torch.bfloat16, device="cuda")
    mask = _bf16(torch.randn(m, n, device="cuda", generator=g))
    P.gemm(a, b, bias=bias, relu=True, mask=mask, alpha=0.5, out_bf16=c16, out_t=ct, err=err)
    torch.cuda.synchronize()
    want = torch.relu(0.5 * ref + bias) * (mask.float() > 0)
    assert (c16.float() - want).abs().max().item() <= 1e-2 * max(1.0, want.abs().max().item())
    assert torch.equal(ct, c16.T.contiguous())


def test_gemm_argmax_matches_torch():
    from cudart_b200 import proposal as P
    g = torch.Generator(device="cuda").manual_seed(7)
    m, n, k = 512, 4096, 128
    a = _bf16(torch.randn(m, k, device="cuda", generator=g))
    b = _bf16(torch.randn(n, k, device="cuda", generator=g))
    bias = torch.randn(n, device="cuda", generator=g)
    logits = a.float() @ b.float().T + bias
    top2 = logits.topk(2, dim=1).values
    clear = (top2[:, 0] - top2[:, 1]) > 1e-3 * top2[:, 0].abs().clamp(min=1)
    idx = torch.empty(m, dtype=torch.int32, device="cuda")
    val = torch.empty(m, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    P.gemm_argmax(a, b, bias=bias, out_index=idx, out_value=val, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert clear.float().mean().item() > 0.9
    assert torch.equal(idx[clear].long(), logits.argmax(1)[clear])
    assert (val - top2[:, 0]).abs().max().item() <= 1e-3 * top2[:, 0].abs().max().item()


def _rays(R, seed, box):
    rng = np.random.default_rng(seed)
    lo, hi = np.array(box[:3]), np.array(box[3:])
    o = np.zeros((R, 4), np.float32)
    d = np.zeros((R, 4), np.float32)
    o[:, :3] = rng.uniform(lo, hi, (R, 3))
    v = rng.normal(size=(R, 3))
    d[:, :3] = v / np.linalg.norm(v, axis=1, keepdims=True)
    return o, d


def test_features_match_oracle():
    from cudart_b200 import proposal as P
    from oracle import mlp_oracle as M
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    o, d = _rays(1000, 3, box)
    X = torch.empty(1000, 192, dtype=torch.bfloat16, device="cuda")
    XT = torch.empty(192, 1000, dtype=torch.bfloat16, device="cuda")
    P.ray_features(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda(), box, out=X, out_t=XT)
    torch.cuda.synchronize()
    want = M.features(o, d, box, rounding=False)
    got = X.float().cpu().numpy()
    assert np.abs(got - want).max() <= 2 ** -7
    assert torch.equal(XT, X.T.contiguous())
    assert (got[:, 144:] == 0).all()


def test_training_step_gradients_match_oracle():
    from cudart_b200 import proposal as P
    from oracle import mlp_oracle as M
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    B = 256
    o, d = _rays(B, 5, box)
    net = P.ProposalNet(classes=4096, seed=3)
    labels = np.random.default_rng(6).integers(0, 4096, B).astype(np.int32)
    loss = net.forward_backward(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda(), torch.from_numpy(labels).cuda(), box)
    torch.cuda.synchronize()
    assert int(net.err.item()) == 0
    ws = net._workspace(B, True)
    X = ws["X"].float().cpu().numpy().astype(np.float64)
    W = [w.float().cpu().numpy() for w in net.W16]
    b = [x.cpu().numpy() for x in net.b]
    ref_loss, dW, db = M.train_grads(X, W, b, labels)
    assert abs(loss.item() - ref_loss) <= 1e-3 * abs(ref_loss)
    for l in range(4):
        g = net.grads[2 * l].cpu().numpy()
        rel = np.linalg.norm(g - dW[l]) / max(np.linalg.norm(dW[l]), 1e-30)
        assert rel <= 2e-2, (l, rel)
        gb = net.grads[2 * l + 1].cpu().numpy()
        relb = np.linalg.norm(gb - db[l]) / max(np.linalg.norm(db[l]), 1e-30)
        assert relb <= 2e-2, (l, relb)
    # one Adam step moves every trained weight and keeps the BF16 copies in sync
    w0 = net.W[3].clone()
    net.adam(lr=1e-3)
    torch.cuda.synchronize()
    assert (net.W[3] - w0).abs().max().item() > 0
    assert torch.equal(net.W16[3], net.W[3].to(torch.bfloat16))
    assert torch.equal(net.W16t[3], net.W[3].t().contiguous().to(torch.bfloat16))
    assert (net.W[0][:, 144:] == 0).all()


def _terrain_tree():
    from cudart_b200 import core, scenes
    mesh = scenes.terrain(128, 0)
    v = torch.from_numpy(mesh.vertices).cuda()
    f = torch.from_numpy(mesh.faces.view(np.int32)).cuda()
    return mesh, core.build_lbvh(v, f)


def _cpu_slots(nodes, depth):
    """Node id and face range per slot from the bvnode words (CPU walk)."""
    S = 1 << depth
    node_of, lo, hi, first = np.zeros(S, np.int64), np.zeros(S, np.int64), np.zeros(S, np.int64), np.zeros(S, bool)
    for s in range(S):
        x, dd = 0, 0
        while dd < depth and not (nodes[x, 0] & 1):
            bit = (s >> (depth - 1 - dd)) & 1
            x = nodes[x, 1] + bit
            dd += 1
        node_of[s] = x
        first[s] = (s & ((1 << (depth - dd)) - 1)) == 0
        y = x
        while not (nodes[y, 0] & 1):
            y = nodes[y, 1]
        lo[s] = nodes[y, 1]
        y = x
        while not (nodes[y, 0] & 1):
            y = nodes[y, 1] + 1
        hi[s] = nodes[y, 1] + (nodes[y, 0] >> 1)
    return node_of, lo, hi, first


@pytest.mark.parametrize("depth", [4, 12])
def test_slot_tables_match_cpu_walk(depth):
    from cudart_b200 import proposal as P
    mesh, tree = _terrain_tree()
    sl = P.subtree_slots(tree, depth)
    torch.cuda.synchronize()
    nodes = tree.nodes_host().numpy().view(np.uint32).astype(np.int64)
    node_of, lo, hi, first = _cpu_slots(nodes, depth)
    sf = sl["slot_first"].cpu().numpy()
    sc = sl["slot_count"].cpu().numpy()
    assert np.array_equal(sf[first], lo[first]) and np.array_equal(sc[first], (hi - lo)[first])
    assert (sc[~first] == 0).all()
    # first slots tile [0, N) in order
    order = np.argsort(sf[first], kind="stable")
    starts, counts = sf[first][order], sc[first][order]
    assert starts[0] == 0 and np.array_equal(starts[1:], (starts + counts)[:-1]) and starts[-1] + counts[-1] == mesh.face_count
    lab = sl["pos_label"].cpu().numpy()
    want = np.repeat(np.nonzero(first)[0][order], counts)
    assert np.array_equal(lab, want)
    # references: internal node x -> record (child(x) - 1) / 2, leaf -> ~(leaf index)
    ref = sl["slot_ref"].cpu().numpy().view(np.uint32)
    internal = (nodes[node_of, 0] & 1) == 0
    assert np.array_equal(ref[internal], ((nodes[node_of[internal], 1] - 1) // 2).astype(np.uint32))
    assert (ref[~internal] >= 0x80000000).all()


def _seeded_equal(tree, o, d, prop, sl, schedule):
    from cudart_b200 import core
    from cudart_b200 import proposal as P
    plain = core.trace(tree, o, d, counters=True, schedule=schedule)
    seeded = P.trace_seeded(tree, o, d, prop, sl, counters=True, in_proposal=True, schedule=schedule)
    torch.cuda.synchronize()
    assert int(plain["err"].item()) == 0 and int(seeded["err"].item()) == 0
    assert torch.equal(plain["id"], seeded["id"])
    assert torch.equal(plain["t"].view(torch.int32), seeded["t"].view(torch.int32))
    assert torch.equal(plain["uv"].view(torch.int32), seeded["uv"].view(torch.int32))
    return plain, seeded


SCHEDULES = [dict(), dict(while_while=True), dict(coop=True), dict(coop=True, sorted=True), dict(persistent=True, while_while=True),
             dict(coop=True, persistent=True), dict(wide=True, while_while=True), dict(wide=True, coop=True, sorted=True)]


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_seeded_trace_is_bit_exact(schedule):
    from cudart_b200 import core
    from cudart_b200 import proposal as P
    mesh, tree = _terrain_tree()
    sl = P.subtree_slots(tree, 12)
    box = (-1.5, -0.6, -1.5, 1.5, 1.0, 1.5)
    o, d = _rays(40000, 11, box)
    o, d = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
    rng = np.random.default_rng(12)
    prop = rng.integers(-3, 4096 + 3, o.shape[0]).astype(np.int32)  # includes "none" and out-of-range proposals
    prop_t = torch.from_numpy(prop).cuda()
    _, seeded = _seeded_equal(tree, o, d, prop_t, sl, schedule)
    # the oracle proposal (the hit's own slot) is always "in proposal" for hits
    plain = core.trace(tree, o, d)
    labels = P.hit_labels(plain["id"], sl["pos_label"])
    _, seeded = _seeded_equal(tree, o, d, labels, sl, schedule)
    hit = (plain["id"] >= 0).cpu().numpy()
    inp = seeded["in_proposal"].cpu().numpy()
    assert (inp[hit] == 1).all() and (inp[~hit] == 0).all()


def test_training_gains_over_untrained():
    """What training buys, measured against the method without it (the plain
    traversal): the trained network's proposal contains the hit for far more
    rays than an untrained one, the hits stay bit-exact, and the traversal work
    stays within 10% of plain. The "oracle" proposal (every ray seeded with its
    true slot) bounds what any proposal can save on this traversal: it already
    visits nearer children first and culls by entry distance, so the closest hit
    is usually the first one found and a seed saves few tests."""
    from cudart_b200 import core, scenes
    from cudart_b200 import proposal as P
    mesh, tree = _terrain_tree()
    sl = P.subtree_slots(tree, 12)
    box = scenes.scene_box(mesh, 1.5)  # origins in the scene box grown 1.5x, as in the 4M-triangle workload
    o, d = _rays(1 << 20, 21, box)
    o, d = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
    plain = core.trace(tree, o, d)
    labels = P.hit_labels(plain["id"], sl["pos_label"])
    hit = labels >= 0
    to, td, tl = o[hit].contiguous(), d[hit].contiguous(), labels[hit].contiguous()
    net = P.ProposalNet(classes=4096, seed=1)
    eo, ed = _rays(1 << 16, 22, box)
    eo, ed = torch.from_numpy(eo).cuda(), torch.from_numpy(ed).cuda()
    sched = dict(coop=True)

    def score(prop):
        p_, s_ = _seeded_equal(tree, eo, ed, prop, sl, sched)
        h = p_["id"] >= 0
        acc = s_["in_proposal"][h].sum().item() / max(1, h.sum().item())
        return acc, s_["visits"].sum().item() / p_["visits"].sum().item(), s_["tests"].sum().item() / p_["tests"].sum().item()

    acc0, v0, t0 = score(net.propose(eo, ed, box))
    B, epochs = 4096, 6
    n = (to.shape[0] // B) * B
    total = epochs * (n // B)
    g = torch.Generator(device="cuda").manual_seed(5)
    losses = []
    for epoch in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        for s in range(0, n, B):
            idx = perm[s:s + B]
            lr = 1e-3 * (1.0 + math.cos(math.pi * len(losses) / total))  # cosine from 2e-3 to 0
            losses.append(net.train_step(to[idx].contiguous(), td[idx].contiguous(), tl[idx].contiguous(), box, lr=lr))
    torch.cuda.synchronize()
    assert int(net.err.item()) == 0
    first, last = losses[0].item(), np.mean([x.item() for x in losses[-5:]])
    acc1, v1, t1 = score(net.propose(eo, ed, box))
    plain_e = core.trace(tree, eo, ed)
    acc_o, v_o, t_o = score(P.hit_labels(plain_e["id"], sl["pos_label"]))
    print(f"\nloss {first:.3f} -> {last:.3f}; proposal contains the hit: untrained {acc0:.4f}, trained {acc1:.4f}, oracle {acc_o:.3f}; "
          f"box reads / triangle tests vs plain: untrained {v0:.3f} / {t0:.3f}, trained {v1:.3f} / {t1:.3f}, oracle {v_o:.3f} / {t_o:.3f}")
    assert last < first - 1.0, (first, last)
    assert acc1 > max(0.05, 10 * acc0), (acc0, acc1)
    assert acc_o == 1.0
    assert t_o <= 1.0 and v_o <= 1.02
    assert v1 <= 1.10 and t1 <= 1.10


@pytest.mark.parametrize("R,margin", [(1000, 0.0), (4096, 0.5), (128 * 150 + 17, 0.0)])
def test_fused_propose_matches_layered(R, margin):
    """rt_mlp_propose (one launch, activations on chip) returns the bits of the
    layer-by-layer path: features, three GEMMs, argmax GEMM."""
    from cudart_b200 import proposal as P
    box = (-1.5, -0.6, -1.5, 1.5, 1.4, 1.5)
    o, d = _rays(R, 17, box)
    o, d = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
    net = P.ProposalNet(seed=3)
    lab = torch.randint(0, 4096, (1024,), dtype=torch.int32, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
    to, td = _rays(1024, 18, box)
    for _ in range(3):  # move the weights off their initial values
        net.train_step(torch.from_numpy(to).cuda(), torch.from_numpy(td).cuda(), lab, box, lr=3e-3)
    m1, m2 = torch.empty(R, device="cuda"), torch.empty(R, device="cuda")
    if margin > 0:  # as a quantile of this network's margins, so that both outcomes occur
        net.propose(o, d, box, margin=m1)
        margin = float(m1.quantile(margin).item())
    a = net.propose(o, d, box, min_margin=margin, margin=m1, fused=True)
    b = net.propose(o, d, box, min_margin=margin, margin=m2, fused=False)
    torch.cuda.synchronize()
    assert int(net.err.item()) == 0
    assert torch.equal(a, b)
    assert torch.equal(m1.view(torch.int32), m2.view(torch.int32))
    if margin > 0:
        assert (a == -1).any() and (a >= 0).any()


@pytest.mark.parametrize("n,groups", [(1024, 1), (4096, 1), (512, 3)])
def test_gemm_xent_matches_torch(n, groups):
    """Fused logits + softmax cross-entropy gradient against torch in FP32 on
    the same logits (the kernel's FP32 GEMM output): |g - g_ref| <= 2^-8 |scale|
    (one BF16 rounding of values <= 1), the transpose exact, the loss within 1e-4."""
    from cudart_b200 import proposal as P
    gen = torch.Generator(device="cuda").manual_seed(11)
    m, k = 256, 128
    a = _bf16(torch.randn(groups * m, k, device="cuda", generator=gen))
    b = _bf16(torch.randn(groups * n, k, device="cuda", generator=gen) * 0.3)
    bias = torch.randn(groups * n, device="cuda", generator=gen)
    labels = torch.randint(-1, n + 2, (groups * m,), dtype=torch.int32, device="cuda", generator=gen)
    scale = 1.0 / m
    g = torch.empty(groups * m, n, dtype=torch.bfloat16, device="cuda")
    gt = torch.empty(groups * n, m, dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    P.gemm_xent(a, b, bias, labels, scale, g, gt, loss=loss, err=err, groups=groups)
    logits = torch.empty(groups * m, n, device="cuda")
    P.gemm(a, b, bias=bias, out_f32=logits, groups=groups)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    valid = (labels >= 0) & (labels < n)
    p = torch.softmax(logits.double(), dim=1)
    onehot = torch.zeros_like(p)
    onehot[valid, labels[valid].long()] = 1.0
    ref = ((p - onehot) * scale).float()
    ref[~valid] = 0.0
    assert (g.float() - ref).abs().max().item() <= scale * 2.0 ** -8
    for q in range(groups):
        assert torch.equal(gt[q * n:(q + 1) * n].view(torch.int16), g[q * m:(q + 1) * m].T.contiguous().view(torch.int16))
    lse = torch.logsumexp(logits.double(), dim=1)
    want = ((lse - logits.double().gather(1, labels.clamp(0, n - 1).long()[:, None])[:, 0])[valid] * scale).sum().item()
    assert abs(loss.item() - want) <= 1e-4 * max(1.0, abs(want))
