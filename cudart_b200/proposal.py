"""Learned subtree proposal over the C ABI of include/rt_propose.h.

A small MLP maps each ray to one of 2^depth slots of the BVH (the tree cut at
a fixed depth; a slot names the node reached by following its bits from the
root). The seeded traversal tests the proposed subtree first and then the whole
tree without it, starting from the hit the first walk found, so its hits are
bit-identical to the plain traversal's; a good proposal only makes it cheaper.

Labels come from the plain traversal itself: a traced ray's label is the slot
holding its hit position (the first slot of that node when the hit leaf is
shallower than the cut depth); rays that miss are left out of training.

Network: 6 inputs -> sin/cos(pi 2^j u), j < 12 (144 features, zero-padded to
192) -> 3 x 128 ReLU -> 2^depth logits; BF16 weights [out][in] (tensor-core
operands), FP32 master weights, biases and Adam state. Every FLOP runs in
librt_core.so (tcgen05 GEMMs with TMA-fed shared memory and tensor-memory
accumulators); torch only holds the device buffers.
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from . import _abi
from .core import Tree, _p, _stream, trace_desc

FEATURES = 144
FEATURES_PAD = 192
HIDDEN = 128
DEPTH = 12


def _check(name, status):
    _abi.check(name, status)


def _bf16(shape, device):
    return torch.empty(shape, dtype=torch.bfloat16, device=device)


def gemm(a: torch.Tensor, b: torch.Tensor, bias=None, relu=False, mask=None, alpha=1.0, out_f32=None, out_bf16=None, out_t=None,
         err=None, groups: int = 1, stream=None):
    """C = alpha * a @ b.T (+ bias) (ReLU) (* (mask > 0)); a: bf16 (m, k), b: bf16 (n, k).
    groups > 1: a holds `groups` stacked (m, k) blocks and b stacked (n, k)
    blocks; block g of C is a_g @ b_g.T (out_t: stacked (n, m) transposes)."""
    m, k = a.shape[0] // groups, a.shape[1]
    n = b.shape[0] // groups
    if b.shape[1] != k:
        raise ValueError("inner dimensions differ")
    if a.shape[0] % groups or b.shape[0] % groups:
        raise ValueError("rows are not a multiple of groups")
    d = _abi.GemmDesc()
    d.groups = groups
    d.a, d.lda, d.b, d.ldb = a.data_ptr(), a.stride(0), b.data_ptr(), b.stride(0)
    d.m, d.n, d.k, d.alpha = m, n, k, alpha
    d.bias = bias.data_ptr() if bias is not None else None
    d.relu = int(relu)
    if mask is not None:
        d.mask, d.ldmask = mask.data_ptr(), mask.stride(0)
    if out_f32 is not None:
        d.c_f32, d.ldc_f32 = out_f32.data_ptr(), out_f32.stride(0)
    if out_bf16 is not None:
        d.c_bf16, d.ldc_bf16 = out_bf16.data_ptr(), out_bf16.stride(0)
    if out_t is not None:
        d.ct_bf16, d.ldct = out_t.data_ptr(), out_t.stride(0)
    if err is not None:
        d.error_word = err.data_ptr()
    _check("rt_gemm_bf16", _abi.lib().rt_gemm_bf16(C.byref(d), _stream(stream)))


def gemm_argmax(a: torch.Tensor, b: torch.Tensor, bias=None, out_index=None, out_value=None, out_margin=None, min_margin=0.0,
                err=None, groups: int = 1, stream=None):
    """Row argmax of a @ b.T + bias without storing the logits (-1 where the
    top-1 / top-2 margin is below min_margin); grouped as in gemm()."""
    m, k = a.shape[0] // groups, a.shape[1]
    n = b.shape[0] // groups
    if out_index is None:
        out_index = torch.empty(a.shape[0], dtype=torch.int32, device=a.device)
    d = _abi.GemmArgmaxDesc()
    d.groups = groups
    d.a, d.lda, d.b, d.ldb = a.data_ptr(), a.stride(0), b.data_ptr(), b.stride(0)
    d.m, d.n, d.k = m, n, k
    d.bias = bias.data_ptr() if bias is not None else None
    d.out_index = out_index.data_ptr()
    d.out_value = out_value.data_ptr() if out_value is not None else None
    d.out_margin = out_margin.data_ptr() if out_margin is not None else None
    d.min_margin = float(min_margin)
    if err is not None:
        d.error_word = err.data_ptr()
    _check("rt_gemm_argmax_bf16", _abi.lib().rt_gemm_argmax_bf16(C.byref(d), _stream(stream)))
    return out_index


def gemm_xent(a: torch.Tensor, b: torch.Tensor, bias, labels, scale: float, g: torch.Tensor, gt: torch.Tensor, loss=None, err=None,
              groups: int = 1, stream=None):
    """Softmax cross-entropy gradient of a @ b.T + bias (logits never stored):
    g = (softmax - onehot(labels)) * scale in BF16 and its (grouped) transpose gt;
    loss += scale * sum of the rows' cross-entropies."""
    m, k = a.shape[0] // groups, a.shape[1]
    n = b.shape[0] // groups
    d = _abi.GemmXentDesc()
    d.a, d.lda, d.b, d.ldb = a.data_ptr(), a.stride(0), b.data_ptr(), b.stride(0)
    d.m, d.n, d.k, d.bias, d.labels, d.scale = m, n, k, _p(bias), labels.data_ptr(), float(scale)
    d.g, d.ldg, d.gt, d.ldgt = g.data_ptr(), g.stride(0), gt.data_ptr(), gt.stride(0)
    d.loss_sum, d.error_word, d.groups = _p(loss), _p(err), groups
    _check("rt_gemm_xent_bf16", _abi.lib().rt_gemm_xent_bf16(C.byref(d), _stream(stream)))


def mlp_propose(orig, dir, box, W16, b, out=None, groups: int = 1, group_rows: int = 0, min_margin: float = 0.0, margin=None,
                value=None, err=None, count=None, tmax=None, stream=None):
    """Fused proposal (rt_mlp_propose): features, hidden layers and argmax in
    one launch. W16 / b: the four BF16 weight matrices and FP32 biases (grouped:
    stacked along rows). tmax: rays with tmax <= 0 get -1 (tiles of 128 such
    rays cost nothing)."""
    R = orig.shape[0] if count is None else count
    if out is None:
        out = torch.empty(R, dtype=torch.int32, device=orig.device)
    d = _abi.MlpProposeDesc()
    d.orig, d.dir, d.count = orig.data_ptr(), dir.data_ptr(), R
    for i in range(3):
        d.box_lo[i] = float(box[i])
        d.box_hi[i] = float(box[3 + i])
    d.w1, d.w2, d.w3, d.w4 = (w.data_ptr() for w in W16)
    d.b1, d.b2, d.b3, d.b4 = (x.data_ptr() for x in b)
    d.n = W16[3].shape[0] // groups
    d.groups, d.group_rows, d.min_margin = groups, group_rows, float(min_margin)
    d.out_index, d.out_value, d.out_margin, d.error_word = out.data_ptr(), _p(value), _p(margin), _p(err)
    d.tmax = _p(tmax)
    _check("rt_mlp_propose", _abi.lib().rt_mlp_propose(C.byref(d), _stream(stream)))
    return out


def ray_features(orig, dir, box, out=None, out_t=None, count=None, group_rows: int = 0, stream=None):
    """bf16 features (count, 192) and/or their transpose (192, count); box = (lo xyz, hi xyz).
    group_rows > 0: out_t holds one (192, group_rows) transpose per group of rays."""
    R = orig.shape[0] if count is None else count
    d = _abi.FeatureDesc()
    d.group_rows = group_rows
    d.orig, d.dir, d.count = orig.data_ptr(), dir.data_ptr(), R
    for i in range(3):
        d.box_lo[i] = float(box[i])
        d.box_hi[i] = float(box[3 + i])
    if out is not None:
        d.out, d.ld_out = out.data_ptr(), out.stride(0)
    if out_t is not None:
        d.out_t, d.ld_out_t = out_t.data_ptr(), out_t.stride(0)
    _check("rt_ray_features", _abi.lib().rt_ray_features(C.byref(d), _stream(stream)))
    return out, out_t


def transpose(x: torch.Tensor, out: torch.Tensor, stream=None):
    _check("rt_transpose_bf16", _abi.lib().rt_transpose_bf16(_p(x), x.shape[0], x.shape[1], x.stride(0), _p(out), out.stride(0), _stream(stream)))


def colsum(x: torch.Tensor, out: torch.Tensor, stream=None):
    _check("rt_colsum_bf16", _abi.lib().rt_colsum_bf16(_p(x), x.shape[0], x.shape[1], x.stride(0), _p(out), _stream(stream)))


def transpose_grouped(x: torch.Tensor, groups: int, out: torch.Tensor, stream=None):
    """x: `groups` stacked (r, c) blocks -> out: stacked (c, r) transposes."""
    r = x.shape[0] // groups
    _check("rt_transpose_bf16_grouped", _abi.lib().rt_transpose_bf16_grouped(_p(x), groups, r, x.shape[1], x.stride(0), _p(out),
                                                                              out.stride(0), _stream(stream)))


def colsum_grouped(x: torch.Tensor, groups: int, out: torch.Tensor, stream=None):
    """Column sums of each of `groups` stacked blocks: out (groups * cols,)."""
    r = x.shape[0] // groups
    _check("rt_colsum_bf16_grouped", _abi.lib().rt_colsum_bf16_grouped(_p(x), groups, r, x.shape[1], x.stride(0), _p(out),
                                                                        _stream(stream)))


def gather_batch(orig, dir, labels, groups: int, group_stride: int, offset: int, batch: int, out: tuple, index=None, count=None,
                 hop: int = 1, stream=None):
    """Rows g * batch + b <- g * group_stride + q: q = k, or index[g][k] with an
    index list (group_select), for k = ((offset + b) * hop) mod n_g."""
    d = _abi.BatchGatherDesc()
    d.orig, d.dir, d.labels = orig.data_ptr(), dir.data_ptr(), _p(labels)
    d.groups, d.group_stride, d.offset, d.batch = groups, group_stride, offset % (1 << 32), batch
    d.out_orig, d.out_dir, d.out_labels = out[0].data_ptr(), out[1].data_ptr(), _p(out[2])
    d.index, d.index_count, d.hop = _p(index), _p(count), hop
    _check("rt_gather_batch", _abi.lib().rt_gather_batch(C.byref(d), _stream(stream)))
    return out


def group_select(labels, groups: int, group_stride: int, index=None, count=None, stream=None):
    """Per group, the rows (ascending) whose label is >= 0, and how many."""
    dev = labels.device
    if index is None:
        index = torch.empty(groups * group_stride, dtype=torch.int32, device=dev)
    if count is None:
        count = torch.empty(groups, dtype=torch.int32, device=dev)
    _check("rt_group_select", _abi.lib().rt_group_select(_p(labels), groups, group_stride, _p(index), _p(count), _stream(stream)))
    return index, count


class ProposalNet:
    """Weights, Adam state and workspaces of the proposal MLP on one device."""

    def __init__(self, classes: int = 1 << DEPTH, device="cuda", seed: int = 0):
        self.classes = classes
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        shapes = [(HIDDEN, FEATURES_PAD, FEATURES), (HIDDEN, HIDDEN, HIDDEN), (HIDDEN, HIDDEN, HIDDEN), (classes, HIDDEN, HIDDEN)]
        self.W, self.b, self.W16, self.W16t = [], [], [], []
        for out_f, in_f, fan_in in shapes:
            bound = 1.0 / math.sqrt(fan_in)
            w = (torch.rand((out_f, in_f), generator=g) * 2 - 1) * bound
            w[:, fan_in:] = 0.0  # padded feature columns stay zero (their gradient is zero)
            bb = (torch.rand(out_f, generator=g) * 2 - 1) * bound
            self.W.append(w.to(self.device))
            self.b.append(bb.to(self.device))
        for w in self.W:
            self.W16.append(w.to(torch.bfloat16).contiguous())
            self.W16t.append(w.t().contiguous().to(torch.bfloat16))
        self.params = [t for pair in zip(self.W, self.b) for t in pair]
        self.m = [torch.zeros_like(t) for t in self.params]
        self.v = [torch.zeros_like(t) for t in self.params]
        self.grads = [torch.zeros_like(t) for t in self.params]
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._ws = {}

    def param_count(self) -> int:
        return sum(w.shape[0] * (FEATURES if i == 0 else w.shape[1]) + w.shape[0] for i, w in enumerate(self.W))

    def _workspace(self, B: int, train: bool):
        key = (B, train)
        ws = self._ws.get(key)
        if ws is None:
            dev = self.device
            ws = dict(X=_bf16((B, FEATURES_PAD), dev), H1=_bf16((B, HIDDEN), dev), H2=_bf16((B, HIDDEN), dev), H3=_bf16((B, HIDDEN), dev))
            if train:
                ws.update(XT=_bf16((FEATURES_PAD, B), dev), H1T=_bf16((HIDDEN, B), dev), H2T=_bf16((HIDDEN, B), dev),
                          H3T=_bf16((HIDDEN, B), dev), G=_bf16((B, self.classes), dev), GT=_bf16((self.classes, B), dev), D3=_bf16((B, HIDDEN), dev),
                          D3T=_bf16((HIDDEN, B), dev), D2=_bf16((B, HIDDEN), dev), D2T=_bf16((HIDDEN, B), dev),
                          D1=_bf16((B, HIDDEN), dev), D1T=_bf16((HIDDEN, B), dev),
                          loss=torch.zeros(1, dtype=torch.float32, device=dev))
            self._ws[key] = ws
        return ws

    # ------------------------------------------------------------- training
    def forward_backward(self, orig, dir, labels, box, stream=None):
        """Gradients of the mean cross-entropy over one batch (B % 128 == 0,
        every label in [0, classes)) into self.grads; returns the loss tensor."""
        B = orig.shape[0]
        if B % 128:
            raise ValueError("batch size must be a multiple of 128")
        ws = self._workspace(B, True)
        W16, W16t, b = self.W16, self.W16t, self.b
        err = self.err
        ray_features(orig, dir, box, out=ws["X"], out_t=ws["XT"], stream=stream)
        gemm(ws["X"], W16[0], bias=b[0], relu=True, out_bf16=ws["H1"], out_t=ws["H1T"], err=err, stream=stream)
        gemm(ws["H1"], W16[1], bias=b[1], relu=True, out_bf16=ws["H2"], out_t=ws["H2T"], err=err, stream=stream)
        gemm(ws["H2"], W16[2], bias=b[2], relu=True, out_bf16=ws["H3"], out_t=ws["H3T"], err=err, stream=stream)
        ws["loss"].zero_()
        gemm_xent(ws["H3"], W16[3], b[3], labels, 1.0 / B, ws["G"], ws["GT"], loss=ws["loss"], err=err, stream=stream)
        gW = self.grads[0::2]
        gb = self.grads[1::2]
        # layer 4
        gemm(ws["GT"], ws["H3T"], out_f32=gW[3], err=err, stream=stream)
        colsum(ws["G"], gb[3], stream=stream)
        gemm(ws["G"], W16t[3], mask=ws["H3"], out_bf16=ws["D3"], out_t=ws["D3T"], err=err, stream=stream)
        # layer 3
        gemm(ws["D3T"], ws["H2T"], out_f32=gW[2], err=err, stream=stream)
        colsum(ws["D3"], gb[2], stream=stream)
        gemm(ws["D3"], W16t[2], mask=ws["H2"], out_bf16=ws["D2"], out_t=ws["D2T"], err=err, stream=stream)
        # layer 2
        gemm(ws["D2T"], ws["H1T"], out_f32=gW[1], err=err, stream=stream)
        colsum(ws["D2"], gb[1], stream=stream)
        gemm(ws["D2"], W16t[1], mask=ws["H1"], out_bf16=ws["D1"], out_t=ws["D1T"], err=err, stream=stream)
        # layer 1
        gemm(ws["D1T"], ws["XT"], out_f32=gW[0], err=err, stream=stream)
        colsum(ws["D1"], gb[0], stream=stream)
        return ws["loss"].clone()  # the workspace is reused by the next step

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        for i, (p, g, m, v) in enumerate(zip(self.params, self.grads, self.m, self.v)):
            d = _abi.AdamDesc()
            d.param, d.grad, d.m, d.v = p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr()
            if p.dim() == 2:
                d.rows, d.cols = p.shape
                w16, w16t = self.W16[i // 2], self.W16t[i // 2]
                d.out_bf16, d.ld_bf16 = w16.data_ptr(), w16.stride(0)
                d.out_bf16_t, d.ld_bf16_t = w16t.data_ptr(), w16t.stride(0)
            else:
                d.rows, d.cols = 1, p.shape[0]
            d.lr, d.beta1, d.beta2, d.eps, d.step = lr, beta1, beta2, eps, self.step_count
            _check("rt_adam_step", _abi.lib().rt_adam_step(C.byref(d), _stream(stream)))

    def train_step(self, orig, dir, labels, box, lr=1e-3, stream=None):
        loss = self.forward_backward(orig, dir, labels, box, stream=stream)
        self.adam(lr=lr, stream=stream)
        return loss

    # ------------------------------------------------------------- inference
    def propose(self, orig, dir, box, out=None, min_margin: float = 0.0, margin=None, chunk: int = 1 << 20, fused: bool = True,
                stream=None):
        """int32 slot proposal per ray: the argmax of the logits, or -1 (no
        proposal) where its margin over the runner-up is below min_margin.
        fused: one rt_mlp_propose launch; otherwise features, three GEMMs and
        the argmax GEMM as separate launches (the same bits)."""
        R = orig.shape[0]
        if out is None:
            out = torch.empty(R, dtype=torch.int32, device=orig.device)
        if fused:
            return mlp_propose(orig, dir, box, self.W16, self.b, out=out, min_margin=min_margin, margin=margin, err=self.err,
                               stream=stream)
        c = min(chunk, ((R + 127) // 128) * 128)
        ws = self._workspace(c, False)
        for s in range(0, R, c):
            e = min(R, s + c)
            n = e - s
            n_pad = ((n + 127) // 128) * 128
            o, d = orig[s:e], dir[s:e]
            X, H1, H2, H3 = ws["X"][:n_pad], ws["H1"][:n_pad], ws["H2"][:n_pad], ws["H3"][:n_pad]
            if n_pad != n:
                X[n:].zero_()
            ray_features(o, d, box, out=X, count=n, stream=stream)
            gemm(X, self.W16[0], bias=self.b[0], relu=True, out_bf16=H1, err=self.err, stream=stream)
            gemm(H1, self.W16[1], bias=self.b[1], relu=True, out_bf16=H2, err=self.err, stream=stream)
            gemm(H2, self.W16[2], bias=self.b[2], relu=True, out_bf16=H3, err=self.err, stream=stream)
            if n_pad == n:
                gemm_argmax(H3, self.W16[3], bias=self.b[3], out_index=out[s:e], out_margin=None if margin is None else margin[s:e],
                            min_margin=min_margin, err=self.err, stream=stream)
            else:
                tmp = torch.empty(n_pad, dtype=torch.int32, device=orig.device)
                tm = torch.empty(n_pad, dtype=torch.float32, device=orig.device)
                gemm_argmax(H3, self.W16[3], bias=self.b[3], out_index=tmp, out_margin=tm, min_margin=min_margin, err=self.err,
                            stream=stream)
                out[s:e].copy_(tmp[:n])
                if margin is not None:
                    margin[s:e].copy_(tm[:n])
        return out


class ProposalGroup:
    """`groups` independent proposal networks (one per mesh of a batched
    build) trained and run in the same launches: every weight, bias and
    activation stacks the groups along its rows, and group g's numbers equal,
    bit for bit, a ProposalNet holding group g's weights fed group g's rays."""

    def __init__(self, groups: int, classes: int = 1 << DEPTH, device="cuda", seed: int = 0, init: "ProposalNet | None" = None):
        self.groups, self.classes = groups, classes
        self.device = torch.device(device)
        base = init if init is not None else ProposalNet(classes, device=self.device, seed=seed)
        G = groups
        self.W = [w.repeat(G, 1).contiguous() for w in base.W]
        self.b = [b.repeat(G).contiguous() for b in base.b]
        self.W16 = [w.to(torch.bfloat16).contiguous() for w in self.W]
        self.W16t = [self._stacked_t(w) for w in self.W]
        self.params = [t for pair in zip(self.W, self.b) for t in pair]
        self.m = [torch.zeros_like(t) for t in self.params]
        self.v = [torch.zeros_like(t) for t in self.params]
        self.grads = [torch.zeros_like(t) for t in self.params]
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._ws = {}

    def _stacked_t(self, w):
        G = self.groups
        out_f, in_f = w.shape[0] // G, w.shape[1]
        return w.view(G, out_f, in_f).transpose(1, 2).reshape(G * in_f, out_f).to(torch.bfloat16).contiguous()

    def net(self, g: int) -> ProposalNet:
        """Group g's weights as a stand-alone ProposalNet (FP32 master copies)."""
        n = ProposalNet(self.classes, device=self.device)
        for i in range(4):
            rows = n.W[i].shape[0]
            n.W[i].copy_(self.W[i][g * rows:(g + 1) * rows])
            n.b[i].copy_(self.b[i][g * rows:(g + 1) * rows])
            n.W16[i].copy_(self.W16[i][g * rows:(g + 1) * rows])
            cols = n.W[i].shape[1]
            n.W16t[i].copy_(self.W16t[i][g * cols:(g + 1) * cols])
        return n

    def _workspace(self, B: int, train: bool):
        """Training: B rays per group (G B rows); inference: B rows in all."""
        key = (B, train)
        ws = self._ws.get(key)
        if ws is None:
            G, dev, K = self.groups, self.device, self.classes
            R = G * B if train else B
            ws = dict(X=_bf16((R, FEATURES_PAD), dev), H1=_bf16((R, HIDDEN), dev), H2=_bf16((R, HIDDEN), dev), H3=_bf16((R, HIDDEN), dev))
            if train:
                ws.update(XT=_bf16((G * FEATURES_PAD, B), dev), H1T=_bf16((G * HIDDEN, B), dev), H2T=_bf16((G * HIDDEN, B), dev),
                          H3T=_bf16((G * HIDDEN, B), dev), G=_bf16((R, K), dev), GT=_bf16((G * K, B), dev), D3=_bf16((R, HIDDEN), dev),
                          D3T=_bf16((G * HIDDEN, B), dev), D2=_bf16((R, HIDDEN), dev), D2T=_bf16((G * HIDDEN, B), dev),
                          D1=_bf16((R, HIDDEN), dev), D1T=_bf16((G * HIDDEN, B), dev),
                          loss=torch.zeros(1, dtype=torch.float32, device=dev),
                          bo=torch.empty((R, 4), dtype=torch.float32, device=dev), bd=torch.empty((R, 4), dtype=torch.float32, device=dev),
                          bl=torch.empty(R, dtype=torch.int32, device=dev))
            self._ws[key] = ws
        return ws

    def forward_backward(self, orig, dir, labels, box, batch: int, stream=None):
        """Gradients of each group's mean cross-entropy over its `batch` rays
        (rows g * batch ..; labels outside [0, classes) are left out); returns
        the sum over groups of the group losses (a workspace tensor: the next
        step overwrites it)."""
        G, B = self.groups, batch
        if B % 128 or orig.shape[0] != G * B:
            raise ValueError("need groups * batch rays with batch % 128 == 0")
        ws = self._workspace(B, True)
        W16, W16t, b, err = self.W16, self.W16t, self.b, self.err
        kw = dict(err=err, groups=G, stream=stream)
        ray_features(orig, dir, box, out=ws["X"], out_t=ws["XT"], group_rows=B, stream=stream)
        gemm(ws["X"], W16[0], bias=b[0], relu=True, out_bf16=ws["H1"], out_t=ws["H1T"], **kw)
        gemm(ws["H1"], W16[1], bias=b[1], relu=True, out_bf16=ws["H2"], out_t=ws["H2T"], **kw)
        gemm(ws["H2"], W16[2], bias=b[2], relu=True, out_bf16=ws["H3"], out_t=ws["H3T"], **kw)
        ws["loss"].zero_()
        gemm_xent(ws["H3"], W16[3], b[3], labels, 1.0 / B, ws["G"], ws["GT"], loss=ws["loss"], **kw)
        gW, gb = self.grads[0::2], self.grads[1::2]
        gemm(ws["GT"], ws["H3T"], out_f32=gW[3], **kw)
        colsum_grouped(ws["G"], G, gb[3], stream=stream)
        gemm(ws["G"], W16t[3], mask=ws["H3"], out_bf16=ws["D3"], out_t=ws["D3T"], **kw)
        gemm(ws["D3T"], ws["H2T"], out_f32=gW[2], **kw)
        colsum_grouped(ws["D3"], G, gb[2], stream=stream)
        gemm(ws["D3"], W16t[2], mask=ws["H2"], out_bf16=ws["D2"], out_t=ws["D2T"], **kw)
        gemm(ws["D2T"], ws["H1T"], out_f32=gW[1], **kw)
        colsum_grouped(ws["D2"], G, gb[1], stream=stream)
        gemm(ws["D2"], W16t[1], mask=ws["H1"], out_bf16=ws["D1"], out_t=ws["D1T"], **kw)
        gemm(ws["D1T"], ws["XT"], out_f32=gW[0], **kw)
        colsum_grouped(ws["D1"], G, gb[0], stream=stream)
        return ws["loss"]

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        for i, (p, g, m, v) in enumerate(zip(self.params, self.grads, self.m, self.v)):
            d = _abi.AdamDesc()
            d.param, d.grad, d.m, d.v = p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr()
            if p.dim() == 2:
                d.rows, d.cols = p.shape
                d.groups = self.groups
                w16, w16t = self.W16[i // 2], self.W16t[i // 2]
                d.out_bf16, d.ld_bf16 = w16.data_ptr(), w16.stride(0)
                d.out_bf16_t, d.ld_bf16_t = w16t.data_ptr(), w16t.stride(0)
            else:
                d.rows, d.cols = 1, p.shape[0]
            d.lr, d.beta1, d.beta2, d.eps, d.step = lr, beta1, beta2, eps, self.step_count
            _check("rt_adam_step", _abi.lib().rt_adam_step(C.byref(d), _stream(stream)))

    def train_step(self, orig, dir, labels, box, batch: int, lr=1e-3, stream=None):
        loss = self.forward_backward(orig, dir, labels, box, batch, stream=stream)
        self.adam(lr=lr, stream=stream)
        return loss

    def fine_tune(self, orig, dir, labels, box, group_rays: int, steps: int, batch: int, lr=1e-3, offset: int = 0, stream=None):
        """`steps` Adam steps; step j trains group g on its rays
        g * group_rays + (offset + j * batch + b) % group_rays, b < batch."""
        ws = self._workspace(batch, True)
        out = (ws["bo"], ws["bd"], ws["bl"])
        loss = None
        for j in range(steps):
            gather_batch(orig, dir, labels, self.groups, group_rays, offset + j * batch, batch, out, stream=stream)
            loss = self.train_step(out[0], out[1], out[2], box, batch, lr=lr, stream=stream)
        return loss

    def propose(self, orig, dir, box, group_rays: int, out=None, min_margin: float = 0.0, chunk_rows: int = 1 << 22, fused: bool = True,
                margin=None, tmax=None, stream=None):
        """Slot proposal per ray; group g's rays are rows g * group_rays ..
        (group_rays % 128 == 0), scored by group g's network; rays with
        tmax <= 0 (when given) get -1."""
        G = self.groups
        if group_rays % 128 or orig.shape[0] != G * group_rays:
            raise ValueError("need groups * group_rays rays with group_rays % 128 == 0")
        if out is None:
            out = torch.empty(G * group_rays, dtype=torch.int32, device=orig.device)
        if fused:
            return mlp_propose(orig, dir, box, self.W16, self.b, out=out, groups=G, group_rows=group_rays, min_margin=min_margin,
                               margin=margin, err=self.err, tmax=tmax, stream=stream)
        cg = max(1, min(G, chunk_rows // group_rays))
        ws = self._workspace(cg * group_rays, False)
        for g0 in range(0, G, cg):
            g1 = min(G, g0 + cg)
            ng, r0, r1 = g1 - g0, g0 * group_rays, g1 * group_rays
            X, H1, H2, H3 = (ws[k][:r1 - r0] for k in ("X", "H1", "H2", "H3"))
            ray_features(orig[r0:r1], dir[r0:r1], box, out=X, stream=stream)
            wv = [w[g0 * (w.shape[0] // G): g1 * (w.shape[0] // G)] for w in self.W16]
            bv = [b[g0 * (b.shape[0] // G): g1 * (b.shape[0] // G)] for b in self.b]
            kw = dict(err=self.err, groups=ng, stream=stream)
            gemm(X, wv[0], bias=bv[0], relu=True, out_bf16=H1, **kw)
            gemm(H1, wv[1], bias=bv[1], relu=True, out_bf16=H2, **kw)
            gemm(H2, wv[2], bias=bv[2], relu=True, out_bf16=H3, **kw)
            gemm_argmax(H3, wv[3], bias=bv[3], out_index=out[r0:r1], min_margin=min_margin, **kw)
        if tmax is not None:
            out.masked_fill_(~(tmax > 0), -1)
        return out


# ----------------------------------------------------------------- tree side
def subtree_slots(tree: Tree, depth: int = DEPTH, stream=None) -> dict:
    """Slot table of a built tree: slot_ref (2^depth blob references), pos_label
    (per face position), slot_first / slot_count (face range of each first slot)."""
    if tree.accel is None:
        raise ValueError("the tree has no traversal blob")
    N = tree.faces.shape[0]
    dev = tree.faces.device
    S = 1 << depth
    out = dict(slot_ref=torch.empty(S, dtype=torch.int32, device=dev), slot_box=torch.empty((S, 8), dtype=torch.float32, device=dev),
               pos_label=torch.empty(N, dtype=torch.int32, device=dev),
               slot_first=torch.empty(S, dtype=torch.int32, device=dev), slot_count=torch.empty(S, dtype=torch.int32, device=dev))
    d = _abi.SlotDesc()
    d.nodes, d.accel, d.face_count, d.depth = tree.nodes.data_ptr(), tree.accel.data_ptr(), N, depth
    d.slot_ref, d.slot_box, d.pos_label = out["slot_ref"].data_ptr(), out["slot_box"].data_ptr(), out["pos_label"].data_ptr()
    d.slot_first, d.slot_count = out["slot_first"].data_ptr(), out["slot_count"].data_ptr()
    _check("rt_subtree_slots", _abi.lib().rt_subtree_slots(C.byref(d), _stream(stream)))
    return out


def hit_labels(hit_pos: torch.Tensor, pos_label: torch.Tensor, out=None, stream=None):
    if out is None:
        out = torch.empty_like(hit_pos)
    _check("rt_hit_labels", _abi.lib().rt_hit_labels(_p(hit_pos), hit_pos.shape[0], _p(pos_label), _p(out), _stream(stream)))
    return out


def trace_seeded(tree: Tree, orig, dir, proposal, slots: dict, tmax=None, id_mode: int = 0, counters: bool = False,
                 in_proposal: bool = False, out: dict | None = None, schedule: dict | None = None, box_test: bool = True,
                 stream=None) -> dict:
    """core.trace with the proposed subtree walked first; same outputs, bit for bit."""
    d, out = trace_desc(tree, orig, dir, tmax, id_mode, counters, True, None, out, None, True, schedule, stream)
    if not d.accel:
        raise ValueError("the seeded trace needs the traversal blob")
    s = _abi.SeedDesc()
    s.proposal, s.slot_ref, s.slot_count = proposal.data_ptr(), slots["slot_ref"].data_ptr(), slots["slot_ref"].shape[0]
    if box_test:
        s.slot_box = slots["slot_box"].data_ptr()
    if in_proposal:
        out["in_proposal"] = torch.empty(orig.shape[0], dtype=torch.int32, device=orig.device)
        s.in_proposal = out["in_proposal"].data_ptr()
    _check("rt_trace_closest_seeded", _abi.lib().rt_trace_closest_seeded(C.byref(d), C.byref(s), _stream(stream)))
    return out


# ----------------------------------------------------------- batched meshes
def batch_subtree_slots(tree, depth: int = DEPTH, stream=None) -> dict:
    """Per-mesh slot tables of a core.batch_build tree: slot_ref (M, 2^depth),
    slot_box (M, 2^depth, 8), pos_label (global face position -> mesh-local slot)."""
    M, N = tree.mesh_count, tree.faces.shape[0]
    dev = tree.faces.device
    S = 1 << depth
    out = dict(slot_ref=torch.empty((M, S), dtype=torch.int32, device=dev), slot_box=torch.empty((M, S, 8), dtype=torch.float32, device=dev),
               pos_label=torch.empty(N, dtype=torch.int32, device=dev))
    d = _abi.BatchSlotDesc()
    d.mesh_count, d.face_offsets, d.nodes, d.accel = M, tree.face_offsets.data_ptr(), tree.nodes.data_ptr(), tree.accel.data_ptr()
    d.face_count, d.depth = N, depth
    d.slot_ref, d.slot_box, d.pos_label = out["slot_ref"].data_ptr(), out["slot_box"].data_ptr(), out["pos_label"].data_ptr()
    _check("rt_batch_subtree_slots", _abi.lib().rt_batch_subtree_slots(C.byref(d), _stream(stream)))
    return out


def batch_hit_labels(tree, hit_pos, ray_offsets, pos_label, out=None, stream=None):
    if out is None:
        out = torch.empty_like(hit_pos)
    _check("rt_batch_hit_labels", _abi.lib().rt_batch_hit_labels(_p(hit_pos), hit_pos.shape[0], tree.mesh_count, _p(ray_offsets),
                                                                  _p(tree.face_offsets), _p(pos_label), _p(out), _stream(stream)))
    return out


def batch_trace_seeded(tree, orig, dir, ray_offsets, proposal, slots: dict, tmax=None, id_mode: int = 0, counters: bool = False,
                       in_proposal: bool = False, while_while: bool = True, box_test: bool = True, out: dict | None = None,
                       schedule: dict | None = None, order=None, stream=None) -> dict:
    """core.batch_trace with each ray's proposed subtree (of its own mesh) walked first; same outputs, bit for bit."""
    from .core import batch_trace_desc
    d, out = batch_trace_desc(tree, orig, dir, ray_offsets, tmax, id_mode, counters, while_while, out, schedule, order)
    s = _abi.SeedDesc()
    s.proposal, s.slot_ref, s.slot_count = proposal.data_ptr(), slots["slot_ref"].data_ptr(), slots["slot_ref"].shape[1]
    if box_test:
        s.slot_box = slots["slot_box"].data_ptr()
    if in_proposal:
        out["in_proposal"] = torch.empty(orig.shape[0], dtype=torch.int32, device=orig.device)
        s.in_proposal = out["in_proposal"].data_ptr()
    _check("rt_batch_trace_seeded", _abi.lib().rt_batch_trace_seeded(C.byref(d), C.byref(s), _stream(stream)))
    return out
