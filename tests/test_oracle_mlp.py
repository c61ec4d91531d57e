"""CPU checks of the proposal-network oracle: its backward formulas against
central finite differences (float64, no BF16 rounding), its BF16 rounding, and
its feature encoding against the formula written out directly."""
import numpy as np

from oracle import mlp_oracle as M


def _tiny_net(rng, d_in=12, hidden=8, classes=16):
    W = [rng.normal(0, 0.5, (hidden, d_in)), rng.normal(0, 0.5, (hidden, hidden)), rng.normal(0, 0.5, (hidden, hidden)),
         rng.normal(0, 0.5, (classes, hidden))]
    b = [rng.normal(0, 0.1, hidden), rng.normal(0, 0.1, hidden), rng.normal(0, 0.1, hidden), rng.normal(0, 0.1, classes)]
    return W, b


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    W, b = _tiny_net(rng)
    X = rng.normal(0, 1, (10, 12))
    labels = rng.integers(0, 16, 10)
    _, dW, db = M.train_grads(X, W, b, labels, rounding=False)
    eps = 1e-6
    for l in range(4):
        for _ in range(6):
            i, j = rng.integers(0, W[l].shape[0]), rng.integers(0, W[l].shape[1])
            Wp = [w.copy() for w in W]
            Wm = [w.copy() for w in W]
            Wp[l][i, j] += eps
            Wm[l][i, j] -= eps
            fd = (M.loss_only(X, Wp, b, labels) - M.loss_only(X, Wm, b, labels)) / (2 * eps)
            assert abs(fd - dW[l][i, j]) <= 1e-6 + 1e-5 * abs(fd), (l, i, j, fd, dW[l][i, j])
        i = rng.integers(0, b[l].shape[0])
        bp = [x.copy() for x in b]
        bm = [x.copy() for x in b]
        bp[l][i] += eps
        bm[l][i] -= eps
        fd = (M.loss_only(X, W, bp, labels) - M.loss_only(X, W, bm, labels)) / (2 * eps)
        assert abs(fd - db[l][i]) <= 1e-6 + 1e-5 * abs(fd)


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3.0e38, 1e-40], np.float32)
    r = M.bf16(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0  # halfway, ties to even (mantissa 0)
    assert r[2] == np.float32(1.0 + 4 * 2 ** -8)  # halfway, ties to even (rounds up)
    assert r[3] == 1.0
    assert r[4] == -2.5
    assert (r.view(np.uint32) & 0xFFFF == 0).all()


def test_features_formula():
    rng = np.random.default_rng(1)
    o = np.zeros((5, 4), np.float32)
    d = np.zeros((5, 4), np.float32)
    o[:, :3] = rng.uniform(-2, 3, (5, 3))
    d[:, :3] = rng.normal(size=(5, 3))
    box = (-2.0, -2.0, -2.0, 3.0, 3.0, 3.0)
    f = M.features(o, d, box, rounding=False)
    u0 = (o[2, 0] - 0.5) * (2.0 / 5.0)
    assert abs(f[2, 2 * 3] - np.sin(np.pi * 8 * u0)) < 1e-5
    dn = d[3, :3] / np.linalg.norm(d[3, :3])
    assert abs(f[3, 24 * 4 + 1] - np.cos(np.pi * dn[1])) < 1e-6
    assert (f[:, 144:] == 0).all()
    fr = M.features(o, d, box)
    assert np.abs(fr - f).max() <= 2 ** -8
