"""The path-guiding network: CUDA forward/backward against the FP64 oracle
(oracle/guide_oracle.py), the oracle's own gradients against finite
differences, the vMF mixture's sampling against its pdf, and online training.

Tolerances: the kernels round the hash features, every hidden activation and
every back-propagated delta to FP16 (the oracle rounds at the same points but
accumulates in FP64), so outputs and gradients are compared with a relative
L2 error of at most 2e-2 and a cosine similarity of at least 0.999.
"""
import math

import numpy as np
import pytest

import guide_oracle as go


def _rel(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def _cos(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))


def _params(seed, table_scale=0.5, out_scale=1.0):
    rng = np.random.default_rng(seed)
    table = rng.uniform(-table_scale, table_scale, (go.LEVELS, go.T, go.FEATS)).astype(np.float32)
    ws = []
    for li, (o, i) in enumerate(go.LAYERS):
        a = math.sqrt(6.0 / (o + i)) * (out_scale if li == len(go.LAYERS) - 1 else 1.0)
        ws.append(rng.uniform(-a, a, (o, i)).astype(np.float32))
    return table, ws


def _samples(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.random((n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = rng.uniform(0.0, 2.0, n).astype(np.float32)
    return pos, d.astype(np.float32), w


def _to16(table, ws):
    return table.astype(np.float16), [w.astype(np.float16) for w in ws]


def test_oracle_gradients_match_finite_differences(monkeypatch):
    """The oracle's analytic gradients (without its FP16 rounding) against central differences."""
    monkeypatch.setattr(go, "f16", lambda a: np.asarray(a, np.float64))
    table, ws = _params(3, table_scale=0.3, out_scale=0.5)
    table64 = table.astype(np.float64)
    ws64 = [w.astype(np.float64) for w in ws]
    pos, d, w = _samples(6, 4)
    res = go.level_resolutions()
    loss, gt, gw, _ = go.loss_and_grads(table64, ws64, pos, d, w.astype(np.float64), res)

    def f(t, wl):
        return go.loss_and_grads(t, wl, pos, d, w.astype(np.float64), res)[0]

    rng = np.random.default_rng(5)
    eps = 1e-6
    for li in range(len(ws64)):
        for _ in range(4):
            i, j = rng.integers(ws64[li].shape[0]), rng.integers(ws64[li].shape[1])
            wp = [x.copy() for x in ws64]
            wm = [x.copy() for x in ws64]
            wp[li][i, j] += eps
            wm[li][i, j] -= eps
            num = (f(table64, wp) - f(table64, wm)) / (2 * eps)
            assert abs(num - gw[li][i, j]) <= 1e-6 + 1e-5 * abs(num)
    idx, wts = go.corner_indices(pos[:1], res)[7]
    for k in range(3):
        e = int(idx[0, k])
        tp, tm = table64.copy(), table64.copy()
        tp[7, e, 1] += eps
        tm[7, e, 1] -= eps
        num = (f(tp, ws64) - f(tm, ws64)) / (2 * eps)
        assert abs(num - gt[7, e, 1]) <= 1e-6 + 1e-5 * abs(num)


def test_level_resolutions():
    assert go.level_resolutions()[0] == 16 and go.level_resolutions()[-1] == 64
    assert go.level_resolutions(2048)[-1] == 2048 and go.level_resolutions(8)[0] == 8


@pytest.mark.gpu
@pytest.mark.parametrize("n_max", [64, 2048])  # dense levels only / dense and hashed levels
def test_forward_matches_oracle(n_max):
    import optixrender_b200 as rt
    table, ws = _params(11)
    g = rt.Guide(max_resolution=n_max)
    g.set_params(table.reshape(-1), np.concatenate([w.reshape(-1) for w in ws]))
    pos, _, _ = _samples(2048, 12)
    out = g.forward(pos)
    t16, w16 = _to16(table, ws)
    ref, _ = go.forward(t16, w16, pos, go.level_resolutions(n_max))
    print("forward rel", _rel(out, ref), "cos", _cos(out, ref))
    assert _rel(out, ref) < 2e-2 and _cos(out, ref) > 0.999


@pytest.mark.gpu
@pytest.mark.parametrize("n_max,n", [(64, 1024), (2048, 1024), (64, 1000), (2048, 40000)])
def test_gradients_match_oracle(n_max, n):
    """Weight and table gradients of n samples.  The weight gradients are
    summed over 64-sample chunks on the tensor cores: 1000 samples end in a
    partial tile and a chunk of three tiles, 40000 give every CTA several
    chunks."""
    import optixrender_b200 as rt
    table, ws = _params(21, table_scale=0.5, out_scale=0.3)
    g = rt.Guide(max_resolution=n_max)
    g.set_params(table.reshape(-1), np.concatenate([w.reshape(-1) for w in ws]))
    pos, d, w = _samples(n, 22)
    loss, gt, gm = g.gradients(pos, d, w)
    t16, w16 = _to16(table, ws)
    rloss, rgt, rgw, _ = go.loss_and_grads(t16, w16, pos, d, w.astype(np.float64), go.level_resolutions(n_max))
    print("loss", loss, rloss)
    assert abs(loss - rloss) <= 1e-2 * abs(rloss)
    off = 0
    for li, rw in enumerate(rgw):
        n = rw.size
        gw_ = gm[off:off + n].reshape(rw.shape)
        off += n
        print("layer", li, "rel", _rel(gw_, rw), "cos", _cos(gw_, rw))
        assert _rel(gw_, rw) < 2e-2 and _cos(gw_, rw) > 0.999
    rgt = rgt.reshape(-1)
    print("table rel", _rel(gt, rgt), "cos", _cos(gt, rgt))
    assert _rel(gt, rgt) < 2e-2 and _cos(gt, rgt) > 0.999
    assert np.count_nonzero(gt) > 0.9 * np.count_nonzero(rgt)


@pytest.mark.gpu
def test_mixture_sampling_matches_its_pdf():
    """E_q[1 / q(w)] = 4 pi for samples w ~ q, and the pdf the sampler returns
    is the pdf evaluated at the sampled direction."""
    import optixrender_b200 as rt
    table, ws = _params(31, table_scale=0.5, out_scale=0.5)
    g = rt.Guide()
    g.set_params(table.reshape(-1), np.concatenate([w.reshape(-1) for w in ws]))
    n = 1 << 18
    pos = np.repeat(np.random.default_rng(1).random((8, 3)), n // 8, axis=0).astype(np.float32)
    u = np.random.default_rng(2).random((n, 3)).astype(np.float32)
    dirs, p = g.sample(pos, u)
    assert np.allclose(np.linalg.norm(dirs, axis=1), 1.0, atol=1e-5)
    p2 = g.pdf(pos, dirs)
    assert np.allclose(p, p2, rtol=1e-5)
    ref = go.pdf(go.forward(*_to16(table, ws), pos[:: n // 8], go.level_resolutions())[0].repeat(n // 8, 0),
                 dirs.astype(np.float64))
    assert _rel(p, ref) < 2e-2
    for k in range(8):
        sl = slice(k * (n // 8), (k + 1) * (n // 8))
        est = float(np.mean(1.0 / p[sl]))
        assert abs(est - 4 * math.pi) < 0.05 * 4 * math.pi, (k, est)


@pytest.mark.gpu
def test_online_training_learns_a_direction_field():
    """Samples whose directions follow a position-dependent vMF: training
    lowers the loss and the mixture concentrates around the target."""
    import optixrender_b200 as rt
    g = rt.Guide(seed=3)
    rng = np.random.default_rng(4)

    def batch(n):
        pos = rng.random((n, 3)).astype(np.float32)
        mu = pos - 0.5
        mu /= np.linalg.norm(mu, axis=1, keepdims=True)
        kappa = 20.0
        w_ = 1 + np.log(rng.random(n) * (1 - np.exp(-2 * kappa)) + np.exp(-2 * kappa)) / kappa
        t = np.cross(mu, rng.normal(size=(n, 3)))
        t /= np.linalg.norm(t, axis=1, keepdims=True)
        d = w_[:, None] * mu + np.sqrt(np.maximum(0, 1 - w_ * w_))[:, None] * t
        return pos, d.astype(np.float32), np.ones(n, np.float32), mu

    losses = [g.train_step(*batch(1 << 14)[:3]) for _ in range(300)]
    print("loss", losses[0], losses[-1])
    assert np.mean(losses[-20:]) < np.mean(losses[:5]) - 1.0
    pos, _, _, mu = batch(4096)
    good = g.pdf(pos, mu)
    bad = g.pdf(pos, -mu)
    assert np.median(good) > 1.0 and np.median(good) > 20 * np.median(bad)


@pytest.mark.gpu
def test_train_step_is_one_adam_step():
    """A first train step moves every parameter with a gradient by -lr *
    g / (|g| + eps), eps = 1e-10 (Adam's first step, bias-corrected), and
    leaves the rest untouched; the table update covers only the entries the
    levels address, so this checks that none with a gradient is left out."""
    import optixrender_b200 as rt
    lr = 1e-3
    g = rt.Guide(learning_rate=lr, max_resolution=64)
    table, ws = _params(41, table_scale=0.5, out_scale=0.3)
    g.set_params(table.reshape(-1), np.concatenate([w.reshape(-1) for w in ws]))
    pos, d, _ = _samples(8192, 42)
    w = np.ones(len(pos), np.float32)
    _, gt, gm = g.gradients(pos, d, w)
    t0, m0 = g.get_params()
    g.train_step(pos, d, w)
    t1, m1 = g.get_params()
    for name, p0, p1, gr in (("table", t0, t1, gt), ("mlp", m0, m1, gm)):
        big = np.abs(gr) > 1e-3 * np.abs(gr).max()
        step = (p1 - p0)[big].astype(np.float64)
        g64 = gr[big].astype(np.float64)
        want = -lr * g64 / (np.abs(g64) + 1e-10)
        print(name, "entries with gradient", int(big.sum()), "worst", np.abs(step - want).max() / lr)
        assert big.sum() > 100
        assert np.allclose(step, want, rtol=0, atol=2e-3 * lr), name
        zero = gr == 0
        assert np.array_equal(p1[zero], p0[zero]), name


@pytest.mark.gpu
def test_adam_keeps_moments_of_entries_a_lower_resolution_drops():
    """After max_resolution goes down, table entries only the old resolution
    addressed get no more gradient but, as in a dense Adam, keep moving on
    their decaying first moment."""
    import optixrender_b200 as rt
    g = rt.Guide(learning_rate=1e-3, max_resolution=64)
    pos, d, w = _samples(8192, 43)
    _, gt, _ = g.gradients(pos, d, w)
    g.train_step(pos, d, w)
    g.set_hyperparameters(max_resolution=32)
    t1, _ = g.get_params()
    _, gt32, _ = g.gradients(pos, d, w)
    g.train_step(pos, d, w)
    t2, _ = g.get_params()
    dropped = (gt != 0) & (gt32 == 0)
    print("entries addressed only at 64:", int(dropped.sum()))
    assert dropped.sum() > 1000
    assert np.count_nonzero(t2[dropped] != t1[dropped]) > 0.9 * dropped.sum()
