"""FP64 restatement of the path-guiding network (the learned proposal).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
guiding kernels.  The network has no counterpart in the reference renderer;
it restates published methods:

* multiresolution hash encoding (Mueller, Evans, Schied, Keller, "Instant
  Neural Graphics Primitives", SIGGRAPH 2022): 16 levels of geometrically
  growing resolution from 16 to 64 (any finest resolution may be chosen), 2
  features per level, 2^19 entries per level, trilinear interpolation of the 8 cell
  corners, dense indexing where the level's grid fits the table and the
  spatial hash (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod 2^19 elsewhere;
* a 32 -> 64 -> 64 -> 64 -> 32 MLP without biases, ReLU on the hidden layers;
* an 8-lobe von Mises-Fisher mixture head (lobe k: weight logit, log
  concentration, polar and azimuth angle through sigmoids), as in neural
  parametric mixtures for path guiding (Dong et al. 2023);
* the KL-divergence training loss of neural importance sampling (Mueller et
  al., ACM TOG 2019): -(1/B) sum_j s_j log q(w_j | x_j), s_j = L_j / p_j.

Precision mirrors the CUDA kernels where it decides results: positions are
scaled per level in float32, hash-table entries and MLP weights are read as
float16, each hidden activation and each back-propagated delta is rounded to
float16 where the kernels round it; everything else is float64.
"""
from __future__ import annotations

import math

import numpy as np

LEVELS, FEATS, LOG2_T = 16, 2, 19
T = 1 << LOG2_T
N_MIN, N_MAX = 16, 64   # coarsest level min(16, n_max), finest n_max
LAYERS = [(64, 32), (64, 64), (64, 64), (32, 64)]  # (out, in)
LOBES = 8
KAPPA_LO, KAPPA_HI = -2.0, 4.0
PRIMES = (1, 2654435761, 805459861)


def level_resolutions(n_max=None):
    n_max = N_MAX if n_max is None else n_max
    lo = min(N_MIN, n_max)
    b = math.exp((math.log(n_max) - math.log(lo)) / (LEVELS - 1))
    return [int(math.floor(lo * b ** l + 1e-6)) for l in range(LEVELS)]


def mlp_param_count():
    return sum(o * i for o, i in LAYERS)


def corner_indices(pos01, level_res):
    """(n, 3) float32 positions in [0, 1] -> per level: (n, 8) table indices, (n, 8) weights (float64)."""
    out = []
    x = pos01.astype(np.float32)
    for res in level_res:
        p = x * np.float32(res)                        # float32, as the kernel
        c = np.minimum(np.floor(p), np.float32(res - 1)).astype(np.int64)
        f = (p - c.astype(np.float32)).astype(np.float64)
        dense = (res + 1) ** 3 <= T
        idx, w = [], []
        for corner in range(8):
            d = np.array([(corner >> a) & 1 for a in range(3)])
            g = c + d
            if dense:
                ii = g[:, 0] + g[:, 1] * (res + 1) + g[:, 2] * (res + 1) ** 2
            else:
                gu = g.astype(np.uint64)
                h = (gu[:, 0] * np.uint64(PRIMES[0])) ^ (gu[:, 1] * np.uint64(PRIMES[1])) ^ \
                    (gu[:, 2] * np.uint64(PRIMES[2]))
                ii = (h & np.uint64(0xFFFFFFFF)).astype(np.int64) & (T - 1)
            ww = np.ones(len(x))
            for a in range(3):
                ww = ww * (f[:, a] if d[a] else 1.0 - f[:, a])
            idx.append(ii)
            w.append(ww)
        out.append((np.stack(idx, 1), np.stack(w, 1)))
    return out


def encode(table16, pos01, level_res):
    """table16: (LEVELS, T, 2) float16.  Returns (n, 32) features (float64, before the float16 rounding)."""
    feats = np.zeros((len(pos01), LEVELS * FEATS))
    for l, (idx, w) in enumerate(corner_indices(pos01, level_res)):
        tab = table16[l].astype(np.float64)
        for k in range(FEATS):
            feats[:, 2 * l + k] = (w * tab[idx, k]).sum(1)
    return feats


def f16(a):
    return np.asarray(a, np.float64).astype(np.float16).astype(np.float64)


def forward(table16, weights16, pos01, level_res):
    """Returns raw outputs (n, 32) and the activations needed by backward."""
    x = f16(encode(table16, pos01, level_res))
    acts = [x]
    h = x
    for li, w in enumerate(weights16):
        z = h @ w.astype(np.float64).T
        if li < len(weights16) - 1:
            h = f16(np.maximum(z, 0.0))
            acts.append(h)
        else:
            out = z
    return out, acts


def head(out):
    """Raw outputs -> (weights (n, 8), kappa (n, 8), mu (n, 8, 3), pieces for the gradient)."""
    o = out.reshape(-1, LOBES, 4)
    logits = o[..., 0]
    e = np.exp(logits - logits.max(1, keepdims=True))
    wts = e / e.sum(1, keepdims=True)
    kr = o[..., 1]
    kraw = np.clip(kr, KAPPA_LO, KAPPA_HI)
    kappa = np.exp(kraw)
    st, sp = 1 / (1 + np.exp(-o[..., 2])), 1 / (1 + np.exp(-o[..., 3]))
    th, ph = math.pi * st, 2 * math.pi * sp
    mu = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1)
    return wts, kappa, mu, dict(kr=kr, st=st, sp=sp, th=th, ph=ph)


def vmf(kappa, mu, d):
    """vMF density of unit directions d (n, 3) for every lobe: (n, 8)."""
    cos = (mu * d[:, None, :]).sum(-1)
    return kappa / (2 * math.pi * -np.expm1(-2 * kappa)) * np.exp(kappa * (cos - 1))


def pdf(out, d):
    wts, kappa, mu, _ = head(out)
    return (wts * vmf(kappa, mu, d)).sum(1)


def loss_and_grad_out(out, d, s, batch):
    """Loss (1/B) sum s_j * -log q_j and its gradient with respect to the raw outputs."""
    wts, kappa, mu, pc = head(out)
    dk = vmf(kappa, mu, d)
    q = (wts * dk).sum(1)
    loss = float((s * -np.log(q)).sum() / batch)
    r = wts * dk / q[:, None]
    g = (s / batch)[:, None]
    cos = (mu * d[:, None, :]).sum(-1)
    dlogk = 1 / kappa - 2 / np.expm1(2 * kappa) + (cos - 1)
    clamp = (pc["kr"] >= KAPPA_LO) & (pc["kr"] <= KAPPA_HI)
    th, ph = pc["th"], pc["ph"]
    dmu_th = np.stack([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)], -1)
    dmu_ph = np.stack([-np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph), np.zeros_like(th)], -1)
    grad = np.zeros_like(out).reshape(-1, LOBES, 4)
    grad[..., 0] = g * (wts - r)
    grad[..., 1] = g * -r * dlogk * kappa * clamp
    grad[..., 2] = g * -r * kappa * (dmu_th * d[:, None, :]).sum(-1) * math.pi * pc["st"] * (1 - pc["st"])
    grad[..., 3] = g * -r * kappa * (dmu_ph * d[:, None, :]).sum(-1) * 2 * math.pi * pc["sp"] * (1 - pc["sp"])
    return loss, grad.reshape(out.shape)


def loss_and_grads(table16, weights16, pos01, d, s, level_res, batch=None):
    """Loss and its gradients with respect to the hash table (LEVELS, T, 2) and each weight matrix."""
    batch = len(pos01) if batch is None else batch
    out, acts = forward(table16, weights16, pos01, level_res)
    loss, dout = loss_and_grad_out(out, d, s, batch)
    gw = [None] * len(weights16)
    delta = f16(dout)
    for li in range(len(weights16) - 1, -1, -1):
        gw[li] = delta.T @ acts[li]
        back = delta @ weights16[li].astype(np.float64)
        if li > 0:
            delta = f16(back * (acts[li] > 0))
        else:
            dx = back
    gtab = np.zeros((LEVELS, T, FEATS))
    for l, (idx, w) in enumerate(corner_indices(pos01, level_res)):
        for k in range(FEATS):
            np.add.at(gtab[l, :, k], idx.reshape(-1), (w * dx[:, 2 * l + k][:, None]).reshape(-1))
    return loss, gtab, gw, out


def init_params(seed):
    """The kernels' initialisation: table U(-1e-4, 1e-4), weights U(+-sqrt(6 / (fan_in + fan_out)))."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1e-4, 1e-4, (LEVELS, T, FEATS)).astype(np.float32)
    ws = [rng.uniform(-1, 1, (o, i)).astype(np.float32) * np.float32(math.sqrt(6.0 / (o + i))) for o, i in LAYERS]
    return table, ws
