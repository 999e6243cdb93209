"""MLP oracle — TEST INFRASTRUCTURE, not part of the product.

A numpy restatement of the learned directional proposal of cavalry_b200/csrc/mlp.cu:
one-blob encoding (5 inputs x 32 Gaussian bins), 160 -> 64 -> 64 -> 64 -> 32 with ReLU,
the 8-lobe von Mises-Fisher mixture decoded from the 32 outputs, the loss
mean(-w log q(omega)) and its gradient with respect to every parameter.

Two modes:
  * ``bf16=True`` rounds to bfloat16 (round-to-nearest-even) exactly where the kernels
    convert: the one-blob features, the weights, each ReLU output, the output gradient and
    each back-propagated gradient; sums are float32.  This is the reference the GPU
    gradients are compared with (tests/test_gpu_mlp.py), within a stated tolerance (the
    GPU's summation order and approximate exp differ).
  * ``bf16=False`` is float64 throughout; tests/test_mlp_oracle.py checks its analytic
    gradient against central finite differences.

Parameter layout (as cav_mlp_get_params): per layer W[out][in] then b[out].
"""
from __future__ import annotations

import numpy as np

N_IN, BINS, F0, H, OUT, LOBES = 5, 32, 160, 64, 32, 8
LAYERS = [(F0, H), (H, H), (H, H), (H, OUT)]


def n_params() -> int:
    return sum(i * o + o for i, o in LAYERS)


def unpack(p: np.ndarray):
    out, off = [], 0
    for i, o in LAYERS:
        W = p[off:off + i * o].reshape(o, i)
        off += i * o
        b = p[off:off + o]
        off += o
        out.append((W, b))
    return out


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    x = np.asarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    r = rounded.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(x), x, r)


def one_blob(x: np.ndarray, dtype) -> np.ndarray:
    c = (np.arange(BINS, dtype=np.float64) + 0.5) / BINS
    z = (x[:, :, None].astype(np.float64) - c[None, None, :]) * BINS
    return np.exp(-0.5 * z * z).reshape(len(x), F0).astype(dtype)


def forward(p: np.ndarray, x: np.ndarray, bf: bool):
    dt = np.float32 if bf else np.float64
    layers = unpack(p.astype(dt))
    rnd = bf16 if bf else (lambda a: a)
    acts = [rnd(one_blob(x, dt))]
    h = acts[0]
    for li, (W, b) in enumerate(layers):
        z = h @ rnd(W).T + b
        if li < 3:
            h = rnd(np.maximum(z, 0))
            acts.append(h)
        else:
            h = z
    return h, acts


def _sig(a):
    return 1.0 / (1.0 + np.exp(-a))


def _softplus(a):
    return np.where(a > 15, a, np.log1p(np.exp(np.minimum(a, 15))))


def decode(o: np.ndarray):
    o = o.reshape(len(o), LOBES, 4).astype(np.float64)
    logit, a, b, c = o[..., 0], o[..., 1], o[..., 2], o[..., 3]
    w = np.exp(logit - logit.max(1, keepdims=True))
    w /= w.sum(1, keepdims=True)
    th, ph = np.pi * _sig(a), 2 * np.pi * _sig(b)
    mu = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1)
    kap = np.minimum(_softplus(c) + 0.01, 500.0)
    norm = kap / (2 * np.pi * (1 - np.exp(-2 * kap)))
    return w, mu, kap, norm


def mixture_pdf(o: np.ndarray, d: np.ndarray) -> np.ndarray:
    w, mu, kap, norm = decode(o)
    c = (mu * d[:, None, :]).sum(-1)
    return (w * norm * np.exp(kap * (c - 1))).sum(1)


def loss_and_dout(o: np.ndarray, d: np.ndarray, wt: np.ndarray):
    """mean(-w log q) and its gradient w.r.t. the 32 outputs (float64)."""
    n = len(o)
    o = o.astype(np.float64)
    w, mu, kap, norm = decode(o)
    c = (mu * d[:, None, :]).sum(-1)
    v = norm * np.exp(kap * (c - 1))
    q = np.maximum((w * v).sum(1), 1e-20)
    r = w * v / q[:, None]
    s = (wt / n)[:, None]
    oo = o.reshape(n, LOBES, 4)
    sa, sb = _sig(oo[..., 1]), _sig(oo[..., 2])
    th, ph = np.pi * sa, 2 * np.pi * sb
    dth = (np.cos(th) * np.cos(ph) * d[:, None, 0] + np.cos(th) * np.sin(ph) * d[:, None, 1]
           - np.sin(th) * d[:, None, 2])
    dph = -np.sin(th) * np.sin(ph) * d[:, None, 0] + np.sin(th) * np.cos(ph) * d[:, None, 1]
    e2 = np.exp(-2 * kap)
    dlv = 1 / kap - 2 * e2 / (1 - e2) + (c - 1)
    dk = np.where(_softplus(oo[..., 3]) + 0.01 < 500, _sig(oo[..., 3]), 0.0)
    g = np.zeros((n, LOBES, 4))
    g[..., 0] = -s * (r - w)
    g[..., 1] = -s * r * kap * dth * np.pi * sa * (1 - sa)
    g[..., 2] = -s * r * kap * dph * 2 * np.pi * sb * (1 - sb)
    g[..., 3] = -s * r * dlv * dk
    loss = float((-(wt / n) * np.log(q)).sum())
    return loss, g.reshape(n, OUT)


def gradients(p: np.ndarray, x: np.ndarray, d: np.ndarray, wt: np.ndarray, bf: bool = True):
    """(loss, gradient vector in the parameter layout)."""
    dt = np.float32 if bf else np.float64
    rnd = bf16 if bf else (lambda a: a)
    out, acts = forward(p, x, bf)
    loss, dout = loss_and_dout(out, d, wt)
    layers = unpack(p.astype(dt))
    grads = [None] * 4
    dy = rnd(dout.astype(dt))  # layer 3 output gradient
    for li in (3, 2, 1, 0):
        W, _ = layers[li]
        x_in = acts[li]
        grads[li] = (dy.T @ x_in, dy.sum(0))
        if li > 0:
            dx = dy @ rnd(W)
            dy = rnd(np.where(acts[li] > 0, dx, 0).astype(dt))
    flat = []
    for gW, gb in grads:
        flat += [gW.reshape(-1), gb]
    return loss, np.concatenate(flat).astype(np.float64)


def loss_only(p: np.ndarray, x: np.ndarray, d: np.ndarray, wt: np.ndarray) -> float:
    out, _ = forward(p, x, False)
    return loss_and_dout(out, d, wt)[0]


def init_params(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    parts = []
    for i, o in LAYERS:
        a = np.sqrt(6.0 / (i + o))
        parts += [rng.uniform(-a, a, i * o), np.zeros(o)]
    return np.concatenate(parts).astype(np.float32)
