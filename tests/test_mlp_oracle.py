"""CPU tests of the MLP oracle: its analytic gradient against central finite differences
(float64), its bf16 rounding, and its mixture density integrating to one."""
import numpy as np


def batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (n, 5))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = rng.uniform(0.1, 2.0, n)
    return x, d, w


def test_analytic_gradient_matches_finite_differences():
    from oracle import mlp_oracle as mo

    p = mo.init_params(3).astype(np.float64)
    # give the biases and logits some spread so every lobe matters
    rng = np.random.default_rng(4)
    p += rng.normal(0, 0.05, p.shape)
    x, d, w = batch(12, 5)
    _, g = mo.gradients(p, x, d, w, bf=False)
    idx = np.concatenate([rng.choice(mo.n_params(), 300, replace=False), np.arange(mo.n_params() - 32, mo.n_params())])
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (mo.loss_only(pp, x, d, w) - mo.loss_only(pm, x, d, w)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    from oracle import mlp_oracle as mo

    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway: ties to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - x[3]) <= 2 ** -7 * abs(x[3])


def test_mixture_integrates_to_one():
    from oracle import mlp_oracle as mo

    rng = np.random.default_rng(7)
    o = rng.normal(0, 1.5, (1, 32))
    # Fibonacci sphere quadrature
    m = 200000
    k = np.arange(m) + 0.5
    z = 1 - 2 * k / m
    phi = np.pi * (1 + 5 ** 0.5) * k
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    pdf = mo.mixture_pdf(np.repeat(o, m, 0), dirs)
    assert abs(pdf.mean() * 4 * np.pi - 1) < 1e-3
