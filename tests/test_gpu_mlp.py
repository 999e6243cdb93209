"""GPU tests of the learned proposal's kernels (mlp.cu) against the numpy oracle
(oracle/mlp_oracle.py, bf16 rounding at the kernels' conversion points).

Tolerances: the kernels sum in a different order than numpy and use the approximate
exp of the GPU for the one-blob features, so a few bf16 roundings land on the other side;
outputs agree within 1e-2 relative to their scale, and each layer's weight gradient within
3 % relative L2 error."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import cavalry_b200 as cav

    return cav.Context(0)


def batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (n, 5)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    w = rng.uniform(0.1, 2.0, n).astype(np.float32)
    return x, d, w


def cuda(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def layer_slices():
    from oracle import mlp_oracle as mo

    out, off = [], 0
    for i, o in mo.LAYERS:
        out.append((slice(off, off + i * o), slice(off + i * o, off + i * o + o)))
        off += i * o + o
    return out


KERNELS = {"tcgen05": 0, "mma_sync": 1}


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("n", [1, 127, 1000, 128 * 148 * 4 + 77])
def test_forward_matches_oracle(ctx, kernel, n):
    """n = 1 and 127: one partial 128-sample tile; 1000: eight tiles, the last partial;
    75,853: every warpgroup of every persistent CTA takes a second tile."""
    import cavalry_b200 as cav
    from oracle import mlp_oracle as mo

    net = cav.Mlp(ctx, seed=5, kernel=KERNELS[kernel])
    p = net.params()
    x, _, _ = batch(n, 1)
    out = net.forward(cuda(x)).cpu().numpy()
    ctx.sync_check()
    sel = np.arange(n) if n <= 4096 else np.random.default_rng(0).choice(n, 4096, replace=False)
    ref, _ = mo.forward(p, x[sel].astype(np.float64), bf=True)
    scale = np.abs(ref).mean()
    assert np.abs(out[sel] - ref).max() <= 1e-2 * scale + 1e-3, np.abs(out[sel] - ref).max()


def test_tcgen05_and_mma_sync_forward_agree(ctx):
    """The two kernels take the same BF16 operands at the same rounding points and differ
    only in the FP32 summation order inside the tensor core, so outputs agree to about
    1e-5 of their scale; a BF16 rounding of an activation that lands on the other side
    moves a few outputs by up to ~1e-3 of scale."""
    import cavalry_b200 as cav

    a = cav.Mlp(ctx, seed=8, kernel=cav.MLP_KERNEL_TCGEN05)
    b = cav.Mlp(ctx, seed=8, kernel=cav.MLP_KERNEL_MMA_SYNC)
    x, _, _ = batch(50_000, 12)
    oa = a.forward(cuda(x)).cpu().numpy()
    ob = b.forward(cuda(x)).cpu().numpy()
    ctx.sync_check()
    scale = np.abs(ob).mean()
    d = np.abs(oa - ob)
    assert np.median(d) <= 1e-5 * scale and d.max() <= 5e-3 * scale, (np.median(d) / scale, d.max() / scale)
    with pytest.raises(cav.CavError):
        a.set_kernel(7)
    a.free()
    b.free()


def test_empty_forward(ctx):
    import torch

    import cavalry_b200 as cav

    net = cav.Mlp(ctx, seed=5)
    assert net.forward(torch.zeros((0, 5), device="cuda")).shape == (0, 32)
    ctx.sync_check()


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_gradients_match_oracle(ctx, kernel):
    import cavalry_b200 as cav
    from oracle import mlp_oracle as mo

    net = cav.Mlp(ctx, seed=6, kernel=KERNELS[kernel])
    rng = np.random.default_rng(9)
    p = net.params()
    p[-32:] = rng.normal(0, 0.5, 32).astype(np.float32)  # spread the lobes
    net.set_params(p)
    x, d, w = batch(4096, 2)
    g, loss = net.gradients(cuda(x), cuda(d), cuda(w))
    ref_loss, ref = mo.gradients(p, x.astype(np.float64), d.astype(np.float64), w.astype(np.float64), bf=True)
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss)
    for k, (sw, sb) in enumerate(layer_slices()):
        for s in (sw, sb):
            err = np.linalg.norm(g[s] - ref[s]) / max(np.linalg.norm(ref[s]), 1e-12)
            assert err < 3e-2, (k, err)


@pytest.mark.parametrize("n", [37, 1000, 16384, 100_003])
def test_tcgen05_and_mma_sync_gradients_agree(ctx, n):
    """The weight gradients of the tcgen05 reduction (per-CTA TMEM partial sums over sample
    ranges, then a fixed-order sum) against the mma.sync kernel's (FP32 atomics) on the same
    batch: both sum the same BF16 products in FP32, so each layer's weights and biases agree
    to FP32 summation order (relative L2 1e-3, allowing a rare activation whose BF16 rounding
    differs between the two forward kernels).  n = 37: one partial stage in one CTA; 1000:
    a stage per CTA; 16,384: the training batch; 100,003: 11 stages per CTA, the last ragged."""
    import cavalry_b200 as cav

    a = cav.Mlp(ctx, seed=6, kernel=cav.MLP_KERNEL_TCGEN05)
    b = cav.Mlp(ctx, seed=6, kernel=cav.MLP_KERNEL_MMA_SYNC)
    rng = np.random.default_rng(9)
    p = a.params()
    p[-32:] = rng.normal(0, 0.5, 32).astype(np.float32)
    a.set_params(p)
    b.set_params(p)
    x, d, w = batch(n, 3)
    ga, la = a.gradients(cuda(x), cuda(d), cuda(w))
    gb, lb = b.gradients(cuda(x), cuda(d), cuda(w))
    ctx.sync_check()
    assert abs(la - lb) <= 1e-4 * abs(lb)
    for k, (sw, sb) in enumerate(layer_slices()):
        for s in (sw, sb):
            err = np.linalg.norm(ga[s] - gb[s]) / max(np.linalg.norm(gb[s]), 1e-12)
            assert err < 1e-3, (k, err)
    a.free()
    b.free()


def test_mixture_pdf_and_sampling(ctx):
    import torch

    import cavalry_b200 as cav
    from oracle import mlp_oracle as mo

    net = cav.Mlp(ctx, seed=7)
    rng = np.random.default_rng(3)
    o = rng.normal(0, 1.5, (1, 32)).astype(np.float32)
    n = 200_000
    outs = cuda(np.repeat(o, n, 0))
    _, d, _ = batch(n, 4)
    pdf = net.pdf(outs, cuda(d)).cpu().numpy()
    ref = mo.mixture_pdf(np.repeat(o, n, 0), d.astype(np.float64))
    assert np.allclose(pdf, ref, rtol=2e-3, atol=1e-6)
    # the sample mean direction equals the mixture's: sum_k w_k mu_k (coth k - 1/k)
    u = torch.rand((n, 3), device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    s = net.sample(outs, u).cpu().numpy()
    assert np.allclose(np.linalg.norm(s, axis=1), 1, atol=1e-4)
    w, mu, kap, _ = mo.decode(o)
    mean = (w[0, :, None] * mu[0] * (1 / np.tanh(kap[0]) - 1 / kap[0])[:, None]).sum(0)
    assert np.abs(s.mean(0) - mean).max() < 0.01


def test_training_learns_a_position_dependent_lobe(ctx):
    """Directions drawn around an axis that depends on the position: training raises the
    log-density of held-out target directions well above the untrained network's."""
    import torch

    import cavalry_b200 as cav

    net = cav.Mlp(ctx, seed=11)
    gen = torch.Generator("cuda").manual_seed(2)

    def make(n):
        x = torch.rand((n, 5), device="cuda", generator=gen)
        axis = torch.stack([x[:, 0] - 0.5, x[:, 1] - 0.5, torch.ones_like(x[:, 0]) * 0.7], 1)
        axis = axis / axis.norm(dim=1, keepdim=True)
        d = axis + 0.15 * torch.randn((n, 3), device="cuda", generator=gen)
        d = d / d.norm(dim=1, keepdim=True)
        return x.contiguous(), d.contiguous(), torch.ones(n, device="cuda")

    xt, dt, _ = make(20000)

    def mean_log_q():
        return float(torch.log(net.pdf(net.forward(xt), dt)).mean())

    before = mean_log_q()
    for _ in range(400):
        x, d, w = make(16384)
        net.train_step(x, d, w, lr=3e-3)
    after = mean_log_q()
    # a uniform density on the sphere has log q = -log(4 pi) = -2.53
    assert after > before + 1.5 and after > 0.5, (before, after)
