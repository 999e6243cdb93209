"""GPU tests of the compressed 8-wide fast traversal mode (CAV_TRACE_FAST): the same
closest-hit distances and any-hit answers as the exact mode; a different triangle only where
two hits tie in distance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mt_distance(rays, v0, v1, v2):
    """Moller-Trumbore distance (float64) of each ray to one triangle; nan on a miss."""
    o, d = rays[:, 0:3].astype(np.float64), rays[:, 4:7].astype(np.float64)
    e1, e2 = (v1 - v0).astype(np.float64), (v2 - v0).astype(np.float64)
    p = np.cross(d, e2)
    det = (e1 * p).sum(1)
    tv = o - v0
    u = (tv * p).sum(1) / det
    q = np.cross(tv, e1)
    v = (d * q).sum(1) / det
    t = (e2 * q).sum(1) / det
    ok = (u >= -1e-6) & (v >= -1e-6) & (u + v <= 1 + 1e-6) & (t > 0)
    return np.where(ok, t, np.nan)


@pytest.mark.parametrize("kind,rounds", [("soup", 0), ("soup", 3), ("room", 0), ("spheres", 2)])
def test_fast_matches_exact(kind, rounds):
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    ctx = cav.Context(0)
    if kind == "soup":
        pos, idx = scenes.soup(200_000, seed=21)
        rays = scenes.closest_rays(400_000, seed=22)
        srays, lim = scenes.shadow_rays(400_000, seed=23)
    else:
        sc = scenes.mini_room() if kind == "room" else scenes.sphere_scene(12, 3, seed=24)
        pos, idx = sc["positions"], sc["indices"]
        lo, hi = pos.min(0), pos.max(0)
        rng = np.random.default_rng(25)
        o = rng.uniform(lo, hi, (300_000, 3)).astype(np.float32)
        d = rng.normal(size=(300_000, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        rays = scenes.make_rays(o, d)
        p = rng.uniform(lo, hi, (300_000, 3)).astype(np.float32)
        v = p - o
        dist = np.linalg.norm(v, axis=1).astype(np.float32)
        srays = scenes.make_rays(o, (v / dist[:, None]).astype(np.float32))
        lim = dist
    # rays parallel to one or two axes (zero direction components, +0 and -0)
    rng = np.random.default_rng(26)
    lo, hi = pos.min(0), pos.max(0)
    m = 3000
    o = rng.uniform(lo, hi, (m, 3)).astype(np.float32)
    d = rng.normal(size=(m, 3)).astype(np.float32)
    zero = rng.integers(0, 3, m)
    d[np.arange(m), zero] = np.where(rng.random(m) < 0.5, 0.0, -0.0)
    two = rng.random(m) < 0.3
    d[two, (zero[two] + 1) % 3] = 0.0
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rays = np.concatenate([rays, scenes.make_rays(o, d)])
    bvh = ctx.build(torch.from_numpy(pos).cuda(), torch.from_numpy(idx).cuda(), rounds=rounds)
    r = torch.from_numpy(rays).cuda()
    pe, te, _ = bvh.trace_closest(r)
    pf, tf, _ = bvh.trace_closest(r, flags=cav.TRACE_FAST)
    pe, te, pf, tf = (x.cpu().numpy() for x in (pe, te, pf, tf))
    assert np.array_equal(pe >= 0, pf >= 0)
    both = pe >= 0
    rel = np.abs(tf[both] - te[both]) / np.abs(te[both])
    assert rel.max(initial=0) <= 1e-6, rel.max()
    diff = both & (pe != pf)
    # a different triangle only at a tie: the fast mode's triangle is hit at the exact mode's
    # distance (coplanar triangles such as a box standing on the floor, shared edges)
    k = np.nonzero(diff)[0]
    if len(k):
        tri = idx[pf[k]].astype(np.int64)
        t_other = mt_distance(rays[k], pos[tri[:, 0]], pos[tri[:, 1]], pos[tri[:, 2]])
        assert np.all(np.abs(t_other - te[k]) <= 1e-5 * np.abs(te[k])), np.abs(t_other - te[k]).max()
    assert diff.mean() <= 1e-2
    sr, sl = torch.from_numpy(srays).cuda(), torch.from_numpy(lim).cuda()
    oe = bvh.trace_any(sr, sl).cpu().numpy()
    of = bvh.trace_any(sr, sl, flags=cav.TRACE_FAST).cpu().numpy()
    assert (oe != of).mean() <= 1e-4
    ctx.sync_check()


@pytest.mark.parametrize("n", [30_000, 70_001, 1_000_017])
def test_reordered_batches_return_the_same_results(n):
    """CAV_TRACE_REORDER traces a batch in the Morton order of its ray origins and writes each
    ray's results back to its own index: closest and any hit, exact and fast modes, equal
    bit for bit to the given order (30,000 rays: below the threshold, traced as given)."""
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    ctx = cav.Context(0)
    try:
        pos, idx = scenes.soup(50_000, seed=71)
        bvh = ctx.build(torch.from_numpy(pos).cuda(), torch.from_numpy(idx).cuda(), rounds=3)
        rays = torch.from_numpy(scenes.closest_rays(n, seed=72)).cuda()
        srays, lim = scenes.shadow_rays(n, seed=73)
        srays, lim = torch.from_numpy(srays).cuda(), torch.from_numpy(lim).cuda()
        for mode in (cav.TRACE_EXACT, cav.TRACE_FAST):
            want = [a.cpu().numpy() for a in bvh.trace_closest(rays, flags=mode)]
            got = [a.cpu().numpy() for a in bvh.trace_closest(rays, flags=mode | cav.TRACE_REORDER)]
            for w, g in zip(want, got):
                assert np.array_equal(np.ascontiguousarray(w).view(np.uint32), np.ascontiguousarray(g).view(np.uint32))
            occ_w = bvh.trace_any(srays, lim, flags=mode).cpu().numpy()
            occ_g = bvh.trace_any(srays, lim, flags=mode | cav.TRACE_REORDER).cpu().numpy()
            assert np.array_equal(occ_w, occ_g)
        if n > 70_001:  # the autotuner accepts the flag and tunes on the reordered sample
            shape = bvh.autotune(rays[:200_000].contiguous(), flags=cav.TRACE_EXACT | cav.TRACE_REORDER)
            assert shape["block_threads"] > 0 and shape["ms"] > 0
        ctx.sync_check()
        bvh.free()
    finally:
        ctx.close()
