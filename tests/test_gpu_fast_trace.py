"""GPU tests of the 4-wide fast traversal mode (CAV_TRACE_FAST): the same closest-hit
distances and any-hit answers as the exact mode; a different triangle only where two hits
tie in distance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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
    assert diff.mean() <= 1e-3  # equal-distance ties only
    sr, sl = torch.from_numpy(srays).cuda(), torch.from_numpy(lim).cuda()
    oe = bvh.trace_any(sr, sl).cpu().numpy()
    of = bvh.trace_any(sr, sl, flags=cav.TRACE_FAST).cpu().numpy()
    assert (oe != of).mean() <= 1e-4
    ctx.sync_check()
