"""GPU tests of the launch-shape autotuner: the installed shape changes speed, never hits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results_and_picks_a_candidate():
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    ctx = cav.Context(0)
    pos, idx = scenes.soup(200_000, seed=12)
    bvh = ctx.build(torch.from_numpy(pos).cuda(), torch.from_numpy(idx).cuda(), rounds=2)
    rays = torch.from_numpy(scenes.closest_rays(300_000, seed=13)).cuda()
    srays, lim = scenes.shadow_rays(300_000, seed=14)
    srays, lim = torch.from_numpy(srays).cuda(), torch.from_numpy(lim).cuda()
    p0, t0, _ = bvh.trace_closest(rays)
    o0 = bvh.trace_any(srays, lim)
    best = bvh.autotune(rays)
    assert best["block_threads"] in (64, 128, 256) and best["batch"] in (1, 2, 4, 8, 16, 32)
    assert best["stack"] in (64, 128) and best["ms"] > 0
    if best["stack"] == 64:
        assert bvh.depth() + 1 < 64
    p1, t1, _ = bvh.trace_closest(rays)
    best_any = bvh.autotune(srays, any_hit=True, limit=lim)
    o1 = bvh.trace_any(srays, lim)
    assert best_any["ms"] > 0
    assert np.array_equal(p0.cpu().numpy(), p1.cpu().numpy())
    assert np.array_equal(t0.cpu().numpy().view(np.uint32), t1.cpu().numpy().view(np.uint32))
    assert np.array_equal(o0.cpu().numpy(), o1.cpu().numpy())
    ctx.sync_check()


def test_autotune_fast_mode_keeps_results_and_its_own_shape():
    """Tuning the compressed 8-wide mode installs its shape without touching the exact mode's."""
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    ctx = cav.Context(0)
    pos, idx = scenes.soup(200_000, seed=15)
    bvh = ctx.build(torch.from_numpy(pos).cuda(), torch.from_numpy(idx).cuda(), rounds=2)
    rays = torch.from_numpy(scenes.closest_rays(300_000, seed=16)).cuda()
    exact = bvh.autotune(rays)
    p0, t0, _ = bvh.trace_closest(rays, flags=cav.TRACE_FAST)
    best = bvh.autotune(rays, flags=cav.TRACE_FAST)
    assert best["block_threads"] in (64, 128, 256) and best["batch"] in (1, 2, 4, 8, 16, 32)
    assert best["stack"] == 0 and best["ms"] > 0
    p1, t1, _ = bvh.trace_closest(rays, flags=cav.TRACE_FAST)
    assert np.array_equal(p0.cpu().numpy(), p1.cpu().numpy())
    assert np.array_equal(t0.cpu().numpy().view(np.uint32), t1.cpu().numpy().view(np.uint32))
    # the exact mode's tuned shape is still the one re-tuning picks as installed
    pe, te, _ = bvh.trace_closest(rays)
    assert exact["ms"] > 0 and (pe.cpu().numpy() >= -1).all()
    ctx.sync_check()


def test_every_stack_placement_gives_the_same_hits():
    """The exact kernels' stack in local memory or with its first 16 entries in shared memory
    (deeper entries spill to local memory: some of these rays go deeper than 16), short or
    full, under several block sizes: identical closest and any hits."""
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    ctx = cav.Context(0)
    try:
        pos, idx = scenes.soup(200_000, seed=17)
        bvh = ctx.build(torch.from_numpy(pos).cuda(), torch.from_numpy(idx).cuda(), rounds=2)
        rays = torch.from_numpy(scenes.closest_rays(300_000, seed=18)).cuda()
        srays, lim = scenes.shadow_rays(300_000, seed=19)
        srays, lim = torch.from_numpy(srays).cuda(), torch.from_numpy(lim).cuda()
        ref = None
        for stack in (128, 64):
            for smem in (0, 16):
                for block in (64, 256):
                    ctx.set_trace_config(block, 0, 4)
                    ctx.set_trace_stack(stack, smem)
                    p, t, uv = bvh.trace_closest(rays)
                    o = bvh.trace_any(srays, lim)
                    got = (p.cpu().numpy(), t.cpu().numpy().view(np.uint32), uv.cpu().numpy().view(np.uint32),
                           o.cpu().numpy())
                    if ref is None:
                        ref = got
                    else:
                        for a, b in zip(ref, got):
                            assert np.array_equal(a, b), (stack, smem, block)
        with pytest.raises(RuntimeError):
            ctx.set_trace_stack(128, 8)
        ctx.set_trace_stack(0, 0)
        # the fast mode's node-group stack: the first 8 groups in shared memory or none
        fref = None
        for smem in (0, 8):
            ctx.set_trace_stack(0, smem, flags=cav.TRACE_FAST)
            p, t, uv = bvh.trace_closest(rays, flags=cav.TRACE_FAST)
            o = bvh.trace_any(srays, lim, flags=cav.TRACE_FAST)
            got = (p.cpu().numpy(), t.cpu().numpy().view(np.uint32), uv.cpu().numpy().view(np.uint32), o.cpu().numpy())
            if fref is None:
                fref = got
            else:
                for a, b in zip(fref, got):
                    assert np.array_equal(a, b), ("fast", smem)
        assert np.array_equal(fref[3], ref[3])  # any-hit answers agree across the modes
        with pytest.raises(RuntimeError):
            ctx.set_trace_stack(0, 16, flags=cav.TRACE_FAST)
        ctx.set_trace_stack(0, 0, flags=cav.TRACE_FAST)
        ctx.sync_check()
        bvh.free()
    finally:
        ctx.close()
