"""GPU tests of the failure paths: each is made to happen on the host side or by input that
the kernels' own checks turn into an error status (no fault, trap or hang is provoked).

* A vertex index outside [0, num_vertices) is flagged by the build's leaf-box pass (no load
  leaves the position array) and reported as CAV_ERR_INVALID_ARGUMENT by cav_sync_check;
  the context stays usable and the next build of valid input is exact.
* Bounded waits (sort look-back, tcgen05 completion) are made to run out by injected stalls
  that withhold what they wait for; the traversal step limit by a small limit.
* Device allocations fail by injection at a chosen point.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CAV_ERR_INVALID_ARGUMENT = 1


def _soup(n, seed):
    from cavalry_b200 import scenes

    return scenes.soup(n, seed=seed)


@pytest.mark.parametrize("bad", [-1, "nv", 2**31 - 1])
@pytest.mark.parametrize("given_bounds", [False, True])
def test_out_of_range_vertex_index_is_reported(bad, given_bounds):
    import torch

    import cavalry_b200 as cav
    from oracle import pyoracle as po

    ctx = cav.Context(0)
    try:
        pos, idx = _soup(3000, seed=21)
        bad_idx = idx.copy()
        nv = pos.shape[0]
        bad_idx[1234, 1] = nv if bad == "nv" else bad
        bounds = [0, 0, 0, 1, 1, 1] if given_bounds else None
        bvh = ctx.build(torch.from_numpy(pos).cuda(), torch.from_numpy(bad_idx).cuda(), scene_bounds=bounds, rounds=1)
        with pytest.raises(cav.CavError) as e:
            ctx.sync_check()
        assert e.value.status == CAV_ERR_INVALID_ARGUMENT
        bvh.free()
        # the flag was cleared and the context still builds exactly
        bvh = ctx.build(torch.from_numpy(pos).cuda(), torch.from_numpy(idx).cuda(), scene_bounds=bounds, rounds=1)
        ctx.sync_check()
        _, ms, perm = bvh.export_stages()
        o = po.build(pos, idx, codes=bvh.export_stages()[0], rounds=1)
        assert np.array_equal(ms, o["sorted"]) and np.array_equal(perm, o["perm"])
        bvh.free()
    finally:
        ctx.close()


def test_out_of_range_vertex_index_in_a_batched_build():
    import torch

    import cavalry_b200 as cav

    ctx = cav.Context(0)
    try:
        scenes = []
        for k in range(3):
            pos, idx = _soup(500 + 300 * k, seed=40 + k)
            if k == 1:
                idx = idx.copy()
                idx[7, 2] = pos.shape[0] + 5
            scenes.append((torch.from_numpy(pos).cuda(), torch.from_numpy(idx).cuda()))
        trees = ctx.build_batch(scenes, rounds=0)
        with pytest.raises(cav.CavError) as e:
            ctx.sync_check()
        assert e.value.status == CAV_ERR_INVALID_ARGUMENT
        for t in trees:
            t.free()
    finally:
        ctx.close()


CAV_ERR_OUT_OF_MEMORY = 3
CAV_ERR_TIMEOUT = 4


def _gpu(a):
    import torch

    return torch.from_numpy(a).cuda()


def test_sort_lookback_wait_runs_out_and_reports():
    """CAV_INJECT_SORT_STALL: the first tile of every sort pass withholds its counts, so the
    later tiles' look-back waits (bounded at 50 ms here) run out.  The build completes, the
    failure is reported as CAV_ERR_TIMEOUT, the failed tree traces safely with no hits, and
    the context builds exactly again once the injection is cleared."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes
    from oracle import pyoracle as po

    ctx = cav.Context(0)
    try:
        pos, idx = _soup(20000, seed=30)
        rays = _gpu(scenes.closest_rays(4096, seed=31))
        srays, lim = scenes.shadow_rays(4096, seed=32)
        ctx.set_limits(sort_wait_s=0.05)
        ctx.inject(cav.INJECT_SORT_STALL, 1)
        bvh = ctx.build(_gpu(pos), _gpu(idx), rounds=1)
        with pytest.raises(cav.CavError) as e:
            ctx.sync_check()
        assert e.value.status == CAV_ERR_TIMEOUT
        prim, _, _ = bvh.trace_closest(rays)
        occ = bvh.trace_any(_gpu(srays), _gpu(lim))
        ctx.sync_check()  # tracing the failed tree raised nothing new
        assert (prim.cpu().numpy() == -1).all() and (occ.cpu().numpy() == 0).all()
        bvh.free()
        ctx.inject(cav.INJECT_NONE)
        ctx.set_limits()
        bvh = ctx.build(_gpu(pos), _gpu(idx), rounds=1)
        ctx.sync_check()
        mu, ms, perm = bvh.export_stages()
        o = po.build(pos, idx, codes=mu, rounds=1)
        assert np.array_equal(ms, o["sorted"]) and np.array_equal(perm, o["perm"])
        bvh.free()
    finally:
        ctx.close()


def test_traversal_step_limit_stops_rays_and_reports():
    """A step limit of 8 visits stops almost every ray of a 20k soup (prim -2, occluded 2) in
    both traversal modes and cav_sync_check reports CAV_ERR_TIMEOUT; with the default limit
    the same rays trace to the same hits as before."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    ctx = cav.Context(0)
    try:
        pos, idx = _soup(20000, seed=33)
        bvh = ctx.build(_gpu(pos), _gpu(idx), rounds=2)
        rays = _gpu(scenes.closest_rays(8192, seed=34))
        srays, lim = scenes.shadow_rays(8192, seed=35)
        srays, lim = _gpu(srays), _gpu(lim)
        want = [bvh.trace_closest(rays, flags=f)[0].cpu().numpy() for f in (cav.TRACE_EXACT, cav.TRACE_FAST)]
        occ_want = bvh.trace_any(srays, lim).cpu().numpy()
        ctx.sync_check()
        ctx.set_limits(max_trace_steps=8)
        for f, w in zip((cav.TRACE_EXACT, cav.TRACE_FAST), want):
            p = bvh.trace_closest(rays, flags=f)[0].cpu().numpy()
            ran = p != -2  # rays that finished within the limit keep their hits
            assert (~ran).mean() > 0.5 and np.array_equal(p[ran], w[ran])
            with pytest.raises(cav.CavError) as e:
                ctx.sync_check()
            assert e.value.status == CAV_ERR_TIMEOUT
        occ = bvh.trace_any(srays, lim).cpu().numpy()
        assert (occ == 2).mean() > 0.1 and np.array_equal(occ[occ != 2], occ_want[occ != 2])
        with pytest.raises(cav.CavError) as e:
            ctx.sync_check()
        assert e.value.status == CAV_ERR_TIMEOUT
        ctx.set_limits()
        for f, w in zip((cav.TRACE_EXACT, cav.TRACE_FAST), want):
            assert np.array_equal(bvh.trace_closest(rays, flags=f)[0].cpu().numpy(), w)
        assert np.array_equal(bvh.trace_any(srays, lim).cpu().numpy(), occ_want)
        ctx.sync_check()
        bvh.free()
    finally:
        ctx.close()


@pytest.mark.parametrize("fail", [1, 2])
def test_injected_allocation_failure_in_build_and_render(fail, tmp_path):
    """The first (arena) or second (scratch) device allocation of a build fails: the build
    returns CAV_ERR_OUT_OF_MEMORY and frees what it took; so does a render whose path state
    cannot be allocated.  The next calls succeed with exact results."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes
    from oracle import pyoracle as po

    ctx = cav.Context(0)
    try:
        pos, idx = _soup(5000, seed=36)
        ctx.inject(cav.INJECT_ALLOC_FAIL, fail)
        with pytest.raises(cav.CavError) as e:
            ctx.build(_gpu(pos), _gpu(idx), rounds=1)
        assert e.value.status == CAV_ERR_OUT_OF_MEMORY
        ctx.inject(cav.INJECT_NONE)
        bvh = ctx.build(_gpu(pos), _gpu(idx), rounds=1)
        ctx.sync_check()
        mu, ms, _ = bvh.export_stages()
        assert np.array_equal(ms, po.build(pos, idx, codes=mu, rounds=1)["sorted"])
        bvh.free()
        path = str(tmp_path / "room.pbrt")
        scenes.write_pbrt(path, scenes.mini_room(), width=32, height=24, spp=2, max_depth=3)
        sc = ctx.load_pbrt(path, bvh_rounds=0)
        s0, w0, _ = sc.render()
        ctx.inject(cav.INJECT_ALLOC_FAIL, 1)
        with pytest.raises(cav.CavError) as e:
            sc.render()
        assert e.value.status == CAV_ERR_OUT_OF_MEMORY
        s1, w1, _ = sc.render()
        assert np.array_equal(w0, w1) and np.allclose(s0, s1, rtol=2e-5, atol=1e-6)
        sc.free()
    finally:
        ctx.close()


def test_mlp_completion_wait_runs_out_and_reports():
    """CAV_INJECT_MLP_STALL: every warpgroup of the tcgen05 forward issues no MMA and no
    commit for its first tile, so its completion wait (bounded at 50 ms here) runs out.  The
    forward returns, cav_sync_check reports CAV_ERR_TIMEOUT, and with the injection cleared
    the same network's outputs equal the mma.sync kernel's within their usual agreement."""
    import torch

    import cavalry_b200 as cav

    ctx = cav.Context(0)
    try:
        net = cav.Mlp(ctx, seed=3, kernel=cav.MLP_KERNEL_TCGEN05)
        ref = cav.Mlp(ctx, seed=3, kernel=cav.MLP_KERNEL_MMA_SYNC)
        x = torch.rand((20000, 5), device="cuda", generator=torch.Generator("cuda").manual_seed(4))
        want = ref.forward(x).cpu().numpy()
        ctx.set_limits(sort_wait_s=0.05)
        ctx.inject(cav.INJECT_MLP_STALL, 1)
        net.forward(x)
        with pytest.raises(cav.CavError) as e:
            ctx.sync_check()
        assert e.value.status == CAV_ERR_TIMEOUT
        ctx.inject(cav.INJECT_NONE)
        ctx.set_limits()
        got = net.forward(x).cpu().numpy()
        ctx.sync_check()
        scale = np.abs(want).mean()
        assert np.abs(got - want).max() <= 5e-3 * scale
        net.free()
        ref.free()
    finally:
        ctx.close()
