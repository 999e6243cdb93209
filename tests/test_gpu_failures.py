"""GPU tests of the failure paths: each is made to happen on the host side or by input that
the kernels' own checks turn into an error status (no fault, trap or hang is provoked).

* A vertex index outside [0, num_vertices) is flagged by the build's leaf-box pass (no load
  leaves the position array) and reported as CAV_ERR_INVALID_ARGUMENT by cav_sync_check;
  the context stays usable and the next build of valid input is exact.
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
