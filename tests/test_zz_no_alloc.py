"""GPU test of cav_morton_sort_noalloc, the allocation-free Morton + sort entry point.

It serves callers that cannot call cudaMalloc (a renderer embedded in a host application
that owns all device memory through a pool fixed at start-up, or a per-frame loop that must
not block on or fail an allocation).  The entry point is called through the C ABI twice in
a row, on different meshes, and each result must equal, bit for bit, the sorted codes and
order that the allocating build (cav_bvh_build + cav_bvh_export_stages) produces for the same
input.  The second call is smaller than the first, so leftovers of the first call in the
shared static scratch array would show.  This file is collected last so that a run stopping
at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CAV_NOALLOC_MAX_TRIANGLES = 131072


def _bind():
    import cavalry_b200 as cav

    L = cav.lib()
    f = L.cav_morton_sort_noalloc
    P = ctypes.c_void_p
    f.argtypes = [P, ctypes.c_int64, P, ctypes.c_int64, P, P, P, P]
    f.restype = ctypes.c_int
    return f


def _noalloc(f, d_pos, d_idx, n, bounds=None):
    import torch

    codes = torch.empty(n, dtype=torch.int64, device="cuda")
    prims = torch.empty(n, dtype=torch.int32, device="cuda")
    b = None if bounds is None else np.ascontiguousarray(bounds, np.float32)
    st = f(d_pos.data_ptr(), d_pos.numel() // 3, d_idx.data_ptr(), n, None if b is None else b.ctypes.data,
           codes.data_ptr(), prims.data_ptr(), torch.cuda.current_stream().cuda_stream or None)
    return st, codes.cpu().numpy().view(np.uint64), prims.cpu().numpy()


def test_noalloc_matches_allocating_build_on_two_calls_in_a_row():
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    f = _bind()
    ctx = cav.Context(0)
    for seed, n in ((61, CAV_NOALLOC_MAX_TRIANGLES), (62, 5000)):
        pos, idx = scenes.soup(n, seed=seed)
        d_pos = torch.from_numpy(pos).cuda()
        d_idx = torch.from_numpy(idx).cuda()
        st, codes, prims = _noalloc(f, d_pos, d_idx, n)
        assert st == 0, cav.lib().cav_status_string(st)
        bvh = ctx.build(d_pos, d_idx, rounds=0)
        _, want_codes, want_prims = bvh.export_stages()
        assert np.array_equal(codes, want_codes), f"n={n}: sorted codes differ"
        assert np.array_equal(prims, want_prims), f"n={n}: sorted order differs"
        bvh.free()
    ctx.close()


def test_noalloc_host_bounds_and_size_limit():
    import torch

    from cavalry_b200 import scenes

    f = _bind()
    pos, idx = scenes.soup(3000, seed=63)
    d_pos = torch.from_numpy(pos).cuda()
    d_idx = torch.from_numpy(idx).cuda()
    lo = pos.min(0)
    hi = pos.max(0)
    st_dev, c_dev, p_dev = _noalloc(f, d_pos, d_idx, 3000)
    st_host, c_host, p_host = _noalloc(f, d_pos, d_idx, 3000, bounds=np.concatenate([lo, hi]))
    assert st_dev == 0 and st_host == 0
    assert np.array_equal(c_dev, c_host) and np.array_equal(p_dev, p_host)
    big = CAV_NOALLOC_MAX_TRIANGLES + 1
    pos_b, idx_b = scenes.soup(big, seed=64)
    st, _, _ = _noalloc(f, torch.from_numpy(pos_b).cuda(), torch.from_numpy(idx_b).cuda(), big)
    assert st == 1  # CAV_ERR_INVALID_ARGUMENT: above the static scratch's maximum


def test_noalloc_rejects_an_out_of_range_vertex_index():
    """A vertex index outside [0, num_vertices) is reported as CAV_ERR_INVALID_ARGUMENT (the
    kernel reads no position outside the array); the next call on valid input is exact."""
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    f = _bind()
    pos, idx = scenes.soup(2000, seed=65)
    bad = idx.copy()
    bad[100, 0] = pos.shape[0]
    d_pos = torch.from_numpy(pos).cuda()
    st, _, _ = _noalloc(f, d_pos, torch.from_numpy(bad).cuda(), 2000)
    assert st == 1
    d_idx = torch.from_numpy(idx).cuda()
    st, codes, prims = _noalloc(f, d_pos, d_idx, 2000)
    assert st == 0
    ctx = cav.Context(0)
    bvh = ctx.build(d_pos, d_idx, rounds=0)
    _, want_codes, want_prims = bvh.export_stages()
    assert np.array_equal(codes, want_codes) and np.array_equal(prims, want_prims)
    bvh.free()
    ctx.close()
