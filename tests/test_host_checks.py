"""CPU tests of the Python layer's buffer checks in front of the traversal entry points: the
kernels read and write through raw pointers, so a tensor of the wrong type, device or size
must be refused before the call rather than overrun on the GPU.  Stand-in tensors carry the
attributes the checks read (no GPU is needed), and a stand-in library records the calls."""
import numpy as np
import pytest
import torch

import cavalry_b200 as cav


class FakeCuda:
    """The attributes of a CUDA tensor that the checks and the pointer lookup read."""

    def __init__(self, shape, dtype, device=0, contiguous=True):
        self.shape = tuple(shape)
        self.dtype = dtype
        self.device = torch.device("cuda", device)
        self.is_cuda = True
        self._contiguous = contiguous

    def is_contiguous(self):
        return self._contiguous

    def numel(self):
        return int(np.prod(self.shape))

    def data_ptr(self):
        return 4096


class FakeLib:
    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        def call(*args):
            self.calls.append(name)
            return 0

        return call


class FakeCtx:
    device = 0
    handle = 1

    def _check(self, st, what):
        assert st == 0


@pytest.fixture
def bvh(monkeypatch):
    fake = FakeLib()
    monkeypatch.setattr(cav, "lib", lambda: fake)
    monkeypatch.setattr(cav, "_stream_ptr", lambda stream: None)
    b = cav.Bvh(FakeCtx(), 2, 10, owned=False)
    b.fake = fake
    return b


def out3(n, **kw):
    return (FakeCuda((n,), torch.int32, **kw), FakeCuda((n,), torch.float32), FakeCuda((n, 2), torch.float32))


def test_valid_buffers_reach_the_library(bvh):
    n = 100
    rays = FakeCuda((n, 8), torch.float32)
    bvh.trace_closest(rays, out=out3(n))
    bvh.trace_closest(rays, out=(FakeCuda((n,), torch.int32), None, None))
    bvh.trace_any(rays, FakeCuda((n,), torch.float32), FakeCuda((n, 2), torch.int32), out=FakeCuda((n,), torch.uint8))
    bvh.trace_any(rays, None, None, out=FakeCuda((2 * n,), torch.uint8))  # larger outputs are fine
    bvh.autotune(rays, any_hit=True, limit=FakeCuda((n,), torch.float32))
    assert bvh.fake.calls == ["cav_trace_closest", "cav_trace_closest", "cav_trace_any", "cav_trace_any",
                              "cav_trace_autotune_flags"]


@pytest.mark.parametrize("bad,msg", [
    (lambda n: (FakeCuda((n - 1,), torch.int32),) + out3(n)[1:], "at least 100"),
    (lambda n: (FakeCuda((n,), torch.int64),) + out3(n)[1:], "dtype"),
    (lambda n: (out3(n)[0], FakeCuda((n,), torch.float32, device=1), out3(n)[2]), "cuda:1"),
    (lambda n: (out3(n)[0], out3(n)[1], FakeCuda((n,), torch.float32)), "at least 200"),
    (lambda n: (out3(n)[0], out3(n)[1], FakeCuda((n, 2), torch.float32, contiguous=False)), "contiguous"),
    (lambda n: (torch.zeros(n, dtype=torch.int32),) + out3(n)[1:], "CUDA tensor"),
])
def test_bad_closest_hit_outputs_are_refused(bvh, bad, msg):
    n = 100
    with pytest.raises(ValueError, match=msg):
        bvh.trace_closest(FakeCuda((n, 8), torch.float32), out=bad(n))
    assert bvh.fake.calls == []


@pytest.mark.parametrize("kw,msg", [
    ({"limit": FakeCuda((99,), torch.float32)}, "limit"),
    ({"limit": FakeCuda((100,), torch.float64)}, "limit"),
    ({"excl": FakeCuda((100,), torch.int32)}, "excl"),
    ({"excl": FakeCuda((100, 2), torch.int64)}, "excl"),
    ({"out": FakeCuda((99,), torch.uint8)}, "out"),
    ({"out": FakeCuda((100,), torch.bool)}, "out"),
])
def test_bad_any_hit_buffers_are_refused(bvh, kw, msg):
    with pytest.raises(ValueError, match=msg):
        bvh.trace_any(FakeCuda((100, 8), torch.float32), **kw)
    assert bvh.fake.calls == []


def test_rays_on_another_gpu_are_refused(bvh):
    with pytest.raises(ValueError, match="cuda:3"):
        bvh.autotune(FakeCuda((64, 8), torch.float32, device=3))
    assert bvh.fake.calls == []


def test_host_buffer_variants_check_their_arrays(bvh):
    n = 50
    rays = np.zeros((n, 8), np.float32)
    bvh.trace_closest_host(rays)
    bvh.trace_closest_host(torch.zeros((n, 8)), out=(torch.zeros(n, dtype=torch.int32), None, None))
    bvh.trace_any_host(rays, np.ones(n, np.float32), np.zeros((n, 2), np.int32))
    assert bvh.fake.calls == ["cav_trace_closest_host"] * 2 + ["cav_trace_any_host"]
    bad = [
        lambda: bvh.trace_closest_host(rays.astype(np.float64)),
        lambda: bvh.trace_closest_host(np.asfortranarray(np.zeros((n, 8), np.float32))),
        lambda: bvh.trace_closest_host(rays, out=(np.zeros(n - 1, np.int32), None, None)),
        lambda: bvh.trace_closest_host(rays, out=(np.zeros(n, np.int32), None, np.zeros((n, 1), np.float32))),
        lambda: bvh.trace_closest_host(FakeCuda((n, 8), torch.float32)),
        lambda: bvh.trace_any_host(rays, np.ones(n, np.float64)),
        lambda: bvh.trace_any_host(rays, None, np.zeros((n, 2), np.int64)),
        lambda: bvh.trace_any_host(rays, out=np.zeros(n - 1, np.uint8)),
    ]
    for call in bad:
        with pytest.raises(ValueError):
            call()
    assert len(bvh.fake.calls) == 3


def test_build_checks_devices_and_mesh_ids(monkeypatch):
    fake = FakeLib()
    monkeypatch.setattr(cav, "lib", lambda: fake)
    monkeypatch.setattr(cav, "_stream_ptr", lambda stream: None)
    ctx = object.__new__(cav.Context)
    ctx.device, ctx.handle = 0, None
    monkeypatch.setattr(ctx, "_check", lambda st, what: None, raising=False)
    pos, idx = FakeCuda((10, 3), torch.float32), FakeCuda((4, 3), torch.int32)
    ctx.build(pos, idx, mesh_ids=FakeCuda((4,), torch.int32))
    assert fake.calls == ["cav_bvh_build"]
    with pytest.raises(ValueError, match="mesh_ids"):
        ctx.build(pos, idx, mesh_ids=FakeCuda((3,), torch.int32))
    with pytest.raises(ValueError, match="cuda:1"):
        ctx.build(FakeCuda((10, 3), torch.float32, device=1), idx)
    # the triangle and vertex counts stay the library's to check (it returns its own status)
    ctx.build(FakeCuda((3, 3), torch.float32), FakeCuda((1, 3), torch.int32))
    assert fake.calls == ["cav_bvh_build"] * 2


def test_server_ray_jobs_check_shapes(monkeypatch):
    fake = FakeLib()
    monkeypatch.setattr(cav, "lib", lambda: fake)
    sv = object.__new__(cav.Server)
    sv.handle, sv.ctx, sv._keep = 1, FakeCtx(), {}
    try:
        bvh = cav.Bvh(FakeCtx(), 2, 10, owned=False)
        rays = np.zeros((20, 8), np.float32)
        sv.submit_rays(bvh, rays, any_hit=True, limit=np.ones(20))
        sv.submit_scene_rays("x.pbrt", rays)
        assert fake.calls == ["cav_server_submit_rays", "cav_server_submit_scene"]
        for call in (lambda: sv.submit_rays(bvh, np.zeros((20, 6), np.float32)),
                     lambda: sv.submit_rays(bvh, rays, any_hit=True, limit=np.ones(19)),
                     lambda: sv.submit_scene_rays("x.pbrt", rays, any_hit=True, excl=np.zeros((20, 1), np.int32))):
            with pytest.raises(ValueError):
                call()
        assert len(fake.calls) == 2
    finally:
        sv.handle = None  # the stand-in handle must never reach the real library's destroy
