"""GPU tests of the serving loop (serve.cu): each job's result is the same through the
server as through the direct entry points, alone and in a mix of concurrent jobs, in the
merged (continuous batching) and sequential modes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import cavalry_b200 as cav

    return cav.Context(0)


@pytest.fixture(scope="module")
def pool(ctx, tmp_path_factory):
    from cavalry_b200 import scenes

    d = tmp_path_factory.mktemp("serve")
    out = {}
    for k, (n, res) in enumerate([(2000, 48), (30000, 64), (120000, 32)]):
        p = str(d / f"s{k}.pbrt")
        scenes.write_pbrt(p, scenes.soup_scene(n, seed=50 + k), width=res, height=res, spp=2, max_depth=4)
        out[k] = ctx.load_pbrt(p, bvh_rounds=2)
    return out


def direct_render(sc, spp):
    s, w, _ = sc.render(spp=spp, max_depth=4, integrator="path")
    return s, w


def test_ray_jobs_match_direct_queries(ctx, pool):
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    bvh = pool[1].bvh()
    rays = scenes.closest_rays(50000, seed=3)
    srays, lim = scenes.shadow_rays(40000, seed=4)
    prim, t, uv = bvh.trace_closest(torch.from_numpy(rays).cuda())
    occ = bvh.trace_any(torch.from_numpy(srays).cuda(), torch.from_numpy(lim).cuda())
    sv = cav.Server(ctx)
    j1, p1, t1, uv1 = sv.submit_rays(bvh, rays)
    j2, o2 = sv.submit_rays(bvh, srays, any_hit=True, limit=lim)
    assert sv.wait(j1, 60).state == cav.JOB_DONE and sv.wait(j2, 60).state == cav.JOB_DONE
    sv.close()
    assert np.array_equal(p1, prim.cpu().numpy())
    assert np.array_equal(t1.view(np.uint32), t.cpu().numpy().view(np.uint32))
    assert np.array_equal(o2, occ.cpu().numpy())


@pytest.mark.parametrize("mode", ["merged", "sequential"])
def test_mixed_jobs_same_as_alone(ctx, pool, mode):
    """Renders of three scenes and two ray-query jobs submitted together: every result
    equals the job run alone (films up to float atomic order).  One lane, so the merged
    server puts every live job in the same launches."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    alone = {k: direct_render(sc, 2) for k, sc in pool.items()}
    sv = cav.Server(ctx, mode=cav.SERVE_MERGED if mode == "merged" else cav.SERVE_SEQUENTIAL, lanes=1)
    subs = []
    for k, sc in pool.items():
        jid, fs, fw = sv.submit_render(sc, spp=2, max_depth=4)
        subs.append((jid, k, fs, fw))
    bvh = pool[2].bvh()
    rays = scenes.closest_rays(30000, seed=9)
    jr, pr, tr, _ = sv.submit_rays(bvh, rays)
    for jid, k, fs, fw in subs:
        st = sv.wait(jid, 120)
        assert st.state == cav.JOB_DONE and st.t_done >= st.t_start >= st.t_submit
        s, w = alone[k]
        assert np.array_equal(fw, w)
        assert np.allclose(fs, s, rtol=2e-5, atol=1e-6)
    sv.wait(jr, 60)
    stats = sv.stats()
    sv.close()
    import torch

    p, _, _ = bvh.trace_closest(torch.from_numpy(rays).cuda())
    assert np.array_equal(pr, p.cpu().numpy())
    if mode == "merged":
        # the five jobs shared traversal launches
        assert stats.max_segments >= 2
    else:
        assert stats.max_segments == 1


@pytest.mark.parametrize("lanes", [2, 3])
def test_lanes_many_jobs_same_as_alone(ctx, pool, lanes):
    """Several lanes (host threads with their own streams) serving a burst of renders and
    ray queries over the same resident scenes, in both traversal modes: every job finishes
    with the result it has alone."""
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    alone = {k: direct_render(sc, 2) for k, sc in pool.items()}
    rays = scenes.closest_rays(20000, seed=11)
    p_ref, _, _ = pool[0].bvh().trace_closest(torch.from_numpy(rays).cuda())
    p_ref = p_ref.cpu().numpy()
    for flags in (cav.TRACE_EXACT, cav.TRACE_FAST):
        sv = cav.Server(ctx, mode=cav.SERVE_MERGED, trace_flags=flags, lanes=lanes, max_paths_per_job=4096)
        subs, rq = [], []
        for rep in range(4):
            for k, sc in pool.items():
                subs.append((k, *sv.submit_render(sc, spp=2, max_depth=4)))
            rq.append(sv.submit_rays(pool[0].bvh(), rays))
        for k, jid, fs, fw in subs:
            assert sv.wait(jid, 120).state == cav.JOB_DONE
            s, w = alone[k]
            assert np.array_equal(fw, w)
            if flags == cav.TRACE_EXACT:
                assert np.allclose(fs, s, rtol=2e-5, atol=1e-6)
            else:
                assert np.abs(fs - s).mean() <= 1e-3 * np.abs(s).mean() + 1e-6
        for jid, pr, _, _ in rq:
            assert sv.wait(jid, 60).state == cav.JOB_DONE
            if flags == cav.TRACE_EXACT:
                assert np.array_equal(pr, p_ref)
            else:
                assert np.array_equal(pr >= 0, p_ref >= 0)
        st = sv.stats()
        assert st.live == 0 and st.pending == 0 and st.hbm_in_use == 0
        sv.close()


def test_small_hbm_budget_still_completes(ctx, pool):
    """Jobs larger than the budget run one at a time instead of waiting forever."""
    import cavalry_b200 as cav

    sv = cav.Server(ctx, hbm_budget_bytes=1 << 20)
    ids = [sv.submit_render(sc, spp=1, max_depth=2)[0] for sc in pool.values()]
    for jid in ids:
        assert sv.wait(jid, 120).state == cav.JOB_DONE
    assert sv.stats().max_segments == 1
    sv.close()


def test_server_close_with_pending_jobs(ctx, pool):
    import cavalry_b200 as cav

    sv = cav.Server(ctx, max_live_jobs=1)
    ids = [sv.submit_render(pool[1], spp=4, max_depth=4)[0] for _ in range(4)]
    sv.wait(ids[0], 120)
    sv.close()  # finishes the live job, fails the never-started ones


def test_fast_trace_server_matches_exact(ctx, pool):
    """The server's merged launches in the compressed 8-wide mode: ray queries hit the same
    distances as direct exact queries and renders agree with the exact renders (a closest
    hit changes only at an equal-distance tie)."""
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    sv = cav.Server(ctx, mode=cav.SERVE_MERGED, trace_flags=cav.TRACE_FAST, lanes=1)
    subs = [(k, *sv.submit_render(sc, spp=2, max_depth=4)) for k, sc in pool.items()]
    bvh = pool[2].bvh()
    rays = scenes.closest_rays(30000, seed=9)
    jr, pr, tr, _ = sv.submit_rays(bvh, rays)
    for k, jid, fs, fw in subs:
        assert sv.wait(jid, 120).state == cav.JOB_DONE
        s, w = direct_render(pool[k], 2)
        assert np.array_equal(fw, w)
        assert np.abs(fs - s).mean() <= 1e-3 * np.abs(s).mean() + 1e-6
    assert sv.wait(jr, 60).state == cav.JOB_DONE
    assert sv.stats().max_segments >= 2
    sv.close()
    assert pool[2].bvh().has_fast_layout()  # the server built the 8-wide view it traced
    p, t, _ = bvh.trace_closest(torch.from_numpy(rays).cuda())
    p, t = p.cpu().numpy(), t.cpu().numpy()
    assert np.array_equal(pr >= 0, p >= 0)
    both = p >= 0
    assert np.all(np.abs(tr[both] - t[both]) <= 1e-6 * np.abs(t[both]))


def _wait_running(sv, jid, timeout=60.0):
    import time

    import cavalry_b200 as cav

    t0 = time.time()
    while sv.poll(jid).state == cav.JOB_PENDING:
        assert time.time() - t0 < timeout
        time.sleep(0.001)


def test_cancel_pending_and_running_jobs(ctx, pool):
    """A job cancelled while pending leaves the queue at once; a job cancelled while running
    stops before its next bounce and frees its state; the job between them finishes with the
    result it has alone, and the server ends with nothing live and no memory in use."""
    import cavalry_b200 as cav

    sv = cav.Server(ctx, max_live_jobs=1, max_paths_per_job=4096)
    long_id, _, _ = sv.submit_render(pool[1], spp=256, max_depth=4, width=64, height=64)  # 256 chunks x 4 bounces
    mid_id, fs, fw = sv.submit_render(pool[0], spp=2, max_depth=4)
    late_id, _, _ = sv.submit_render(pool[2], spp=2, max_depth=4)
    sv.cancel(late_id)
    st = sv.poll(late_id)
    assert st.state == cav.JOB_CANCELLED and st.status == 7
    _wait_running(sv, long_id)
    sv.cancel(long_id)
    assert sv.wait(long_id, 120).state == cav.JOB_CANCELLED
    assert sv.wait(mid_id, 120).state == cav.JOB_DONE
    s, w = direct_render(pool[0], 2)
    assert np.array_equal(fw, w) and np.allclose(fs, s, rtol=2e-5, atol=1e-6)
    sv.cancel(mid_id)  # finished: unchanged
    assert sv.poll(mid_id).state == cav.JOB_DONE
    st = sv.stats()
    assert st.live == 0 and st.pending == 0 and st.hbm_in_use == 0
    sv.close()


def test_admission_rejects_jobs_over_the_budget(ctx, pool):
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    sv = cav.Server(ctx, hbm_budget_bytes=1 << 20, reject_over_budget=True)
    with pytest.raises(cav.CavError) as e:
        sv.submit_render(pool[1], spp=2, max_depth=4)
    assert e.value.status == 3  # CAV_ERR_OUT_OF_MEMORY, and no job was created
    rays = scenes.closest_rays(1000, seed=12)  # ~50 KB: admitted
    jid, p, _, _ = sv.submit_rays(pool[1].bvh(), rays)
    assert sv.wait(jid, 60).state == cav.JOB_DONE and (p >= -1).all()
    sv.close()


def test_injected_allocation_failure_fails_only_that_job(ctx, pool):
    """While a long render runs, the next device allocation is made to fail: the job that
    makes it (a render submitted then) fails with CAV_ERR_OUT_OF_MEMORY, the running job and
    a job submitted afterwards finish with the results they have alone."""
    import cavalry_b200 as cav

    sv = cav.Server(ctx, max_paths_per_job=4096)
    long_id, fs_l, fw_l = sv.submit_render(pool[1], spp=16, max_depth=4, width=64, height=64)
    _wait_running(sv, long_id)
    ctx.inject(cav.INJECT_ALLOC_FAIL, 1)
    bad_id, _, _ = sv.submit_render(pool[0], spp=2, max_depth=4)
    with pytest.raises(cav.CavError) as e:
        sv.wait(bad_id, 120)
    assert e.value.status == 3 and sv.poll(bad_id).state == cav.JOB_FAILED
    ctx.inject(cav.INJECT_NONE)
    ok_id, fs, fw = sv.submit_render(pool[0], spp=2, max_depth=4)
    assert sv.wait(ok_id, 120).state == cav.JOB_DONE
    assert sv.wait(long_id, 120).state == cav.JOB_DONE
    s, w = direct_render(pool[0], 2)
    assert np.array_equal(fw, w) and np.allclose(fs, s, rtol=2e-5, atol=1e-6)
    s, w, _ = pool[1].render(spp=16, max_depth=4, width=64, height=64, integrator="path",
                             max_paths_in_flight=4096)
    assert np.array_equal(fw_l, w) and np.allclose(fs_l, s, rtol=2e-5, atol=1e-6)
    sv.close()


@pytest.mark.parametrize("flags", ["exact", "fast"])
def test_scene_jobs_same_as_load_and_render(ctx, tmp_path, flags):
    """Jobs that bring their own scene file: a small render (replayed as one CUDA graph), a
    larger render (merged ticks), a closest-hit and an any-hit ray job, submitted together.
    The server parses the files on its loader threads, builds the trees of the scenes admitted
    together in one batched build, runs the jobs and frees the scenes; every result equals
    loading the same file (cav_scene_load_pbrt) and rendering or tracing it alone."""
    import torch

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    tf = cav.TRACE_FAST if flags == "fast" else cav.TRACE_EXACT
    paths = []
    for k, n in enumerate([2000, 30000, 8000, 60000]):
        p = str(tmp_path / f"job{k}.pbrt")
        scenes.write_pbrt(p, scenes.soup_scene(n, seed=70 + k), width=32, height=32, spp=2, max_depth=4)
        paths.append(p)
    rays = scenes.closest_rays(20000, seed=13)
    srays, lim = scenes.shadow_rays(20000, seed=14)
    sv = cav.Server(ctx, trace_flags=tf, graph_max_paths=64 * 64 * 2, lanes=1)
    j0, fs0, fw0 = sv.submit_scene_render(paths[0], 64, 64, spp=2, max_depth=4)
    j1, fs1, fw1 = sv.submit_scene_render(paths[1], 96, 96, spp=4, max_depth=4)
    j2, p2, t2, _ = sv.submit_scene_rays(paths[2], rays)
    j3, o3 = sv.submit_scene_rays(paths[3], srays, any_hit=True, limit=lim)
    jbad, _, _ = sv.submit_scene_render(str(tmp_path / "missing.pbrt"), 16, 16)
    for j in (j0, j1, j2, j3):
        assert sv.wait(j, 120).state == cav.JOB_DONE
    with pytest.raises(cav.CavError) as e:
        sv.wait(jbad, 60)
    assert e.value.status == 1 and sv.poll(jbad).state == cav.JOB_FAILED
    st = sv.stats()
    assert st.live == 0 and st.pending == 0 and st.hbm_in_use == 0
    sv.close()
    fast = flags == "fast"
    for p, (w_, h_, spp), fs, fw in ((paths[0], (64, 64, 2), fs0, fw0), (paths[1], (96, 96, 4), fs1, fw1)):
        sc = ctx.load_pbrt(p)
        s, w, _ = sc.render(spp=spp, max_depth=4, width=w_, height=h_, integrator="path", fast_trace=fast)
        sc.free()
        assert np.array_equal(fw, w)
        if fast:
            assert np.abs(fs - s).mean() <= 1e-3 * np.abs(s).mean() + 1e-6
        else:
            assert np.allclose(fs, s, rtol=2e-5, atol=1e-6)
    sc = ctx.load_pbrt(paths[2])
    p, t, _ = sc.bvh().trace_closest(torch.from_numpy(rays).cuda(), flags=tf)
    assert np.array_equal(p2, p.cpu().numpy()) and np.array_equal(t2.view(np.uint32), t.cpu().numpy().view(np.uint32))
    sc.free()
    sc = ctx.load_pbrt(paths[3])
    o = sc.bvh().trace_any(torch.from_numpy(srays).cuda(), torch.from_numpy(lim).cuda(), flags=tf)
    assert np.array_equal(o3, o.cpu().numpy())
    sc.free()


def test_scene_job_cancelled_before_it_runs(ctx, tmp_path):
    """A scene job cancelled while it waits to be parsed or admitted never runs; the others do."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    p = str(tmp_path / "s.pbrt")
    scenes.write_pbrt(p, scenes.soup_scene(20000, seed=80), width=32, height=32, spp=1, max_depth=3)
    sv = cav.Server(ctx, max_live_jobs=1, loaders=1)
    ids = [sv.submit_scene_render(p, 32, 32)[0] for _ in range(6)]
    sv.cancel(ids[-1])
    assert sv.wait(ids[-1], 60).state == cav.JOB_CANCELLED
    for j in ids[:-1]:
        assert sv.wait(j, 120).state == cav.JOB_DONE
    assert sv.stats().hbm_in_use == 0
    sv.close()
