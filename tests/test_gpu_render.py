"""GPU parity tests of the render path (the reference's PathTracingIntegrator behind
Integrator::render and the CLI), through the C ABI.

* Against the reference renderer's own PNGs (tests/golden/render_ref.npz, made by
  tests/golden/make_render_golden.py on a B200 from the same seeded .pbrt scenes).
* Against the path-tracing oracle's float film (oracle/pt_oracle.c).
* Invariances: chunking of paths in flight, device-film entry on a side stream, the CLI.
"""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden" / "render_ref.npz"
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def render_cases():
    if not GOLDEN.exists():
        return []
    return json.loads(str(np.load(GOLDEN)["meta"]))


def make_scene(gen):
    import make_render_golden

    return make_render_golden.make_scene(gen)


@pytest.fixture(scope="module")
def ctx():
    import cavalry_b200 as cav

    return cav.Context(0)


def load(ctx, tmp_path, name, scene, render, rounds=0):
    from cavalry_b200 import scenes

    path = str(tmp_path / f"{name}.pbrt")
    scenes.write_pbrt(path, scene, **render)
    return ctx.load_pbrt(path, bvh_rounds=rounds), path


# Device maths is the reference's (fast-math, same expression shapes), so the room agrees
# to the 8-bit value almost everywhere; glass chains keep a few flipped lobe choices.
TOL = {"room": dict(exact=0.999, le2=0.9998, gt8=0.0002),
       "spheres": dict(exact=0.96, le2=0.99, gt8=0.003),
       "shapes": dict(exact=0.96, le2=0.99, gt8=0.003),
       "courtyard": dict(exact=0.96, le2=0.99, gt8=0.003),
       # rlpath learns its table with float atomics in both renderers, so the order of
       # proposals (and with it a few samples) differs from run to run
       "rlpath": dict(exact=0.95, le2=0.99, gt8=0.005)}


def tol_of(case):
    t = TOL["rlpath"] if case["render"].get("integrator") == "rlpath" else TOL[case["gen"]["kind"]]
    if case["gen"].get("hdr_sky"):
        # an HDR sun 6x brighter than the 8-bit sky: one flipped path choice that reaches it
        # moves its pixel far, so more pixels differ by more than 8 (the oracle shows it too)
        t = dict(t, gt8=0.005)
    return t


@pytest.mark.parametrize("case", render_cases(), ids=[c["name"] for c in render_cases()])
def test_render_matches_reference_png(ctx, tmp_path, case):
    import cavalry_b200 as cav

    sc, _ = load(ctx, tmp_path, case["name"], make_scene(case["gen"]), case["render"])
    s, w, ms = sc.render()
    img = cav.film_to_rgb8(s, w)
    ref = np.load(GOLDEN)[case["name"]]
    d = np.abs(img.astype(int) - ref.astype(int)).max(2)
    t = tol_of(case)
    assert (d == 0).mean() >= t["exact"], (d == 0).mean()
    assert (d <= 2).mean() >= t["le2"], (d <= 2).mean()
    assert (d > 8).mean() <= t["gt8"], (d > 8).mean()
    # films hold whole samples: weight = number of splats per pixel
    assert np.all(w >= case["render"]["spp"])


@pytest.mark.parametrize("name", ["room_d5_s16", "spheres_mixed", "spheres_glass", "spheres_roughglass"])
def test_fast_trace_render_matches_reference_png(ctx, tmp_path, name):
    """The compressed 8-wide traversal changes a closest hit only at an equal-distance tie, so
    its renders meet the same 8-bit agreement with the reference's PNGs."""
    import cavalry_b200 as cav

    case = next(c for c in render_cases() if c["name"] == name)
    sc, _ = load(ctx, tmp_path, name, make_scene(case["gen"]), case["render"])
    s, w, _ = sc.render(fast_trace=True)
    img = cav.film_to_rgb8(s, w)
    d = np.abs(img.astype(int) - np.load(GOLDEN)[name].astype(int)).max(2)
    t = tol_of(case)
    assert (d == 0).mean() >= t["exact"], (d == 0).mean()
    assert (d <= 2).mean() >= t["le2"], (d <= 2).mean()
    assert (d > 8).mean() <= t["gt8"], (d > 8).mean()


@pytest.mark.parametrize("name", ["room_d5_s16", "spheres_mixed"])
def test_render_film_matches_oracle(ctx, tmp_path, name):
    """Float films against the CPU restatement: weights identical (same jitter), radiance
    within 1e-3 relative on all but a few pixels, image means within 2e-3."""
    from oracle import pyoracle as po

    case = next(c for c in render_cases() if c["name"] == name)
    scene = make_scene(case["gen"])
    sc, _ = load(ctx, tmp_path, name, scene, case["render"])
    s, w, _ = sc.render()
    os_, ow = po.render_path(scene, **case["render"])
    assert np.array_equal(w, ow)
    rel = np.abs(s - os_) / (np.abs(os_) + 1e-2)
    assert (rel > 1e-3).mean() <= 0.01, (rel > 1e-3).mean()
    assert abs(s.mean() - os_.mean()) <= 2e-3 * abs(os_.mean())


def test_render_chunking_and_device_film(ctx, tmp_path):
    """Paths in flight split into small chunks, rendered into device films on a side
    stream, give the host-film render (up to float atomic order)."""
    import torch

    from cavalry_b200 import scenes

    sc, _ = load(ctx, tmp_path, "chunk", scenes.mini_room(), dict(width=96, height=64, spp=8, max_depth=5))
    s, w, _ = sc.render()
    fs = torch.zeros(64 * 96 * 3, device="cuda")
    fw = torch.zeros(64 * 96, device="cuda")
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        sc.render_into(fs, fw, max_paths_in_flight=5000, stream=st)
    st.synchronize()
    assert np.array_equal(fw.cpu().numpy().reshape(64, 96), w)
    assert np.allclose(fs.cpu().numpy().reshape(64, 96, 3), s, rtol=2e-5, atol=1e-5)


def test_render_spp_and_depth_options(ctx, tmp_path):
    """Render options override the file's Sampler/Integrator values (--spp / maxdepth)."""
    from cavalry_b200 import scenes

    sc, _ = load(ctx, tmp_path, "opts", scenes.mini_room(), dict(width=32, height=32, spp=1, max_depth=1))
    ref, _ = load(ctx, tmp_path, "opts4", scenes.mini_room(), dict(width=32, height=32, spp=4, max_depth=3))
    s4, w4, _ = sc.render(spp=4, max_depth=3)
    r4, rw4, _ = ref.render()
    assert np.array_equal(w4, rw4)
    assert np.allclose(s4, r4, rtol=1e-5, atol=1e-6)
    s_d1, _, _ = sc.render(spp=4, max_depth=1)
    s_d3, _, _ = sc.render(spp=4, max_depth=3)
    assert s_d3.sum() > s_d1.sum()


def test_render_treelet_rounds_do_not_change_the_image(ctx, tmp_path):
    """Treelet restructuring changes the tree, not the hits: the images agree up to ties."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    render = dict(width=128, height=96, spp=4, max_depth=6)
    scene = scenes.sphere_scene(12, 3, seed=11)
    a, _ = load(ctx, tmp_path, "r0", scene, render, rounds=0)
    b, _ = load(ctx, tmp_path, "r3", scene, render, rounds=3)
    ia = cav.film_to_rgb8(*a.render()[:2])
    ib = cav.film_to_rgb8(*b.render()[:2])
    d = np.abs(ia.astype(int) - ib.astype(int)).max(2)
    assert (d == 0).mean() >= 0.999
    assert b.info().bvh_rounds == 3


def test_cli_renders_png(tmp_path):
    """The `cavalry` CLI (main.cu:25-96 surface) writes the PNG the library renders."""
    import cavalry_b200 as cav
    from cavalry_b200 import build_ext, scenes
    from oracle import ref_cli

    cli = build_ext.CLI
    assert cli.exists(), "cavalry CLI not built"
    path = str(tmp_path / "room.pbrt")
    scenes.write_pbrt(path, scenes.mini_room(), width=64, height=64, spp=2, max_depth=3)
    out = tmp_path / "out.png"
    r = subprocess.run([str(cli), "--input", path, "--output", str(out), "--spp", "4", "--bvh-opt-rounds", "0"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Rendering took" in r.stdout
    png = ref_cli.read_png(out)
    sc = cav.Context(0).load_pbrt(path, spp=4, bvh_rounds=0)
    img = cav.film_to_rgb8(*sc.render()[:2])
    d = np.abs(png.astype(int) - img.astype(int)).max(2)  # float atomics may round differently
    assert d.max() <= 1 and (d == 0).mean() >= 0.999


def test_rlpath_converges_to_path(ctx, tmp_path):
    """The learned proposal keeps the estimator unbiased: at 64 spp the rlpath image agrees
    with a 1024-spp path render as closely as a 64-spp path render does."""
    from cavalry_b200 import scenes

    sc, _ = load(ctx, tmp_path, "conv", scenes.sphere_scene(12, 3, seed=5), dict(width=96, height=64, spp=16,
                                                                                   max_depth=8))
    s, w, _ = sc.render(spp=1024, integrator="path")
    ref = s / w[..., None]

    def relmse(x):
        return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))

    s, w, _ = sc.render(spp=64, integrator="path")
    e_path = relmse(s / w[..., None])
    s, w, _ = sc.render(spp=64, integrator="rlpath")
    e_rl = relmse(s / w[..., None])
    assert e_rl <= 1.5 * e_path, (e_rl, e_path)
    assert abs((s / w[..., None]).mean() - ref.mean()) <= 0.01 * ref.mean()


def test_resolution_override_matches_scene_film(ctx, tmp_path):
    """Render options' width/height give the image of a scene whose Film has that size."""
    from cavalry_b200 import scenes

    room = scenes.mini_room()
    small, _ = load(ctx, tmp_path, "res_a", room, dict(width=32, height=24, spp=2, max_depth=3))
    big, _ = load(ctx, tmp_path, "res_b", room, dict(width=80, height=60, spp=2, max_depth=3))
    s1, w1, _ = small.render(width=80, height=60)
    s2, w2, _ = big.render()
    assert s1.shape == (60, 80, 3)
    assert np.array_equal(w1, w2)
    assert np.allclose(s1, s2, rtol=2e-5, atol=1e-6)


@pytest.mark.parametrize("fast", [False, True])
@pytest.mark.parametrize("chunk", [0, 3000])
def test_graph_replayed_render_matches(ctx, tmp_path, chunk, fast):
    """The CUDA-graph render (queue sizes on the device, one graph per chunk) gives the
    stream-ordered render's film and ray counts, in both traversal modes."""
    from cavalry_b200 import scenes

    sc, _ = load(ctx, tmp_path, f"graph{chunk}{fast}", scenes.sphere_scene(8, 2, seed=5),
                 dict(width=64, height=48, spp=4, max_depth=6))
    s1, w1, _ = sc.render(max_paths_in_flight=chunk, fast_trace=fast)
    st1 = sc.stats()
    s2, w2, _ = sc.render(max_paths_in_flight=chunk, graph=True, fast_trace=fast)
    st2 = sc.stats()
    assert np.array_equal(w1, w2)
    assert np.allclose(s1, s2, rtol=2e-5, atol=1e-6)
    assert st2.closest_rays == st1.closest_rays and st2.shadow_rays == st1.shadow_rays


def test_sample_ranges_sum_to_the_whole_render(ctx, tmp_path):
    """Films of disjoint camera-sample ranges sum to the whole render's (the shard of a
    multi-GPU render); one NCCL process group of one rank runs the sharded path end to end."""
    import os
    import socket

    import torch
    import torch.distributed as dist

    from cavalry_b200 import distributed

    case = next(c for c in render_cases() if c["name"] == "spheres_mixed")
    sc, _ = load(ctx, tmp_path, "ranges", make_scene(case["gen"]), case["render"])
    s, w, _ = sc.render()
    info = sc.info()
    total = info.width * info.height * info.spp
    cut = total // 3 + 17
    s1, w1, _ = sc.render(sample_range=(0, cut))
    s2, w2, _ = sc.render(sample_range=(cut, total))
    assert np.array_equal(w1 + w2, w)
    assert np.allclose(s1 + s2, s, rtol=1e-5, atol=1e-5)
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        fs, fw = distributed.render_scene_sharded(sc)
        assert np.array_equal(fw.view(info.height, info.width).cpu().numpy(), w)
        assert np.allclose(fs.view(info.height, info.width, 3).cpu().numpy(), s, rtol=1e-5, atol=1e-5)
    finally:
        dist.destroy_process_group()
    with pytest.raises(Exception, match="sample ranges"):
        sc.render(integrator="rlpath", sample_range=(0, 10))
    ctx.sync_check()


CONFIG3 = Path(__file__).resolve().parent / "golden" / "render_spheres5m_sub4.npz"


@pytest.mark.skipif(not CONFIG3.exists(), reason="fixture made by tests/golden/make_config3_golden.py")
def test_full_size_scene_matches_reference_png(ctx, tmp_path):
    """The full-size path-traced scene (64 level-6 icospheres, 5.24M triangles, 1920 x 1080, 64
    spp, depth 8), compared with the reference renderer's PNG on every 4th row and column.
    This project's render uses its own 3-round tree (a closest hit changes only at an exact
    distance tie) in the exact traversal mode.  The tolerance is stated for this size: each
    pixel averages 64 sample paths of up to 8 bounces, and a discrete choice flipped by
    last-bit rounding in any of them (a glass lobe, a roulette draw) moves the pixel's 8-bit
    value, so fewer pixels are exactly equal than in the 8-16 spp goldens.  Measured on a
    B200: 88.7 % exact, 99.5 % within 2, 0.32 % over 8, mean signed difference +0.03 of 255;
    the same with the reference's own tree (0 rounds) and in the fast traversal mode, so the
    differences come from shading arithmetic, not from hits."""
    import json

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    g = np.load(CONFIG3)
    meta = json.loads(str(g["meta"]))
    path = str(tmp_path / "spheres5m.pbrt")
    scenes.write_pbrt(path, scenes.sphere_scene(**meta["scene"]), **meta["render"])
    sc = ctx.load_pbrt(path, bvh_rounds=3)
    s, w, _ = sc.render()
    sc.free()
    img = cav.film_to_rgb8(s, w)[:: meta["step"], :: meta["step"]]
    diff = img.astype(int) - g["sub"].astype(int)
    d = np.abs(diff).max(2)
    assert (d == 0).mean() >= 0.87, (d == 0).mean()
    assert (d <= 2).mean() >= 0.99, (d <= 2).mean()
    assert (d > 8).mean() <= 0.005, (d > 8).mean()
    assert abs(diff.mean()) <= 0.1, diff.mean()  # no bias: differences are rounding flips both ways
