"""CPU tests of the render path's checker and host code: the path-tracing oracle against
the reference renderer's own PNGs (tests/golden/render_ref.npz), and the host .pbrt parser
(the reference's SceneLoading/Lexing.cu and Parsing.cu surface)."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden" / "render_ref.npz"
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def render_cases():
    """Path and direct-lighting cases (the oracle restates those two integrators)."""
    if not GOLDEN.exists():
        return []
    g = np.load(GOLDEN)
    return [c for c in json.loads(str(g["meta"])) if c["render"].get("integrator", "path") in ("path", "directlighting")]


def make_scene(gen):
    import make_render_golden

    return make_render_golden.make_scene(gen)


# 8-bit agreement required of a film against the reference's PNG.  The room is diffuse and
# agrees almost everywhere; glass and mirror chains amplify rounding (approximate device
# maths vs IEEE host maths) into flipped lobe / roulette choices on a few percent of pixels.
TOL = {"room": dict(exact=0.999, le2=0.9995, max_frac_gt8=0.0005),
       "spheres": dict(exact=0.95, le2=0.985, max_frac_gt8=0.004),
       "shapes": dict(exact=0.95, le2=0.985, max_frac_gt8=0.004),
       "courtyard": dict(exact=0.95, le2=0.985, max_frac_gt8=0.004)}


def check_against_png(img, ref, kind):
    d = np.abs(img.astype(int) - ref.astype(int)).max(2)
    t = TOL[kind]
    assert (d == 0).mean() >= t["exact"], (d == 0).mean()
    assert (d <= 2).mean() >= t["le2"], (d <= 2).mean()
    assert (d > 8).mean() <= t["max_frac_gt8"], (d > 8).mean()


@pytest.mark.parametrize("case", render_cases(), ids=[c["name"] for c in render_cases()])
def test_oracle_render_matches_reference_png(case):
    """Pins the path-tracing oracle: its float film, tone-mapped as the reference does
    (Core/Film.cu:20-28), reproduces the reference renderer's PNG."""
    import cavalry_b200 as cav
    from oracle import pyoracle as po

    g = np.load(GOLDEN)
    s, w = po.render_path(make_scene(case["gen"]), **case["render"])
    img = cav.film_to_rgb8(s, w)
    check_against_png(img, g[case["name"]], case["gen"]["kind"])


def test_oracle_sample_ranges_compose():
    """Rendering the samples in two ranges gives the film of one range (the CPU baseline
    times a bounded range)."""
    from cavalry_b200 import scenes
    from oracle import pyoracle as po

    room = scenes.mini_room()
    kw = dict(width=32, height=24, spp=4, max_depth=3)
    s, w = po.render_path(room, **kw)
    n = 32 * 24 * 4
    s1, w1 = po.render_path(room, first=0, count=n // 3, **kw)
    s2, w2 = po.render_path(room, first=n // 3, **kw)
    assert np.array_equal(w1 + w2, w)
    assert np.allclose(s1 + s2, s, rtol=1e-5, atol=1e-5)


def test_halton_tables_are_permutations():
    import ctypes

    from oracle import pyoracle as po

    L = po._pt_lib()
    n = L.orc_halton_tables(None, None, None)
    primes = np.zeros(1024, np.uint32)
    start = np.zeros(1024, np.uint32)
    perms = np.zeros(n, np.uint16)
    L.orc_halton_tables(primes.ctypes.data, start.ctypes.data, perms.ctypes.data)
    assert primes[0] == 2 and primes[1023] == 8161
    for k in (0, 1, 5, 100, 1023):
        p = perms[start[k]:start[k] + primes[k]]
        assert np.array_equal(np.sort(p), np.arange(primes[k]))
    assert ctypes.sizeof(ctypes.c_int64) == 8


# ------------------------------------------------------------------------ .pbrt parser
def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


HEADER = """LookAt 0 1 -4  0 1 0  0 1 0
Camera "perspective" "float fov" [45]
Film "image" "integer xresolution" [64] "integer yresolution" [48] "string filename" "x.png"
Sampler "halton" "integer pixelsamples" [8]
Integrator "path" "integer maxdepth" [6]
"""
QUAD = 'Shape "trianglemesh" "integer indices" [0 1 2 0 2 3] "point P" [-1 0 -1 1 0 -1 1 0 1 -1 0 1]\n'


def test_parser_reads_generated_scene_and_camera(tmp_path):
    import cavalry_b200 as cav
    from cavalry_b200 import scenes
    from oracle import pyoracle as po

    room = scenes.mini_room()
    path = str(tmp_path / "room.pbrt")
    scenes.write_pbrt(path, room, width=200, height=100, spp=3, max_depth=7)
    info, c2w = cav.parse_pbrt(path)
    assert (info.width, info.height, info.spp, info.max_depth) == (200, 100, 3, 7)
    assert info.triangles == len(room["indices"]) and info.meshes == len(room["meshes"]) and info.lights == 1
    want = po.look_at_c2w((0, 0, -3.8), (0, 0, 0), (0, 1, 0)).reshape(4, 4).T
    assert np.allclose(c2w, want, atol=1e-6)


def test_parser_overrides(tmp_path):
    import cavalry_b200 as cav

    p = write(tmp_path, "a.pbrt", HEADER + 'WorldBegin\nAreaLightSource "diffuse" "rgb L" [1 1 1]\n' + QUAD +
              "WorldEnd\n")
    info, _ = cav.parse_pbrt(p, spp=32, integrator="rlpath")
    assert info.spp == 32 and info.integrator == 1
    info, _ = cav.parse_pbrt(p)
    assert info.spp == 8 and info.integrator == 0 and info.triangles == 2


def test_parser_reads_a_stream_that_cannot_seek(tmp_path):
    """A .pbrt given as a FIFO (tellg fails) parses like the same text in a regular file."""
    import os
    import threading

    import cavalry_b200 as cav

    text = HEADER + 'WorldBegin\nAreaLightSource "diffuse" "rgb L" [1 1 1]\n' + QUAD + "WorldEnd\n"
    fifo = tmp_path / "scene.fifo"
    os.mkfifo(fifo)

    def feed():
        with open(fifo, "w") as f:
            f.write(text)

    th = threading.Thread(target=feed)
    th.start()
    info, _ = cav.parse_pbrt(str(fifo))
    th.join(timeout=10)
    want, _ = cav.parse_pbrt(write(tmp_path, "same.pbrt", text))
    assert (info.spp, info.triangles, info.lights) == (want.spp, want.triangles, want.lights) == (8, 2, 1)


def test_parser_rejects_scene_without_lights(tmp_path):
    """The reference's light pick randInt(0) yields index -1 (HaltonSampler.h:41-47); the
    loader refuses such a scene instead."""
    import cavalry_b200 as cav

    p = write(tmp_path, "dark.pbrt", HEADER + "WorldBegin\n" + QUAD + "WorldEnd\n")
    with pytest.raises(cav.CavError) as e:
        cav.parse_pbrt(p)
    assert "no lights" in str(e.value)


def test_parser_include_and_named_material(tmp_path):
    import cavalry_b200 as cav

    write(tmp_path, "geo.pbrt", 'NamedMaterial "red"\n' + QUAD)
    p = write(tmp_path, "main.pbrt", HEADER + 'WorldBegin\nMakeNamedMaterial "red" "string type" "matte" '
              '"rgb Kd" [0.8 0.1 0.1]\nAttributeBegin\nAreaLightSource "diffuse" "rgb L" [1 1 1]\n' + QUAD +
              'AttributeEnd\nInclude "geo.pbrt"\nWorldEnd\n')
    info, _ = cav.parse_pbrt(p)
    assert info.meshes == 2 and info.lights == 1 and info.triangles == 4


def test_parser_refuses_include_cycles_and_keeps_repeated_includes(tmp_path):
    """Included files are spliced in place; a file that includes itself, directly, through
    another file or as its last directive, would splice without end and is refused, while
    including the same file several times without a cycle is kept."""
    import cavalry_b200 as cav

    light = 'AttributeBegin\nAreaLightSource "diffuse" "rgb L" [1 1 1]\n' + QUAD + 'AttributeEnd\n'
    write(tmp_path, "leaf.pbrt", QUAD)
    write(tmp_path, "twice.pbrt", 'Include "leaf.pbrt"\nInclude "leaf.pbrt"\n')
    write(tmp_path, "self.pbrt", QUAD + 'Include "self.pbrt"\n')
    write(tmp_path, "a.pbrt", 'Include "b.pbrt"\n')
    write(tmp_path, "b.pbrt", QUAD + 'Include "a.pbrt"\n')
    ok = write(tmp_path, "ok.pbrt", HEADER + "WorldBegin\n" + light +
               'Include "twice.pbrt"\nInclude "leaf.pbrt"\nWorldEnd\n')
    info, _ = cav.parse_pbrt(ok)
    assert info.meshes == 4 and info.triangles == 8
    for target in ("self.pbrt", "a.pbrt"):
        p = write(tmp_path, "main.pbrt", HEADER + "WorldBegin\n" + light + f'Include "{target}"\nWorldEnd\n')
        with pytest.raises(cav.CavError, match="Include cycle"):
            cav.parse_pbrt(p)
        with pytest.raises(cav.CavError, match="Include cycle"):
            cav.load_pbrt_triangles(p)
    p = write(tmp_path, "main.pbrt", HEADER + "WorldBegin\n" + light + 'Include "main.pbrt"\nWorldEnd\n')
    with pytest.raises(cav.CavError, match="Include cycle"):
        cav.parse_pbrt(p)


@pytest.mark.parametrize("text,msg", [
    ('Camera "perspective" "float fov" [1e+05]\n', "unrecognized character"),
    ("Frobnicate 1 2 3\n", "Unrecognized Keyword"),
    ('Shape "trianglemesh" "integer indices" [0 1 2 "point P" [0 0 0]\n', ""),
])
def test_parser_rejects_like_the_reference(tmp_path, text, msg):
    """Lexing.cu:47-49 has no '+' in numbers; Lexing.h:33-36 rejects unknown keywords."""
    import cavalry_b200 as cav

    p = write(tmp_path, "bad.pbrt", text)
    with pytest.raises(cav.CavError) as e:
        cav.parse_pbrt(p)
    assert msg in str(e.value)


def test_parser_missing_file():
    import cavalry_b200 as cav

    with pytest.raises(cav.CavError) as e:
        cav.parse_pbrt("/nonexistent/scene.pbrt")
    assert "fileNotFound" in str(e.value)


def test_sphere_scene_sizes():
    from cavalry_b200 import scenes

    v, f = scenes.icosphere(3)
    assert len(f) == 20 * 4 ** 3 and len(v) == 10 * 4 ** 3 + 2
    assert np.allclose(np.linalg.norm(v, axis=1), 1)
    sc = scenes.sphere_scene(4, 2, seed=1)
    assert len(sc["indices"]) == 12 + 4 * 320 + 3 * 2
    assert len(sc["lights"]) == 3


def test_golden_sphere_scenes_have_disjoint_lights():
    """The generator places light quads in one plane under the ceiling; two that overlap make
    a shadow ray end inside both, so its visibility turns on the last bit of `t < limit` and
    no two renderers agree there.  Every golden case keeps its quads apart."""
    import make_render_golden

    for name, gen, _ in make_render_golden.CASES:
        if gen["kind"] != "spheres":
            continue
        sc = make_scene(gen)
        boxes = []
        for mid, _ in sc["lights"]:
            _, first, n, _ = sc["meshes"][mid]
            p = sc["positions"][np.unique(sc["indices"][first:first + n])]
            boxes.append((p[:, 0].min(), p[:, 0].max(), p[:, 2].min(), p[:, 2].max()))
        for i in range(len(boxes)):
            for j in range(i + 1, len(boxes)):
                a, b = boxes[i], boxes[j]
                assert not (a[0] < b[1] and b[0] < a[1] and a[2] < b[3] and b[2] < a[3]), (name, i, j)


def _ply_text(P, faces, fmt, extra=True):
    """A PLY of the given format with an extra vertex property and an extra element."""
    import struct

    head = ["ply", f"format {fmt} 1.0", "comment written by the test", f"element vertex {len(P)}",
            "property float x", "property float y", "property float z"]
    if extra:
        head.append("property double confidence")
    head += [f"element face {len(faces)}", "property list uchar int vertex_indices"]
    if extra:
        head += ["element edge 1", "property int vertex1", "property int vertex2"]
    head.append("end_header")
    out = ("\n".join(head) + "\n").encode()
    if fmt == "ascii":
        body = [" ".join(f"{c:.9g}" for c in p) + (" 0.5" if extra else "") for p in P]
        body += [" ".join(map(str, [len(f)] + list(f))) for f in faces]
        if extra:
            body.append("0 1")
        return out + ("\n".join(body) + "\n").encode()
    e = "<" if fmt == "binary_little_endian" else ">"
    for p in P:
        out += struct.pack(e + "fff", *p) + (struct.pack(e + "d", 0.5) if extra else b"")
    for f in faces:
        out += struct.pack(e + "B" + "i" * len(f), len(f), *f)
    if extra:
        out += struct.pack(e + "ii", 0, 1)
    return out


def _scene_with_shape(tmp_path, shape_line, name="s.pbrt"):
    text = ('LookAt 0 0 -3  0 0 0  0 1 0\nCamera "perspective" "float fov" [40]\n'
            'Film "image" "integer xresolution" [32] "integer yresolution" [32]\n'
            'Sampler "halton" "integer pixelsamples" [1]\nIntegrator "path" "integer maxdepth" [2]\nWorldBegin\n'
            'AttributeBegin\nAreaLightSource "diffuse" "rgb L" [1 1 1]\n'
            'Shape "trianglemesh" "integer indices" [0 1 2] "point P" [0 1 0 1 1 0 0 1 1]\nAttributeEnd\n'
            f'AttributeBegin\nTranslate 0.25 -0.5 1\n{shape_line}\nAttributeEnd\nWorldEnd\n')
    p = tmp_path / name
    p.write_text(text)
    return str(p)


@pytest.mark.parametrize("extra", [True, False])
@pytest.mark.parametrize("fmt", ["ascii", "binary_little_endian", "binary_big_endian"])
def test_ply_mesh_loads_like_the_inline_mesh(tmp_path, fmt, extra):
    """Core/TriangleMesh.cu:53-108: x/y/z of any PLY encoding, each face's first three indices
    (a quad keeps one triangle), other properties and elements skipped; the CTM applies.
    Without the extra property and element, a little-endian file takes the block-read path
    (float vertices only, faces holding only their index list)."""
    import cavalry_b200 as cav

    rng = np.random.default_rng(1)
    P = rng.uniform(-1, 1, (7, 3)).astype(np.float32)
    faces = [(0, 1, 2), (2, 3, 4, 5), (5, 6, 0)]
    (tmp_path / "m.ply").write_bytes(_ply_text(P, faces, fmt, extra=extra))
    a = cav.load_pbrt_triangles(_scene_with_shape(tmp_path, 'Shape "plymesh" "string filename" "m.ply"', "a.pbrt"))
    flat = " ".join("%.9g" % c for c in P.reshape(-1))
    b = cav.load_pbrt_triangles(_scene_with_shape(
        tmp_path, f'Shape "trianglemesh" "integer indices" [0 1 2 2 3 4 5 6 0] "point P" [{flat}]', "b.pbrt"))
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert len(a[1]) == 1 + 3


def test_ply_errors_are_reported(tmp_path):
    import cavalry_b200 as cav

    P = np.zeros((3, 3), np.float32)
    (tmp_path / "short.ply").write_bytes(_ply_text(P, [(0, 1)], "ascii", extra=False))
    with pytest.raises(cav.CavError, match="read ply file failed"):
        cav.load_pbrt_triangles(_scene_with_shape(tmp_path, 'Shape "plymesh" "string filename" "short.ply"'))
    with pytest.raises(cav.CavError, match="read ply file failed"):
        cav.load_pbrt_triangles(_scene_with_shape(tmp_path, 'Shape "plymesh" "string filename" "missing.ply"'))
    with pytest.raises(cav.CavError, match="ShapeMesh type not supported"):
        cav.load_pbrt_triangles(_scene_with_shape(tmp_path, 'Shape "cylinder" "float radius" [1]'))


def test_sphere_and_disk_shapes_follow_the_reference_tessellation(tmp_path):
    """ShapeMesh/Sphere.cu:3-94 (2046 vertices, 2048 triangles) and ShapeMesh/Disk.cu:4-50
    (361 vertices, 360 triangles), placed by the CTM; the scene generator's copies agree."""
    import os

    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    P, I, _ = cav.load_pbrt_triangles(_scene_with_shape(tmp_path, 'Shape "sphere" "float radius" [0.75]'))
    assert len(I) == 1 + 2048 and len(P) == 3 + 2046
    sp = P[3:] - np.array([0.25, -0.5, 1], np.float32)
    assert np.allclose(np.linalg.norm(sp, axis=1), 0.75, atol=1e-6)
    _, ref_p, ref_i = scenes.sphere_shape_mesh(0.75)
    assert np.array_equal(I[1:] - 3, ref_i)
    assert np.abs(sp - ref_p).max() < 1e-6
    P, I, _ = cav.load_pbrt_triangles(_scene_with_shape(tmp_path, 'Shape "disk" "float radius" [0.5] "float height" [0.2]'))
    assert len(I) == 1 + 360 and len(P) == 3 + 361
    dp, di = scenes.disk_shape_mesh(0.5, 0.2)
    assert np.array_equal(I[1:] - 3, di)
    assert np.abs(P[3:] - np.array([0.25, -0.5, 1], np.float32) - dp).max() < 1e-6
    sc = scenes.shapes_scene(31, quad_light=True)
    path = str(tmp_path / "shapes.pbrt")
    scenes.write_pbrt(path, sc, width=32, height=24, spp=1, max_depth=2)
    P, I, _ = cav.load_pbrt_triangles(path)
    assert os.path.exists(path) and np.abs(P[I] - sc["positions"][sc["indices"]]).max() < 1e-6


def test_parser_reads_the_direct_lighting_integrator(tmp_path):
    """CreateIntegrator.cu:12-14: "directlighting" takes no maxdepth; the scene reports it as 3."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    path = str(tmp_path / "d.pbrt")
    scenes.write_pbrt(path, scenes.mini_room(), width=32, height=32, spp=2, max_depth=7, integrator="directlighting")
    info, _ = cav.parse_pbrt(path)
    assert info.integrator == 3 and info.max_depth == 1
    info, _ = cav.parse_pbrt(path, integrator="path")
    assert info.integrator == 0 and info.max_depth == 7


def test_textures_and_light_sources_parse_like_the_reference(tmp_path):
    """Texture / "texture Kd" / LightSource (Core/Texture.cu:12-25, Lights/LightObject.h:89-127):
    a PNG image or one black texel, an unknown texture name refused, an "infinite" light with
    a map, and an unrecognised LightSource kept in the light list (black)."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    scenes.write_png(str(tmp_path / "t.png"), np.full((4, 8, 4), 200, np.uint8))
    head = ('LookAt 0 0 -3  0 0 0  0 1 0\nCamera "perspective" "float fov" [40]\n'
            'Film "image" "integer xresolution" [16] "integer yresolution" [16]\n'
            'Sampler "halton" "integer pixelsamples" [1]\nIntegrator "path" "integer maxdepth" [2]\nWorldBegin\n')
    tri = 'Shape "trianglemesh" "integer indices" [0 1 2] "point P" [0 0 0 1 0 0 0 1 0] "float uv" [0 0 1 0 0 1]\n'

    def parse(body):
        p = tmp_path / "s.pbrt"
        p.write_text(head + body + "WorldEnd\n")
        return cav.parse_pbrt(str(p))[0]

    info = parse('LightSource "infinite" "rgb L" [1 1 1] "string mapname" "t.png"\nLightSource "point"\n'
                 'Texture "a" "spectrum" "imagemap" "string filename" "t.png"\nTexture "b" "spectrum" "imagemap"\n'
                 'Material "matte" "texture Kd" "a"\n' + tri + 'Material "plastic" "texture Kd" "b"\n' + tri)
    assert info.lights == 2 and info.triangles == 2
    with pytest.raises(cav.CavError, match="texture not found"):
        parse('LightSource "infinite"\nMaterial "matte" "texture Kd" "missing"\n' + tri)
    (tmp_path / "t.jpg").write_bytes(b"\xff\xd8\xff")
    with pytest.raises(cav.CavError, match="only PNG"):
        parse('LightSource "infinite"\nTexture "a" "spectrum" "imagemap" "string filename" "t.jpg"\n' + tri)
    with pytest.raises(cav.CavError, match="no lights"):
        parse(tri)


@pytest.mark.parametrize("text,value", [(".5", 0.5), ("-.5", -0.5), ("1e", 1.0), ("2.5e1", 25.0), ("1-2", 1.0),
                                        ("0.1", float(np.float32(0.1))), ("3.4028235e38", float(np.finfo(np.float32).max)),
                                        ("1.17549435e-38", float(np.finfo(np.float32).tiny))])
def test_lexer_numbers_read_like_stof(tmp_path, text, value):
    """Numbers are read as the reference's lexer reads them with std::stof (Lexing.cu:88-103): the
    longest prefix of the token that is a number, a leading '.' read as "0.", correctly
    rounded to float."""
    import cavalry_b200 as cav

    p = tmp_path / "n.pbrt"
    p.write_text('LookAt 0 0 -3  0 0 0  0 1 0\nCamera "perspective" "float fov" [40]\n'
                 'Film "image" "integer xresolution" [16] "integer yresolution" [16]\n'
                 'Sampler "halton" "integer pixelsamples" [1]\nIntegrator "path" "integer maxdepth" [2]\nWorldBegin\n'
                 'AttributeBegin\nAreaLightSource "diffuse" "rgb L" [1 1 1]\n'
                 'Shape "trianglemesh" "integer indices" [0 1 2] "point P" [0 0 5 1 0 5 0 1 5]\nAttributeEnd\n'
                 f'AttributeBegin\nScale {text} 1 1\n'
                 'Shape "trianglemesh" "integer indices" [0 1 2] "point P" [1 0 0 0 1 0 0 0 1]\nAttributeEnd\nWorldEnd\n')
    pos, _, _ = cav.load_pbrt_triangles(str(p))
    assert pos[3, 0] == np.float32(value)


@pytest.mark.parametrize("text", ["1e-40", "1e39", "-"])
def test_lexer_rejects_numbers_stof_rejects(tmp_path, text):
    """Out-of-range (std::stof's ERANGE: overflow, or underflow into the subnormals) and
    non-numbers are lexing errors, as in the reference."""
    import cavalry_b200 as cav

    p = tmp_path / "n.pbrt"
    p.write_text(f'LookAt 0 0 -3  0 0 0  0 1 0\nCamera "perspective" "float fov" [{text}]\nWorldBegin\nWorldEnd\n')
    with pytest.raises(cav.CavError, match="bad number"):
        cav.parse_pbrt(str(p))


@pytest.mark.parametrize("args,msg", [
    ([], "usage"),
    (["--input"], "missing value for --input"),
    (["--bogus"], "unknown argument --bogus"),
    (["--input", "x.pbrt", "--spp", "abc"], "invalid integer value 'abc' for --spp"),
    (["--input", "x.pbrt", "--spp", "12x"], "invalid integer value '12x' for --spp"),
    (["--input", "x.pbrt", "--spp", "99999999999999"], "invalid integer value"),
    (["--input", "x.pbrt", "--bvh-opt-rounds", ""], "invalid integer value '' for --bvh-opt-rounds"),
    (["--input", "x.pbrt", "--device", "1.5"], "invalid integer value '1.5' for --device"),
])
def test_cli_refuses_bad_arguments(args, msg):
    """The `cavalry` CLI reads --spp, --bvh-opt-rounds and --device as whole ints (the reference
    parses them as ints through cxxopts, main.cu:25-96) and exits with status 2 on bad or
    missing arguments, before it touches a GPU."""
    import subprocess

    from cavalry_b200 import build_ext

    cli = build_ext.CLI
    if not cli.exists():
        build_ext.build_cli()
    r = subprocess.run([str(cli), *args], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    assert msg in r.stderr
