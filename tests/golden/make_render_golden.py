"""Generates tests/golden/render_ref.npz: 8-bit renders by the reference's own renderer.

Runs on a machine with a GPU and the reference renderer built by oracle/build_ref_full.sh
(oracle/_ref/cavalry_ref); writes the .pbrt scenes from the seeded generators of
cavalry_b200.scenes, renders each with ``--bvh-opt-rounds 0`` and stores the PNG pixels
with the case parameters.  The tests regenerate the same .pbrt text from the parameters.

    python tests/golden/make_render_golden.py OUT.npz
"""
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cavalry_b200 import scenes  # noqa: E402
from oracle import ref_cli  # noqa: E402

# (name, generator kwargs, render kwargs)
CASES = [
    ("room_d1_s1", {"kind": "room"}, dict(width=256, height=256, spp=1, max_depth=1)),
    ("room_d2_s16", {"kind": "room"}, dict(width=256, height=256, spp=16, max_depth=2)),
    ("room_d5_s1", {"kind": "room"}, dict(width=256, height=256, spp=1, max_depth=5)),
    ("room_d5_s16", {"kind": "room"}, dict(width=256, height=256, spp=16, max_depth=5)),
    ("spheres_mixed", {"kind": "spheres", "n_spheres": 12, "level": 2, "seed": 5},
     dict(width=128, height=96, spp=8, max_depth=8)),
    ("spheres_glass", {"kind": "spheres", "n_spheres": 10, "level": 3, "seed": 6, "materials": ["glass"]},
     dict(width=128, height=96, spp=8, max_depth=8)),
    ("spheres_mirror", {"kind": "spheres", "n_spheres": 10, "level": 3, "seed": 7, "materials": ["mirror"]},
     dict(width=128, height=96, spp=8, max_depth=8)),
    ("spheres_plastic", {"kind": "spheres", "n_spheres": 10, "level": 3, "seed": 8, "materials": ["plastic"]},
     dict(width=128, height=96, spp=8, max_depth=8)),
    ("spheres_metal", {"kind": "spheres", "n_spheres": 10, "level": 3, "seed": 11, "materials": ["metal", "gold"]},
     dict(width=128, height=96, spp=8, max_depth=8)),
    ("spheres_substrate", {"kind": "spheres", "n_spheres": 10, "level": 3, "seed": 12, "materials": ["substrate"]},
     dict(width=128, height=96, spp=8, max_depth=8)),
    ("spheres_roughglass", {"kind": "spheres", "n_spheres": 10, "level": 3, "seed": 15,
                            "materials": ["roughglass"]},
     dict(width=128, height=96, spp=8, max_depth=8)),
    # pbrt sphere / disk shapes (tessellated by both loaders) and a cone-sampled sphere light
    ("shapes_sphere_light", {"kind": "shapes", "seed": 31}, dict(width=160, height=120, spp=8, max_depth=5)),
    ("shapes_two_lights", {"kind": "shapes", "seed": 32, "quad_light": True},
     dict(width=160, height=120, spp=8, max_depth=5)),
    # the spheres_mixed scene with every triangle mesh in a binary PLY file ("plymesh")
    ("spheres_mixed_ply", {"kind": "spheres", "n_spheres": 12, "level": 2, "seed": 5, "ply": True},
     dict(width=128, height=96, spp=8, max_depth=8)),
    # DirectLightingIntegrator: emission + one light sample per camera ray, no MIS
    ("room_direct_s16", {"kind": "room"}, dict(width=256, height=256, spp=16, max_depth=5, integrator="directlighting")),
    ("spheres_direct", {"kind": "spheres", "n_spheres": 12, "level": 2, "seed": 5},
     dict(width=128, height=96, spp=8, max_depth=8, integrator="directlighting")),
    ("shapes_direct", {"kind": "shapes", "seed": 32, "quad_light": True},
     dict(width=160, height=120, spp=8, max_depth=5, integrator="directlighting")),
    # image textures ("texture Kd" on matte and plastic, uv coordinates) under an environment
    # map ("infinite" with "mapname"): alone, with an area light, and with direct lighting
    ("courtyard_env", {"kind": "courtyard", "seed": 41}, dict(width=160, height=120, spp=8, max_depth=5)),
    ("courtyard_env_area", {"kind": "courtyard", "seed": 42, "area_light": True},
     dict(width=160, height=120, spp=8, max_depth=5)),
    ("courtyard_direct", {"kind": "courtyard", "seed": 41},
     dict(width=160, height=120, spp=8, max_depth=5, integrator="directlighting")),
    # the environment as an HDR OpenEXR map (HALF channels, ZIP compression; tinyexr in the
    # reference, this project's EXR loader here): alone and with an area light
    ("courtyard_env_exr", {"kind": "courtyard", "seed": 41, "hdr_sky": True},
     dict(width=160, height=120, spp=8, max_depth=5)),
    ("courtyard_env_exr_area", {"kind": "courtyard", "seed": 42, "area_light": True, "hdr_sky": True},
     dict(width=160, height=120, spp=8, max_depth=5)),
    # the learning integrator (the .pbrt names it; both renderers read the Integrator line)
    ("room_rlpath_s16", {"kind": "room"}, dict(width=128, height=128, spp=16, max_depth=5, integrator="rlpath")),
    ("spheres_rlpath_s16", {"kind": "spheres", "n_spheres": 12, "level": 3, "seed": 5},
     dict(width=128, height=96, spp=16, max_depth=8, integrator="rlpath")),
    ("spheres_rough_rlpath_s16", {"kind": "spheres", "n_spheres": 12, "level": 3, "seed": 14,
                                  "materials": ["metal", "gold", "substrate", "roughglass"]},
     dict(width=128, height=96, spp=16, max_depth=8, integrator="rlpath")),
    ("courtyard_rlpath_s16", {"kind": "courtyard", "seed": 42, "area_light": True},
     dict(width=160, height=120, spp=16, max_depth=5, integrator="rlpath")),
]


def make_scene(gen: dict) -> dict:
    g = dict(gen)
    kind = g.pop("kind")
    ply = g.pop("ply", False)
    if kind == "room":
        sc = scenes.mini_room()
    elif kind == "shapes":
        sc = scenes.shapes_scene(**g)
    elif kind == "courtyard":
        sc = scenes.courtyard_scene(**g)
    else:
        if "materials" in g:
            g["materials"] = tuple(g["materials"])
        sc = scenes.sphere_scene(**g)
    if ply:
        sc["write_ply"] = True
    return sc


def main(out: str):
    """Renders every case with the reference CLI; a case already in `out` with the same
    scene and render settings keeps its image (the renders take minutes on a GPU)."""
    arrays = {}
    meta = []
    old = {}
    if Path(out).exists():
        g = np.load(out)
        old = {c["name"]: (c, g[c["name"]]) for c in json.loads(str(g["meta"]))}
    with tempfile.TemporaryDirectory() as tmp:
        for name, gen, rk in CASES:
            entry = {"name": name, "gen": gen, "render": rk}
            if name in old and json.dumps(old[name][0], sort_keys=True) == json.dumps(entry, sort_keys=True):
                arrays[name] = old[name][1]
                meta.append(entry)
                print(name, "kept", flush=True)
                continue
            pbrt = Path(tmp) / f"{name}.pbrt"
            scenes.write_pbrt(pbrt, make_scene(gen), **rk)
            img, _ = ref_cli.render(str(pbrt), str(Path(tmp) / f"{name}.png"), spp=rk["spp"],
                                    integrator=rk.get("integrator", "path"))
            arrays[name] = img
            meta.append({"name": name, "gen": gen, "render": rk})
            print(name, img.shape, float(img.mean()), flush=True)
    np.savez_compressed(out, meta=json.dumps(meta), **arrays)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(ROOT / "tests" / "golden" / "render_ref.npz"))
