"""Fixture of the full-size path-traced scene (config 3): the reference renderer's PNG of the
5.24M-triangle icosphere scene at 1920 x 1080, 64 spp, depth 8, run by oracle/ref_cli (the
reference CLI built by oracle/build_ref_full.sh; always --bvh-opt-rounds 0, its treelet
kernel faults on the B200).  Every 4th row and column of the 8-bit image is kept (480 x 270
pixels), which is what tests/test_gpu_render.py compares against this project's render.

    python tests/golden/make_config3_golden.py [OUT.npz]      (on a machine with a GPU)
"""
import json
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cavalry_b200 import scenes  # noqa: E402
from oracle import ref_cli  # noqa: E402

SCENE = {"n_spheres": 64, "level": 6, "seed": 9}
RENDER = {"width": 1920, "height": 1080, "spp": 64, "max_depth": 8}
STEP = 4


def main(out: str):
    with tempfile.TemporaryDirectory() as tmp:
        pbrt = Path(tmp) / "spheres.pbrt"
        scenes.write_pbrt(pbrt, scenes.sphere_scene(**SCENE), **RENDER)
        t0 = time.time()
        img, text = ref_cli.render(str(pbrt), str(Path(tmp) / "ref.png"), spp=RENDER["spp"], timeout=3000)
        wall = time.time() - t0
    meta = {"scene": SCENE, "render": RENDER, "step": STEP, "ref_wall_s": round(wall, 1),
            "rendering": [ln for ln in text.splitlines() if ln.startswith("Rendering took")]}
    np.savez_compressed(out, meta=json.dumps(meta), sub=img[::STEP, ::STEP])
    print(json.dumps(meta))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(ROOT / "tests" / "golden" / "render_spheres5m_sub4.npz"))
