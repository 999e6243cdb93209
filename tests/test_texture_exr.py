"""CPU tests of the OpenEXR texture loader (the reference reads .exr through tinyexr's LoadEXR,
Core/Texture.cu:34-57): files written and decoded by OpenCV's EXR codec (the OpenEXR library;
tests/golden/make_exr_golden.py) must decode to the same RGBA floats, bit for bit, for every
codec the loader reads; a PIZ file is refused with a message; the project's own writer (the
scene generator's) round-trips through the loader."""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "exr"


def cases():
    if not (GOLDEN / "expected.npz").exists():
        return []
    return sorted(k for k in np.load(GOLDEN / "expected.npz").files if not k.startswith("piz"))


@pytest.mark.parametrize("name", cases())
def test_exr_fixture_decodes_like_openexr(name):
    import cavalry_b200 as cav

    want = np.load(GOLDEN / "expected.npz")[name]
    got = cav.load_texture_exr(str(GOLDEN / f"{name}.exr"))
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), name


def test_exr_piz_is_refused_with_a_message():
    import cavalry_b200 as cav

    with pytest.raises(cav.CavError) as e:
        cav.load_texture_exr(str(GOLDEN / "piz_half_3.exr"))
    assert "compression 4" in str(e.value)


@pytest.mark.parametrize("comp", ["none", "rle", "zips", "zip"])
@pytest.mark.parametrize("dtype", [np.float16, np.float32])
@pytest.mark.parametrize("channels", [1, 3, 4])
def test_exr_writer_round_trips(tmp_path, comp, dtype, channels):
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    rng = np.random.default_rng(channels)
    img = (rng.random((21, 34, channels)) * 5 - 1).astype(dtype)
    img[3:8, 2:30] = 2.0
    p = str(tmp_path / "t.exr")
    scenes.write_exr(p, img, compression=comp)
    got = cav.load_texture_exr(p)
    ref = img.astype(np.float32)
    if channels == 1:
        want = np.repeat(ref, 4, axis=2)
    elif channels == 3:
        want = np.concatenate([ref, np.ones(ref.shape[:2] + (1,), np.float32)], axis=2)
    else:
        want = ref
    assert np.array_equal(got, want)


def test_exr_layer_prefixes_and_the_first_four_channels(tmp_path):
    """LoadEXR strips layer prefixes and looks for R, G, B, A among the first four channels
    in header (name) order only."""
    import cavalry_b200 as cav
    from cavalry_b200 import scenes

    img = np.arange(5 * 7 * 3, dtype=np.float32).reshape(5, 7, 3)
    p = str(tmp_path / "layer.exr")
    scenes.write_exr(p, img, channels=["diffuse.R", "diffuse.G", "diffuse.B"])
    got = cav.load_texture_exr(p)
    assert np.array_equal(got[..., :3], img) and (got[..., 3] == 1).all()
    # five channels whose first four in name order (A, B, C, D) hold no R or G: refused
    five = np.zeros((4, 4, 5), np.float32)
    p = str(tmp_path / "five.exr")
    scenes.write_exr(p, five, channels=["A", "B", "C", "D", "R"])
    with pytest.raises(cav.CavError) as e:
        cav.load_texture_exr(p)
    assert "not found" in str(e.value)
