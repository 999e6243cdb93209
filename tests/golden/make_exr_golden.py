"""Generates the OpenEXR fixtures of tests/test_texture_exr.py with an independent encoder and
decoder: OpenCV's EXR codec (the OpenEXR library), never this project's writer or reader.

    OPENCV_IO_ENABLE_OPENEXR=1 python tests/golden/make_exr_golden.py

For each compression OpenCV writes (NONE, RLE, ZIPS, ZIP; PIZ for the refusal case), each
pixel type (HALF, FLOAT) and 1, 3 and 4 channels, a small seeded image is written to
tests/golden/exr/<compression>_<type>_<channels>.exr; OpenCV's own decode of every file is
stored, in the loader's RGBA layout (R, G, B, A; a single channel in all four; A = 1 when
absent), in tests/golden/exr/expected.npz.
"""
import os

os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")

from pathlib import Path  # noqa: E402

import cv2  # noqa: E402
import numpy as np  # noqa: E402

HERE = Path(__file__).resolve().parent / "exr"
COMP = {"none": cv2.IMWRITE_EXR_COMPRESSION_NO, "rle": cv2.IMWRITE_EXR_COMPRESSION_RLE,
        "zips": cv2.IMWRITE_EXR_COMPRESSION_ZIPS, "zip": cv2.IMWRITE_EXR_COMPRESSION_ZIP,
        "piz": cv2.IMWRITE_EXR_COMPRESSION_PIZ}
TYPES = {"half": cv2.IMWRITE_EXR_TYPE_HALF, "float": cv2.IMWRITE_EXR_TYPE_FLOAT}


def image(c: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    h, w = 19, 37
    a = (rng.standard_normal((h, w, c)) * 3).astype(np.float32)
    a[2:6, 4:30] = 1.25                                  # runs (RLE)
    a[0, 0] = 0.0
    a[0, 1] = -0.0
    a[0, 2] = 6.0e-6                                     # a half subnormal
    a[0, 3] = 65504.0                                    # the largest half
    a[0, 4] = 1.0e-3
    return a[..., 0] if c == 1 else a


def rgba(decoded: np.ndarray) -> np.ndarray:
    d = decoded.astype(np.float32)
    if d.ndim == 2:
        return np.repeat(d[..., None], 4, axis=2)
    if d.shape[2] == 3:  # OpenCV's B, G, R
        return np.concatenate([d[..., ::-1], np.ones(d.shape[:2] + (1,), np.float32)], axis=2)
    return np.concatenate([d[..., 2::-1], d[..., 3:4]], axis=2)  # B, G, R, A


def main():
    HERE.mkdir(exist_ok=True)
    expected = {}
    seed = 0
    for comp, cflag in COMP.items():
        for tname, tflag in TYPES.items():
            for c in (1, 3, 4):
                if comp == "piz" and (tname, c) != ("half", 3):
                    continue
                seed += 1
                name = f"{comp}_{tname}_{c}"
                path = HERE / f"{name}.exr"
                img = image(c, seed)
                ok = cv2.imwrite(str(path), img, [cv2.IMWRITE_EXR_COMPRESSION, cflag, cv2.IMWRITE_EXR_TYPE, tflag])
                assert ok, name
                expected[name] = rgba(cv2.imread(str(path), cv2.IMREAD_UNCHANGED))
    np.savez_compressed(HERE / "expected.npz", **expected)
    print(f"wrote {len(expected)} files to {HERE}")


if __name__ == "__main__":
    main()
