"""Test infrastructure: runs the reference renderer (oracle/_ref/cavalry_ref, built by
oracle/build_ref_full.sh) and reads its PNG.

The reference is always run with --bvh-opt-rounds 0: its treelet kernel raised an illegal
memory access on the B200 and is never launched again (see oracle/ref_harness.cu).
"""
from __future__ import annotations

import struct
import subprocess
import zlib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_BIN = HERE / "_ref" / "cavalry_ref"


def available() -> bool:
    return REF_BIN.exists()


def render(pbrt: str, out_png: str, spp: int | None = None, integrator: str = "path", timeout: float = 600.0):
    """Runs the reference CLI (main.cu:25-96).  Returns (rgb8 image [H,W,3], stdout text)."""
    pbrt = str(Path(pbrt).resolve())
    out_png = str(Path(out_png).resolve())
    cmd = [str(REF_BIN), "--input", pbrt, "--output", out_png, "--integrator", integrator, "--bvh-opt-rounds", "0"]
    if spp is not None:
        cmd += ["--spp", str(int(spp))]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=str(Path(out_png).parent))
    if r.returncode != 0:
        raise RuntimeError(f"reference renderer failed ({r.returncode}): {r.stdout[-1500:]} {r.stderr[-1500:]}")
    return read_png(out_png), r.stdout


def read_png(path) -> np.ndarray:
    """8-bit RGB PNG reader (filter types 0-4), enough for the reference's svpng output."""
    data = Path(path).read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n", "not a PNG"
    pos, idat, w = 8, b"", 0
    h = 0
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if typ == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and ctype in (2, 6), (depth, ctype)
            bpp = 3 if ctype == 2 else 4
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    stride = w * bpp
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        f = raw[y * (stride + 1)]
        line = np.frombuffer(raw, np.uint8, stride, y * (stride + 1) + 1).astype(np.int32)
        cur = np.zeros(stride, np.int32)
        for x in range(stride):
            a = cur[x - bpp] if x >= bpp else 0
            b = prev[x]
            c = prev[x - bpp] if x >= bpp else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) // 2
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            cur[x] = (line[x] + p) & 0xFF
        out[y] = cur
        prev = cur
    return out.reshape(h, w, bpp)[:, :, :3]
