"""The texture loader (image_load.cpp, through cav_load_texture_png, no GPU) against PNGs
written here with every scanline filter, colour type and bit depth it accepts: the result is
the source pixels as RGBA8 (16-bit samples by their high byte, palettes and their tRNS
alpha, greyscale replicated), rows bottom-up, colour channels mapped through the oracle's
load-time inverse sRGB table (Core/Texture.cu:19, :61-71)."""
import struct
import zlib

import numpy as np
import pytest


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    if pa <= pb and pa <= pc:
        return a
    return b if pb <= pc else c


def _filter_rows(raw_rows, bpp):
    """Filter type y % 5 on row y (None, Sub, Up, Average, Paeth)."""
    out, prev = [], bytes(len(raw_rows[0]))
    for y, row in enumerate(raw_rows):
        f = y % 5
        enc = bytearray()
        for x, v in enumerate(row):
            a = row[x - bpp] if x >= bpp else 0
            b = prev[x]
            c = prev[x - bpp] if x >= bpp else 0
            pred = [0, a, b, (a + b) // 2, _paeth(a, b, c)][f]
            enc.append((v - pred) & 0xFF)
        out.append(bytes([f]) + bytes(enc))
        prev = row
    return b"".join(out)


def _chunk(t, d):
    return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)


def write_png(path, samples, ctype, depth, palette=None, trns=None, interlace=0):
    """samples: [H, W, channels] integer array in the sample range of `depth`."""
    h, w, ch = samples.shape
    dt = ">u2" if depth == 16 else "u1"
    rows = [samples[y].astype(dt).tobytes() for y in range(h)]
    bpp = ch * depth // 8
    data = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, interlace))
    if palette is not None:
        data += _chunk(b"PLTE", palette.astype(np.uint8).tobytes())
    if trns is not None:
        data += _chunk(b"tRNS", trns.astype(np.uint8).tobytes())
    data += _chunk(b"IDAT", zlib.compress(_filter_rows(rows, bpp), 6)) + _chunk(b"IEND", b"")
    path.write_bytes(data)


CASES = [(0, 8), (0, 16), (2, 8), (2, 16), (3, 8), (4, 8), (4, 16), (6, 8), (6, 16)]
CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}


@pytest.mark.parametrize("ctype,depth", CASES)
def test_png_decodes_like_the_reference_loader(tmp_path, ctype, depth):
    import cavalry_b200 as cav
    from oracle import pyoracle as po

    rng = np.random.default_rng(100 * ctype + depth)
    h, w = 5, 7
    ch = CHANNELS[ctype]
    palette = trns = None
    if ctype == 3:
        palette = rng.integers(0, 256, (6, 3))
        trns = rng.integers(0, 256, 4)  # entries 4 and 5 are opaque
        samples = rng.integers(0, 6, (h, w, 1))
    else:
        samples = rng.integers(0, 1 << depth, (h, w, ch))
    path = tmp_path / f"t{ctype}_{depth}.png"
    write_png(path, samples, ctype, depth, palette, trns)

    top8 = (samples >> 8) if depth == 16 else samples  # 16-bit samples keep their high byte
    if ctype == 3:
        k = samples[..., 0]
        rgb = palette[k]
        alpha = np.where(k < len(trns), trns[np.minimum(k, len(trns) - 1)], 255)
    elif ch <= 2:
        rgb = np.repeat(top8[..., :1], 3, axis=2)
        alpha = top8[..., 1] if ch == 2 else np.full((h, w), 255)
    else:
        rgb = top8[..., :3]
        alpha = top8[..., 3] if ch == 4 else np.full((h, w), 255)
    lut = po.load_gamma_table()
    want = np.concatenate([lut[rgb.astype(np.uint8)], alpha.astype(np.uint8)[..., None]], axis=2)[::-1]
    got = cav.load_texture_png(str(path))
    assert got.shape == (h, w, 4)
    assert np.array_equal(got, want)


def test_png_errors_are_reported(tmp_path):
    import cavalry_b200 as cav

    good = np.zeros((2, 2, 4), np.int64)
    write_png(tmp_path / "inter.png", good, 6, 8, interlace=1)
    with pytest.raises(cav.CavError, match="interlaced"):
        cav.load_texture_png(str(tmp_path / "inter.png"))
    (tmp_path / "x.png").write_bytes(b"not a png at all")
    with pytest.raises(cav.CavError, match="not a PNG"):
        cav.load_texture_png(str(tmp_path / "x.png"))
    write_png(tmp_path / "ok.png", good, 6, 8)
    (tmp_path / "cut.png").write_bytes((tmp_path / "ok.png").read_bytes()[:40])
    with pytest.raises(cav.CavError, match="truncated|corrupt|bad size"):
        cav.load_texture_png(str(tmp_path / "cut.png"))
    with pytest.raises(cav.CavError, match="only PNG"):
        cav.load_texture_png(str(tmp_path / "x.jpg"))
    with pytest.raises(cav.CavError, match="cannot open"):
        cav.load_texture_png(str(tmp_path / "missing.png"))
