"""Seeded synthetic scenes and ray batches (numpy, host side).

The reference benchmarks on scenes that are not distributed with it; every workload
here is generated from a seed with the shapes, sizes and value distributions of the
configurations this project measures:

* ``soup``: N triangles whose anchor points are uniform in [0,1]^3; each vertex is
  the anchor plus an isotropic offset of length log-uniform in [1e-3, 1e-1].
* ``closest_rays``: origins uniform in [-0.1,1.1]^3, directions uniform on the sphere,
  tmax = +inf.
* ``shadow_rays``: origins as above, each aimed at a point uniform in [0,1]^3, with
  the distance to that point as the any-hit limit.
* ``mini_room``: the 34-triangle room (5 walls + 2 rotated boxes) plus its 2-triangle
  area light.
"""
from __future__ import annotations

import os

import numpy as np

RAY_DTYPE = np.float32


def _unit_vectors(rng: np.random.Generator, n: int) -> np.ndarray:
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def soup(n: int, seed: int = 2):
    """Triangle soup.  Returns (positions float32 [3n,3], indices int32 [n,3])."""
    rng = np.random.default_rng(seed)
    anchor = rng.uniform(0.0, 1.0, (n, 1, 3))
    dirs = _unit_vectors(rng, 3 * n).reshape(n, 3, 3)
    length = np.exp(rng.uniform(np.log(1e-3), np.log(1e-1), (n, 3, 1)))
    verts = (anchor + dirs * length).astype(np.float32).reshape(3 * n, 3)
    idx = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    return np.ascontiguousarray(verts), idx


def make_rays(origins: np.ndarray, dirs: np.ndarray, tmax=np.inf) -> np.ndarray:
    n = origins.shape[0]
    r = np.zeros((n, 8), dtype=RAY_DTYPE)
    r[:, 0:3] = origins
    r[:, 3] = 0.0
    r[:, 4:7] = dirs
    r[:, 7] = tmax
    return r


def closest_rays(m: int, seed: int = 20) -> np.ndarray:
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.1, 1.1, (m, 3))
    d = _unit_vectors(rng, m)
    return make_rays(o.astype(np.float32), d.astype(np.float32))


def shadow_rays(m: int, seed: int = 21):
    """Returns (rays float32 [m,8], limit float32 [m])."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.1, 1.1, (m, 3)).astype(np.float32)
    p = rng.uniform(0.0, 1.0, (m, 3)).astype(np.float32)
    v = (p - o).astype(np.float32)
    dist = np.sqrt((v.astype(np.float64) ** 2).sum(1)).astype(np.float32)
    dist = np.maximum(dist, np.float32(1e-6))
    d = (v / dist[:, None]).astype(np.float32)
    return make_rays(o, d), dist


def _box_triangles(size, angle_deg: float, centre):
    """12 triangles of an axis-aligned box of `size`, rotated about y, resting on y=-1."""
    sx, sy, sz = size
    c = np.array([[x, y, z] for x in (-sx / 2, sx / 2) for y in (0.0, sy) for z in (-sz / 2, sz / 2)])
    a = np.deg2rad(angle_deg)
    rot = np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]])
    v = c @ rot.T + np.array(centre)
    # corner index = 4*ix + 2*iy + iz
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    tris = []
    for q in quads:
        tris.append((q[0], q[1], q[2]))
        tris.append((q[0], q[2], q[3]))
    return v, np.array(tris)


def mini_room():
    """Config-1 room: 5 walls of a 2x2x2 box (10 tris), two boxes rotated +-18 deg (24 tris)
    and the 0.5x0.5 light quad under the ceiling (2 tris, facing down).

    Returns dict(positions [V,3] f32, indices [T,3] i32, mesh_ids [T] i32, meshes: list of
    (name, first_tri, count, material)).  Mesh order is walls (5 meshes), boxes (2), light (1).
    """
    verts = []
    tris = []
    mesh_ids = []
    meshes = []

    def add(v, t, name, mat):
        base = sum(len(x) for x in verts)
        mid = len(meshes)
        first = sum(len(x) for x in tris)
        verts.append(np.asarray(v, np.float64))
        tris.append(np.asarray(t) + base)
        mesh_ids.extend([mid] * len(t))
        meshes.append((name, first, len(t), mat))

    grey = (0.73, 0.73, 0.73)
    # floor y=-1, ceiling y=1, back z=1, left x=-1, right x=1 (camera looks down +z from z<-1)
    add([[-1, -1, -1], [1, -1, -1], [1, -1, 1], [-1, -1, 1]], [(0, 2, 1), (0, 3, 2)], "floor", grey)
    add([[-1, 1, -1], [1, 1, -1], [1, 1, 1], [-1, 1, 1]], [(0, 1, 2), (0, 2, 3)], "ceiling", grey)
    add([[-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], [(0, 2, 1), (0, 3, 2)], "back", grey)
    add([[-1, -1, -1], [-1, -1, 1], [-1, 1, 1], [-1, 1, -1]], [(0, 1, 2), (0, 2, 3)], "left", (0.63, 0.06, 0.05))
    add([[1, -1, -1], [1, -1, 1], [1, 1, 1], [1, 1, -1]], [(0, 2, 1), (0, 3, 2)], "right", (0.14, 0.45, 0.09))
    v, t = _box_triangles((0.6, 0.6, 0.6), 18.0, (0.35, -1.0, -0.2))
    add(v, t, "short_box", grey)
    v, t = _box_triangles((0.6, 1.2, 0.6), -18.0, (-0.35, -1.0, 0.3))
    add(v, t, "tall_box", grey)
    y = 0.999
    # wound so that the face normal points down into the room (the light emits on that side)
    add([[-0.25, y, -0.25], [0.25, y, -0.25], [0.25, y, 0.25], [-0.25, y, 0.25]], [(0, 1, 2), (0, 2, 3)], "light",
        (0.0, 0.0, 0.0))
    return {
        "positions": np.ascontiguousarray(np.concatenate(verts).astype(np.float32)),
        "indices": np.ascontiguousarray(np.concatenate(tris).astype(np.int32)),
        "mesh_ids": np.asarray(mesh_ids, np.int32),
        "meshes": meshes,
        "light_radiance": (17.0, 12.0, 4.0),
    }


def _num(x: float) -> str:
    """A number the reference's lexer accepts: characters [0-9.-e] only (no '+')."""
    t = "%.9g" % float(x)
    if "+" in t or "inf" in t or "nan" in t:
        t = ("%.6f" % float(x)).rstrip("0").rstrip(".")
    return t


def _nums(v) -> str:
    return " ".join(_num(x) for x in np.asarray(v).reshape(-1))


def _floats_text(a) -> str:
    """Exact float32 text without '+' (the reference's lexer reads [0-9.-e] only)."""
    a = np.asarray(a, np.float32).reshape(-1)
    if a.size and np.abs(a[np.isfinite(a)]).max(initial=0) >= 1e9:
        return _nums(a)
    return " ".join(["%.9g"] * a.size) % tuple(a.tolist())


def _material_line(mat) -> str:
    """pbrt Material directive of a scene material: a tuple is a matte Kd, a dict names
    "type" (matte, plastic, glass, mirror, metal, substrate) and its parameters; a metal's
    "eta" and "k" are rgb triples (complex index of refraction)."""
    if not isinstance(mat, dict):
        return f'Material "matte" "rgb Kd" [{_nums(mat)}]'
    t = mat["type"]
    parts = [f'Material "{t}"']
    for key, kind in (("Kd", "rgb"), ("Ks", "rgb"), ("Kr", "rgb"), ("Kt", "rgb"), ("roughness", "float"),
                      ("eta", "float"), ("k", "rgb")):
        if key in mat:
            if t == "metal" and key == "eta":
                parts.append(f'"rgb eta" [{_nums(mat[key])}]')
            elif t == "mirror" and key == "Kr":
                parts.append(f'"float Kr" [{_num(mat[key])}]')
            else:
                parts.append(f'"{kind} {key}" [{_nums(mat[key])}]')
    if "remaproughness" in mat:
        parts.append(f'"string remaproughness" "{"true" if mat["remaproughness"] else "false"}"')
    if mat.get("Kd_texture"):
        parts.append(f'"texture Kd" "{mat["Kd_texture"]}"')
    return " ".join(parts)


def write_pbrt(path, room: dict, *, width=256, height=256, spp=16, max_depth=5, fov=None, eye=None, look=None,
               up=None, integrator="path", ply: bool | None = None):
    """Write a scene dict (mini_room, sphere_scene) as a .pbrt file in the subset the
    reference's loader reads (SceneLoading/Lexing.cu, Parsing.cu): one trianglemesh Shape per
    mesh with its Material; light meshes (``room["lights"]`` = [(mesh, L)], or a mesh named
    "light" with ``room["light_radiance"]``) as diffuse AreaLightSources over a black matte.
    Camera arguments default to ``room["camera"]``, else the config-1 view.  Meshes listed in
    ``room["shapes"]`` are written as pbrt ``sphere`` / ``disk`` Shapes under a Translate;
    with `ply` (default ``room.get("write_ply")``), triangle meshes go to binary PLY files
    beside the .pbrt ("plymesh")."""
    if ply is None:
        ply = bool(room.get("write_ply", False))
    cam = dict(eye=(0.0, 0.0, -3.8), look=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), fov=40.0)
    cam.update(room.get("camera", {}))
    for k, v in (("eye", eye), ("look", look), ("up", up), ("fov", fov)):
        if v is not None:
            cam[k] = v
    pos, idx = room["positions"], room["indices"]
    lines = [
        f"LookAt {_nums(cam['eye'])}  {_nums(cam['look'])}  {_nums(cam['up'])}",
        f'Camera "perspective" "float fov" [{_num(cam["fov"])}]',
        f'Film "image" "integer xresolution" [{width}] "integer yresolution" [{height}] "string filename" "out.png"',
        f'Sampler "halton" "integer pixelsamples" [{spp}]',
        f'Integrator "{integrator}" "integer maxdepth" [{max_depth}]',
        'PixelFilter "box"',
        "WorldBegin",
    ]
    light_of = dict(room.get("lights", []))
    here = os.path.dirname(os.path.abspath(str(path)))
    stem = os.path.splitext(os.path.basename(str(path)))[0]
    env = room.get("environment")

    def image_file(name, img):  # 8-bit arrays as PNG, float arrays as OpenEXR (ZIP)
        if np.asarray(img).dtype.kind == "f":
            fn = f"{stem}_{name}.exr"
            write_exr(os.path.join(here, fn), img, compression=room.get("exr_compression", "zip"))
        else:
            fn = f"{stem}_{name}.png"
            write_png(os.path.join(here, fn), img)
        return fn

    if env is not None:  # first, so it is light 0
        line = f'LightSource "infinite" "rgb L" [{_nums(env["L"])}]'
        if env.get("map") is not None:
            line += f' "string mapname" "{image_file("env", env["map"])}"'
        lines.append(line)
    for t in room.get("textures", []):
        fn = image_file(t["name"], t["rgba"])
        lines.append(f'Texture "{t["name"]}" "spectrum" "imagemap" "string filename" "{fn}"')
    uvs = room.get("uvs")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
        for k, (name, first, count, mat) in enumerate(room["meshes"]):
            tris = idx[first:first + count]
            used, inv = np.unique(tris, return_inverse=True)
            I = inv.reshape(-1)
            P = pos[used]
            L = light_of.get(k)
            if L is None and name == "light":
                L = room.get("light_radiance", (17.0, 12.0, 4.0))
            out = ["AttributeBegin"]
            shape = room.get("shapes", {}).get(k)
            if shape is not None:
                out.append(f"Translate {_nums(shape['center'])}")
            if L is not None:
                out.append(f'AreaLightSource "diffuse" "rgb L" [{_nums(L)}]')
                out.append('Material "matte" "rgb Kd" [0 0 0]')
            else:
                out.append(_material_line(mat))
            if shape is not None and shape["type"] == "sphere":
                out.append(f'Shape "sphere" "float radius" [{_num(shape["radius"])}]')
            elif shape is not None:
                out.append(f'Shape "disk" "float radius" [{_num(shape["radius"])}] '
                           f'"float height" [{_num(shape.get("height", 0.0))}]')
            elif ply:
                fn = f"{os.path.splitext(os.path.basename(str(path)))[0]}_{k}.ply"
                _write_ply(os.path.join(os.path.dirname(os.path.abspath(str(path))), fn), P, I)
                out.append(f'Shape "plymesh" "string filename" "{fn}"')
            else:
                uv_text = "" if uvs is None else ' "float uv" [' + _floats_text(uvs[used]) + "]"
                out.append('Shape "trianglemesh" "integer indices" [' + " ".join(map(str, I.tolist())) + '] "point P" ['
                           + _floats_text(P) + "]" + uv_text)
            out.append("AttributeEnd")
            f.write("\n".join(out) + "\n")
        f.write("WorldEnd\n")


def _write_ply(path, P, I):
    """Binary little-endian PLY: float x/y/z and a uchar/int "vertex_indices" list per face."""
    P = np.ascontiguousarray(P, np.float32)
    I = np.asarray(I, np.int32).reshape(-1, 3)
    head = ("ply\nformat binary_little_endian 1.0\n"
            f"element vertex {len(P)}\nproperty float x\nproperty float y\nproperty float z\n"
            f"element face {len(I)}\nproperty list uchar int vertex_indices\nend_header\n")
    face = np.zeros(len(I), np.dtype([("n", "u1"), ("i", "<i4", (3,))]))
    face["n"] = 3
    face["i"] = I
    with open(path, "wb") as f:
        f.write(head.encode())
        f.write(P.tobytes())
        f.write(face.tobytes())


def write_png(path, rgba) -> None:
    """8-bit RGBA PNG (filter 0 on every row) of an [H, W, 4] uint8 array, top row first."""
    import struct
    import zlib

    a = np.ascontiguousarray(rgba, np.uint8)
    h, w = a.shape[:2]
    raw = b"".join(b"\x00" + a[y].tobytes() for y in range(h))

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0))
                + chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


EXR_COMPRESSION = {"none": 0, "rle": 1, "zips": 2, "zip": 3}


def _exr_pack(raw: bytes) -> bytes:
    """The OpenEXR ZIP/RLE pre-pass: bytes split into even and odd halves, then each byte
    stored as its difference to the previous one plus 128."""
    a = np.frombuffer(raw, np.uint8)
    t = np.concatenate([a[0::2], a[1::2]]).astype(np.int16)
    d = t.copy()
    d[1:] = (t[1:] - t[:-1] + 128) & 255
    return d.astype(np.uint8).tobytes()


def _exr_rle(data: bytes) -> bytes:
    out = bytearray()
    i, n = 0, len(data)
    while i < n:
        j = i
        while j + 1 < n and data[j + 1] == data[i] and j - i < 127:
            j += 1
        if j - i >= 2:  # a run of 3..128 equal bytes
            out += bytes([j - i]) + data[i:i + 1]
            i = j + 1
        else:  # literals up to the next run of 3 (at most 127)
            k = i
            while k < n and k - i < 127 and not (k + 2 < n and data[k] == data[k + 1] == data[k + 2]):
                k += 1
            out += bytes([(256 - (k - i)) & 255]) + data[i:k]
            i = k
    return bytes(out)


def write_exr(path, img, compression: str = "zip", channels: list[str] | None = None) -> None:
    """A single-part scanline OpenEXR file of an [H, W, C] (or [H, W]) float array, top row first
    (data window from (0, 0)): float16 arrays as HALF channels, float32 as FLOAT.  C = 1, 3 or
    4 with default names Y / R G B / R G B A; channels are stored in name order, as the format
    requires.  compression: "none", "rle", "zips" (one line per block) or "zip" (16 lines)."""
    import struct
    import zlib

    a = np.asarray(img)
    if a.ndim == 2:
        a = a[..., None]
    h, w, c = a.shape
    names = channels or {1: ["Y"], 3: ["R", "G", "B"], 4: ["R", "G", "B", "A"]}[c]
    half = a.dtype == np.float16
    a = a.astype(np.float16 if half else np.float32)
    order = sorted(range(c), key=lambda k: names[k])
    ptype = 1 if half else 2

    def attr(name, typ, value):
        return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(value)) + value

    chl = b"".join(names[k].encode() + b"\0" + struct.pack("<iB3xii", ptype, 0, 1, 1) for k in order) + b"\0"
    head = struct.pack("<ii", 20000630, 2)
    head += attr("channels", "chlist", chl)
    head += attr("compression", "compression", bytes([EXR_COMPRESSION[compression]]))
    head += attr("dataWindow", "box2i", struct.pack("<iiii", 0, 0, w - 1, h - 1))
    head += attr("displayWindow", "box2i", struct.pack("<iiii", 0, 0, w - 1, h - 1))
    head += attr("lineOrder", "lineOrder", b"\0")
    head += attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    head += attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
    head += attr("screenWindowWidth", "float", struct.pack("<f", 1.0)) + b"\0"
    lines = 16 if compression == "zip" else 1
    blocks = []
    for y0 in range(0, h, lines):
        raw = b"".join(a[y, :, k].tobytes() for y in range(y0, min(y0 + lines, h)) for k in order)
        if compression in ("zip", "zips"):
            packed = zlib.compress(_exr_pack(raw), 6)
        elif compression == "rle":
            packed = _exr_rle(_exr_pack(raw))
        else:
            packed = raw
        if len(packed) >= len(raw):  # stored as is when the codec does not pay
            packed = raw
        blocks.append(struct.pack("<ii", y0, len(packed)) + packed)
    offsets, off = [], len(head) + 8 * len(blocks)
    for b in blocks:
        offsets.append(off)
        off += len(b)
    with open(path, "wb") as f:
        f.write(head + struct.pack(f"<{len(offsets)}Q", *offsets) + b"".join(blocks))


def courtyard_scene(seed: int = 41, area_light: bool = False, hdr_sky: bool = False):
    """An open-topped courtyard under an environment map: a floor with a tiled checker
    texture ("texture Kd" on matte, uv 0..4), two walls, a textured plastic box, and sphere
    shapes of assorted materials; the environment ("infinite", a sky gradient with a bright
    sun patch) is the only light unless `area_light` adds a 1 x 1 quad.  The dict carries
    ``textures`` ([{"name", "rgba"}], PNG rows top-down), per-vertex ``uvs`` and
    ``environment = {"L", "map"}``."""
    rng = np.random.default_rng(seed)
    verts, tris, mesh_ids, meshes, nrms, uvs, shapes, lights = [], [], [], [], [], [], {}, []
    nv = nt = 0

    def add(v, t, name, mat, n=None, uv=None):
        nonlocal nv, nt
        mid = len(meshes)
        verts.append(np.asarray(v, np.float32))
        nrms.append(np.zeros_like(verts[-1]) if n is None else np.asarray(n, np.float32))
        uvs.append(np.zeros((len(v), 2), np.float32) if uv is None else np.asarray(uv, np.float32))
        tris.append(np.asarray(t, np.int64) + nv)
        mesh_ids.append(np.full(len(t), mid, np.int32))
        meshes.append((name, nt, len(t), mat))
        nv += len(v)
        nt += len(t)
        return mid

    # textures: an 8 x 8-cell checker (64 x 64 texels) and a 32 x 32 stripe pattern
    ij = np.add.outer(np.arange(64) // 8, np.arange(64) // 8) % 2
    checker = np.zeros((64, 64, 4), np.uint8)
    checker[..., :3] = np.where(ij[..., None] == 0, np.array([220, 210, 190]), np.array([60, 80, 120]))
    checker[..., 3] = 255
    stripes = np.zeros((32, 32, 4), np.uint8)
    stripes[..., :3] = np.where((np.arange(32) // 4 % 2)[None, :, None] == 0, np.array([200, 60, 40]),
                                np.array([240, 220, 120]))
    stripes[..., 3] = 255
    S = 3.0
    add([[-S, 0, -S], [S, 0, -S], [S, 0, S], [-S, 0, S]], [(0, 2, 1), (0, 3, 2)], "floor",
        {"type": "matte", "Kd": (0.9, 0.9, 0.9), "Kd_texture": "checker"},
        uv=[[0, 0], [4, 0], [4, 4], [0, 4]])
    add([[-S, 0, S], [S, 0, S], [S, 2, S], [-S, 2, S]], [(0, 2, 1), (0, 3, 2)], "back", (0.6, 0.6, 0.65))
    add([[-S, 0, -S], [-S, 0, S], [-S, 2, S], [-S, 2, -S]], [(0, 1, 2), (0, 2, 3)], "left", (0.5, 0.3, 0.25))
    bv, bt = _box_triangles((0.8, 0.8, 0.8), 20.0, (0.9, 0.0, 0.6))
    buv = np.tile(np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32), (len(bv) // 4 + 1, 1))[:len(bv)]
    add(bv, bt, "box", {"type": "plastic", "Kd": (0.5, 0.5, 0.5), "roughness": 0.1, "Kd_texture": "stripes"},
        uv=buv)
    kinds = [{"type": "glass", "eta": 1.5}, {"type": "metal", "roughness": 0.15}, (0.3, 0.7, 0.4)]
    for k, mat in enumerate(kinds):
        r = float(rng.uniform(0.3, 0.45))
        c = (float(-1.4 + 1.0 * k), r, float(rng.uniform(-1.2, -0.2)))
        unit, P, I = sphere_shape_mesh(r)
        mid = add(P + np.array(c, np.float32), I, f"sphere{k}", mat, n=unit)
        shapes[mid] = {"type": "sphere", "radius": r, "center": c}
    if area_light:
        y = 2.4
        mid = add([[-1.5, y, 0.5], [-0.5, y, 0.5], [-0.5, y, 1.5], [-1.5, y, 1.5]], [(0, 1, 2), (0, 2, 3)],
                  "light_quad", (0.0, 0.0, 0.0))
        lights.append((mid, (6.0, 5.0, 4.0)))
    # environment: sky gradient over the latitude (rows) with a warm sun patch
    H_, W_ = 32, 64
    sky = np.zeros((H_, W_, 4), np.uint8)
    t = np.linspace(0, 1, H_)[:, None]
    sky[..., 0] = (80 + 140 * t).astype(np.uint8)
    sky[..., 1] = (120 + 110 * t).astype(np.uint8)
    sky[..., 2] = (200 + 40 * t).astype(np.uint8)
    sky[10:14, 20:26, :3] = (255, 240, 200)
    sky[..., 3] = 255
    if hdr_sky:  # the same sky as an HDR map (HALF floats, written as OpenEXR), the sun 6x brighter
        hdr = np.zeros((H_, W_, 3), np.float32)
        hdr[..., 0] = 0.3 + 0.5 * t
        hdr[..., 1] = 0.45 + 0.4 * t
        hdr[..., 2] = 0.8 + 0.15 * t
        hdr[10:14, 20:26] = (6.0, 5.6, 4.7)
        sky = hdr.astype(np.float16)
    return {
        "positions": np.ascontiguousarray(np.concatenate(verts)),
        "normals": np.ascontiguousarray(np.concatenate(nrms)),
        "uvs": np.ascontiguousarray(np.concatenate(uvs)),
        "indices": np.ascontiguousarray(np.concatenate(tris).astype(np.int32)),
        "mesh_ids": np.concatenate(mesh_ids),
        "meshes": meshes,
        "lights": lights,
        "shapes": shapes,
        "textures": [{"name": "checker", "rgba": checker}, {"name": "stripes", "rgba": stripes}],
        "environment": {"L": (1.5, 1.5, 1.5), "map": sky},
        "camera": {"eye": (0.0, 1.6, -4.5), "look": (0.0, 0.5, 0.0), "up": (0.0, 1.0, 0.0), "fov": 55.0},
    }


def sphere_shape_mesh(radius: float):
    """The mesh the reference makes for a ``Shape "sphere"`` (ShapeMesh/Sphere.cu:3-94): an
    octahedron split four times, every split pushing its three midpoints (normalised) as new
    vertices, 2046 vertices and 2048 triangles.  Returns (unit positions = normals [V,3],
    positions * radius [V,3], indices [T,3]) in object space, float32."""
    p = [np.array(v, np.float32) for v in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))]
    cur = [(0, 2, 4), (0, 2, 5), (0, 3, 4), (0, 3, 5), (1, 2, 4), (1, 2, 5), (1, 3, 4), (1, 3, 5)]

    def nrm(v):
        inv = np.float32(1.0 / np.sqrt(np.float64(np.float32(v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])))
        return (v * inv).astype(np.float32)

    for _ in range(4):
        nxt = []
        for i0, i1, i2 in cur:
            p.append(nrm((p[i0] + p[i1]) * np.float32(0.5)))
            i01 = len(p) - 1
            p.append(nrm((p[i0] + p[i2]) * np.float32(0.5)))
            i02 = len(p) - 1
            p.append(nrm((p[i1] + p[i2]) * np.float32(0.5)))
            i12 = len(p) - 1
            nxt += [(i01, i02, i12), (i0, i01, i02), (i1, i01, i12), (i2, i02, i12)]
        cur = nxt
    unit = np.array(p, np.float32)
    return unit, (unit * np.float32(radius)).astype(np.float32), np.array(cur, np.int32)


def disk_shape_mesh(radius: float, height: float = 0.0):
    """The mesh of a ``Shape "disk"`` (ShapeMesh/Disk.cu:4-50): 360 rim vertices at
    (sin t r, cos t r, height), the centre last, triangles (s+1, s, centre)."""
    th = (2.0 * np.pi * np.arange(360, dtype=np.float32).astype(np.float64) / 360.0).astype(np.float32)
    rim = np.stack([np.sin(th) * np.float32(radius), np.cos(th) * np.float32(radius),
                    np.full(360, height, np.float32)], 1).astype(np.float32)
    P = np.concatenate([rim, np.array([[0, 0, height]], np.float32)])
    s = np.arange(360)
    return P, np.stack([(s + 1) % 360, s, np.full(360, 360)], 1).astype(np.int32)


def shapes_scene(seed: int = 31, quad_light: bool = False):
    """A 4 x 3 x 4 room (matte walls) holding tessellated ``sphere`` shapes of assorted
    materials, a matte ``disk`` on the back wall and a sphere area light under the ceiling
    (plus a 1 x 1 quad light when `quad_light`).  The scene dict carries
    ``shapes = {mesh: {"type", "radius", "center", ("height")}}`` (written as pbrt Shapes with
    Translate) and per-vertex ``normals`` (the spheres'; zero elsewhere)."""
    rng = np.random.default_rng(seed)
    verts, tris, mesh_ids, meshes, lights, nrms, shapes = [], [], [], [], [], [], {}
    nv = nt = 0

    def add(v, t, name, mat, n=None):
        nonlocal nv, nt
        mid = len(meshes)
        verts.append(np.asarray(v, np.float32))
        nrms.append(np.zeros_like(verts[-1]) if n is None else np.asarray(n, np.float32))
        tris.append(np.asarray(t, np.int64) + nv)
        mesh_ids.append(np.full(len(t), mid, np.int32))
        meshes.append((name, nt, len(t), mat))
        nv += len(v)
        nt += len(t)
        return mid

    W, H, D = 4.0, 3.0, 4.0
    x0, x1, z0, z1 = -W / 2, W / 2, -D / 2, D / 2
    grey = (0.7, 0.7, 0.7)
    add([[x0, 0, z0], [x1, 0, z0], [x1, 0, z1], [x0, 0, z1]], [(0, 2, 1), (0, 3, 2)], "floor", grey)
    add([[x0, H, z0], [x1, H, z0], [x1, H, z1], [x0, H, z1]], [(0, 1, 2), (0, 2, 3)], "ceiling", grey)
    add([[x0, 0, z1], [x1, 0, z1], [x1, H, z1], [x0, H, z1]], [(0, 2, 1), (0, 3, 2)], "back", grey)
    add([[x0, 0, z0], [x0, 0, z1], [x0, H, z1], [x0, H, z0]], [(0, 1, 2), (0, 2, 3)], "left", (0.6, 0.15, 0.1))
    add([[x1, 0, z0], [x1, 0, z1], [x1, H, z1], [x1, H, z0]], [(0, 2, 1), (0, 3, 2)], "right", (0.15, 0.5, 0.2))
    kinds = [{"type": "matte", "Kd": (0.8, 0.5, 0.2)}, {"type": "plastic", "Kd": (0.2, 0.3, 0.7), "roughness": 0.1},
             {"type": "glass", "eta": 1.5}, {"type": "metal", "roughness": 0.2},
             {"type": "substrate", "Kd": (0.5, 0.6, 0.3), "Ks": (0.3, 0.3, 0.3), "roughness": 0.15}]
    for k, mat in enumerate(kinds):
        r = float(rng.uniform(0.25, 0.45))
        c = (float(-1.4 + 0.7 * k), r, float(rng.uniform(-0.6, 0.8)))
        unit, P, I = sphere_shape_mesh(r)
        mid = add(P + np.array(c, np.float32), I, f"sphere{k}", mat, n=unit)
        shapes[mid] = {"type": "sphere", "radius": r, "center": c}
    dP, dI = disk_shape_mesh(0.6, 0.0)
    dc = (0.8, 1.6, z1 - 0.01)
    mid = add(dP + np.array(dc, np.float32), dI, "disk", (0.75, 0.75, 0.3))
    shapes[mid] = {"type": "disk", "radius": 0.6, "height": 0.0, "center": dc}
    lr = 0.25
    lc = (-0.3, H - 0.6, 0.2)
    unit, P, I = sphere_shape_mesh(lr)
    mid = add(P + np.array(lc, np.float32), I, "light_sphere", (0.0, 0.0, 0.0), n=unit)
    shapes[mid] = {"type": "sphere", "radius": lr, "center": lc}
    lights.append((mid, (14.0, 12.0, 9.0)))
    if quad_light:
        y = H - 0.01
        mid = add([[0.4, y, -0.9], [1.4, y, -0.9], [1.4, y, 0.1], [0.4, y, 0.1]], [(0, 1, 2), (0, 2, 3)],
                  "light_quad", (0.0, 0.0, 0.0))
        lights.append((mid, (4.0, 4.0, 6.0)))
    return {
        "positions": np.ascontiguousarray(np.concatenate(verts)),
        "normals": np.ascontiguousarray(np.concatenate(nrms)),
        "indices": np.ascontiguousarray(np.concatenate(tris).astype(np.int32)),
        "mesh_ids": np.concatenate(mesh_ids),
        "meshes": meshes,
        "lights": lights,
        "shapes": shapes,
        "camera": {"eye": (0.0, 1.5, z0 + 0.1), "look": (0.0, 1.1, 0.0), "up": (0.0, 1.0, 0.0), "fov": 65.0},
    }


_ICO_CACHE: dict = {}


def icosphere(level: int):
    """Unit icosphere: the icosahedron with each triangle split into 4, `level` times, new
    vertices pushed onto the sphere (20 * 4**level triangles).  Outward winding."""
    if level in _ICO_CACHE:
        return _ICO_CACHE[level]
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        nv = len(v)
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.minimum(e[:, 0], e[:, 1]) * nv + np.maximum(e[:, 0], e[:, 1])
        uk, inv = np.unique(key, return_inverse=True)
        a, b = uk // nv, uk % nv
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = (inv + nv).reshape(3, -1)
        m01, m12, m20 = m[0], m[1], m[2]
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
        v = np.concatenate([v, mid])
    # outward winding: cross(e1, e2) along the centroid
    c = v[f].mean(1)
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    flip = (n * c).sum(1) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    _ICO_CACHE[level] = (v, f)
    return v, f


def sphere_scene(n_spheres: int = 64, level: int = 6, seed: int = 3, room=(20.0, 10.0, 20.0), n_lights: int = 3,
                 materials=("matte", "plastic", "glass", "mirror")):
    """Config-3 scene: `n_spheres` icospheres (20 * 4**level triangles each; 64 x level 6 =
    5,242,880), radii log-uniform in [0.05, 0.5], centres from 4 Gaussian clusters (sigma 1.5)
    clipped into a W x H x D room (floor y = 0, centred in x and z); each sphere's material
    uniform over `materials` (matte; plastic roughness 0.1; glass eta 1.5; mirror; metal =
    copper roughness 0.2; gold = metal with gold's complex index, roughness 0.05; substrate
    Ks 0.3 roughness 0.15; roughglass = glass roughness 0.1) with albedo uniform in [0.1, 0.9]; `n_lights` 2 x 2 emissive quads under the ceiling facing down with
    radiance uniform in [10, 30].  Room walls are matte 0.73 grey, outward-facing normals in.
    Returns the scene dict of mini_room plus "lights" and "camera"."""
    rng = np.random.default_rng(seed)
    W, H, D = room
    verts, tris, mesh_ids, meshes, lights = [], [], [], [], []
    nv = 0
    nt = 0

    def add(v, t, name, mat):
        nonlocal nv, nt
        mid = len(meshes)
        verts.append(np.asarray(v, np.float32))
        tris.append(np.asarray(t, np.int64) + nv)
        mesh_ids.append(np.full(len(t), mid, np.int32))
        meshes.append((name, nt, len(t), mat))
        nv += len(v)
        nt += len(t)
        return mid

    x0, x1, z0, z1 = -W / 2, W / 2, -D / 2, D / 2
    grey = (0.73, 0.73, 0.73)
    add([[x0, 0, z0], [x1, 0, z0], [x1, 0, z1], [x0, 0, z1]], [(0, 2, 1), (0, 3, 2)], "floor", grey)
    add([[x0, H, z0], [x1, H, z0], [x1, H, z1], [x0, H, z1]], [(0, 1, 2), (0, 2, 3)], "ceiling", grey)
    add([[x0, 0, z1], [x1, 0, z1], [x1, H, z1], [x0, H, z1]], [(0, 2, 1), (0, 3, 2)], "back", grey)
    add([[x0, 0, z0], [x1, 0, z0], [x1, H, z0], [x0, H, z0]], [(0, 1, 2), (0, 2, 3)], "front", grey)
    add([[x0, 0, z0], [x0, 0, z1], [x0, H, z1], [x0, H, z0]], [(0, 1, 2), (0, 2, 3)], "left", grey)
    add([[x1, 0, z0], [x1, 0, z1], [x1, H, z1], [x1, H, z0]], [(0, 2, 1), (0, 3, 2)], "right", grey)
    uv, uf = icosphere(level)
    centres_c = np.stack([rng.uniform(x0 + 3, x1 - 3, 4), rng.uniform(2, H - 3, 4), rng.uniform(z0 + 3, z1 - 3, 4)], 1)
    for k in range(n_spheres):
        r = float(np.exp(rng.uniform(np.log(0.05), np.log(0.5))))
        c = centres_c[rng.integers(0, 4)] + rng.normal(0, 1.5, 3)
        c = np.clip(c, [x0 + r, r, z0 + r], [x1 - r, H - 1 - r, z1 - r])
        kind = materials[rng.integers(0, len(materials))]
        alb = tuple(float(a) for a in rng.uniform(0.1, 0.9, 3))
        if kind == "matte":
            mat = {"type": "matte", "Kd": alb}
        elif kind == "plastic":
            mat = {"type": "plastic", "Kd": alb, "roughness": 0.1}
        elif kind == "glass":
            mat = {"type": "glass", "eta": 1.5}
        elif kind == "metal":
            mat = {"type": "metal", "roughness": 0.2}
        elif kind == "gold":
            mat = {"type": "metal", "eta": (0.143, 0.374, 1.442), "k": (3.983, 2.385, 1.603), "roughness": 0.05}
        elif kind == "substrate":
            mat = {"type": "substrate", "Kd": alb, "Ks": (0.3, 0.3, 0.3), "roughness": 0.15}
        elif kind == "roughglass":
            mat = {"type": "glass", "eta": 1.5, "roughness": 0.1}
        else:
            mat = {"type": "mirror"}
        add(uv * r + c, uf, f"sphere{k}", mat)
    for k in range(n_lights):
        cx, cz = rng.uniform(x0 + 2, x1 - 2), rng.uniform(z0 + 2, z1 - 2)
        y = H - 0.01
        L = tuple(float(a) for a in rng.uniform(10, 30, 3))
        mid = add([[cx - 1, y, cz - 1], [cx + 1, y, cz - 1], [cx + 1, y, cz + 1], [cx - 1, y, cz + 1]],
                  [(0, 1, 2), (0, 2, 3)], f"light{k}", (0.0, 0.0, 0.0))
        lights.append((mid, L))
    return {
        "positions": np.ascontiguousarray(np.concatenate(verts)),
        "indices": np.ascontiguousarray(np.concatenate(tris).astype(np.int32)),
        "mesh_ids": np.concatenate(mesh_ids),
        "meshes": meshes,
        "lights": lights,
        "camera": {"eye": (0.0, H * 0.45, z0 + 0.5), "look": (0.0, H * 0.35, 0.0), "up": (0.0, 1.0, 0.0),
                   "fov": 60.0},
    }


def soup_scene(n: int, seed: int):
    """A config-2-type soup (`soup(n, seed)`, matte grey) under a 0.6 x 0.6 area light
    (radiance 20) above the unit cube, seen from the front: the scenes of the served job
    stream."""
    pos, idx = soup(n, seed=seed)
    light_v = np.array([[0.2, 1.5, 0.2], [0.8, 1.5, 0.2], [0.8, 1.5, 0.8], [0.2, 1.5, 0.8]], np.float32)
    positions = np.concatenate([pos.astype(np.float32), light_v])
    base = len(pos)
    indices = np.concatenate([idx.astype(np.int32), np.array([[base, base + 1, base + 2], [base, base + 2, base + 3]],
                                                               np.int32)])
    mesh_ids = np.concatenate([np.zeros(len(idx), np.int32), np.ones(2, np.int32)])
    return {
        "positions": np.ascontiguousarray(positions),
        "indices": np.ascontiguousarray(indices),
        "mesh_ids": mesh_ids,
        "meshes": [("soup", 0, len(idx), (0.6, 0.6, 0.6)), ("light0", len(idx), 2, (0.0, 0.0, 0.0))],
        "lights": [(1, (20.0, 20.0, 20.0))],
        "camera": {"eye": (0.5, 0.6, -1.6), "look": (0.5, 0.5, 0.5), "up": (0.0, 1.0, 0.0), "fov": 45.0},
    }


def aperture_scene(n_spheres: int = 24, level: int = 3, seed: int = 5, room=(8.0, 4.0, 8.0), aperture: float = 0.3):
    """Config-5 layout: a closed room split by a wall with one square aperture (side
    `aperture`, centred at mid height); the only light is a 2 x 2 quad under the ceiling of
    the far side, so the near side, where the camera and the spheres are, is lit only
    through the aperture (strong indirect light).  Spheres are 80 % plastic at roughness
    0.05 (remapped) and 20 % matte."""
    rng = np.random.default_rng(seed)
    W, H, D = room
    verts, tris, mesh_ids, meshes, lights = [], [], [], [], []
    nv = nt = 0

    def add(v, t, name, mat):
        nonlocal nv, nt
        mid = len(meshes)
        verts.append(np.asarray(v, np.float32))
        tris.append(np.asarray(t, np.int64) + nv)
        mesh_ids.append(np.full(len(t), mid, np.int32))
        meshes.append((name, nt, len(t), mat))
        nv += len(v)
        nt += len(t)
        return mid

    def rect_z(xa, xb, ya, yb, z):  # a rectangle in the plane z = const
        return [[xa, ya, z], [xb, ya, z], [xb, yb, z], [xa, yb, z]], [(0, 1, 2), (0, 2, 3)]

    x0, x1, z0, z1 = -W / 2, W / 2, -D / 2, D / 2
    grey = (0.73, 0.73, 0.73)
    add([[x0, 0, z0], [x1, 0, z0], [x1, 0, z1], [x0, 0, z1]], [(0, 2, 1), (0, 3, 2)], "floor", grey)
    add([[x0, H, z0], [x1, H, z0], [x1, H, z1], [x0, H, z1]], [(0, 1, 2), (0, 2, 3)], "ceiling", grey)
    add(*rect_z(x0, x1, 0, H, z1), "back", grey)
    add(*rect_z(x0, x1, 0, H, z0), "front", grey)
    add([[x0, 0, z0], [x0, 0, z1], [x0, H, z1], [x0, H, z0]], [(0, 1, 2), (0, 2, 3)], "left", (0.63, 0.06, 0.05))
    add([[x1, 0, z0], [x1, 0, z1], [x1, H, z1], [x1, H, z0]], [(0, 2, 1), (0, 3, 2)], "right", (0.14, 0.45, 0.09))
    # the dividing wall at z = zw with the aperture around (0, H/2)
    zw, a, yc = z1 - 2.5, aperture / 2, H / 2
    parts = [rect_z(x0, -a, 0, H, zw), rect_z(a, x1, 0, H, zw), rect_z(-a, a, 0, yc - a, zw), rect_z(-a, a, yc + a, H, zw)]
    wv = np.concatenate([np.asarray(v) for v, _ in parts])
    wt = np.concatenate([np.asarray(t) + 4 * k for k, (_, t) in enumerate(parts)])
    add(wv, wt, "divider", (0.5, 0.5, 0.5))
    uv, uf = icosphere(level)
    for k in range(n_spheres):
        r = float(rng.uniform(0.2, 0.6))
        c = np.array([rng.uniform(x0 + r + 0.2, x1 - r - 0.2), r, rng.uniform(z0 + 2.0, zw - r - 0.3)])
        alb = tuple(float(v) for v in rng.uniform(0.1, 0.9, 3))
        if rng.random() < 0.8:
            mat = {"type": "plastic", "Kd": alb, "roughness": 0.05, "remaproughness": True}
        else:
            mat = {"type": "matte", "Kd": alb}
        add(uv * r + c, uf, f"sphere{k}", mat)
    lz = (zw + z1) / 2
    mid = add([[-1, H - 0.01, lz - 1], [1, H - 0.01, lz - 1], [1, H - 0.01, lz + 1], [-1, H - 0.01, lz + 1]],
              [(0, 1, 2), (0, 2, 3)], "light0", (0.0, 0.0, 0.0))
    lights.append((mid, (50.0, 50.0, 50.0)))
    return {
        "positions": np.ascontiguousarray(np.concatenate(verts)),
        "indices": np.ascontiguousarray(np.concatenate(tris).astype(np.int32)),
        "mesh_ids": np.concatenate(mesh_ids),
        "meshes": meshes,
        "lights": lights,
        "camera": {"eye": (0.0, 1.8, z0 + 0.3), "look": (0.0, 1.2, zw), "up": (0.0, 1.0, 0.0), "fov": 70.0},
    }
