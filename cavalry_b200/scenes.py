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


def write_pbrt(path, room: dict, *, width=256, height=256, spp=16, max_depth=5, fov=40.0,
               eye=(0.0, 0.0, -3.8), look=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), integrator="path"):
    """Write a scene dict (as returned by mini_room) as a .pbrt file in the subset the
    reference's loader reads (SceneLoading/Lexing.cu, Parsing.cu): one trianglemesh Shape per
    mesh, matte materials, the light mesh as a diffuse AreaLightSource."""
    pos, idx = room["positions"], room["indices"]
    lines = [
        f"LookAt {_nums(eye)}  {_nums(look)}  {_nums(up)}",
        f'Camera "perspective" "float fov" [{_num(fov)}]',
        f'Film "image" "integer xresolution" [{width}] "integer yresolution" [{height}] "string filename" "out.png"',
        f'Sampler "halton" "integer pixelsamples" [{spp}]',
        f'Integrator "{integrator}" "integer maxdepth" [{max_depth}]',
        'PixelFilter "box"',
        "WorldBegin",
    ]
    L = room.get("light_radiance", (17.0, 12.0, 4.0))
    for name, first, count, mat in room["meshes"]:
        tris = idx[first:first + count]
        used = np.unique(tris)
        remap = {int(v): k for k, v in enumerate(used)}
        P = pos[used]
        I = np.vectorize(remap.get)(tris)
        lines.append("AttributeBegin")
        if name == "light":
            lines.append(f'AreaLightSource "diffuse" "rgb L" [{_nums(L)}]')
            lines.append('Material "matte" "rgb Kd" [0 0 0]')
        else:
            lines.append(f'Material "matte" "rgb Kd" [{_nums(mat)}]')
        lines.append(f'Shape "trianglemesh" "integer indices" [{_nums(I)}] "point P" [{_nums(P)}]')
        lines.append("AttributeEnd")
    lines.append("WorldEnd")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
