"""Test infrastructure: ctypes bindings of the C oracle (``libcavoracle.so``) and of the
reference-build harness (``_ref/libcavref.so``).

Node arrays use ``ONODE_DTYPE``, the field order of the reference's BVHRestructureNode
(BVH/BVHNode.h:50-68): box, prim range, children, parent, leaf flag, SAH area and cost.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import build as _build

ONODE_DTYPE = np.dtype(
    [("bmin", "<f4", (3,)), ("bmax", "<f4", (3,)), ("begin", "<i4"), ("end", "<i4"), ("left", "<i4"),
     ("right", "<i4"), ("parent", "<i4"), ("is_leaf", "<i4"), ("area", "<f4"), ("cost", "<f4")]
)
assert ONODE_DTYPE.itemsize == 56

_orc = None
_ref = None


def _c(a):
    return None if a is None else a.ctypes.data


def oracle_lib() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        path = _build.ORACLE_LIB
        if not path.exists():
            path = _build.build_oracle()
        L = ctypes.CDLL(str(path))
        P, I64 = ctypes.c_void_p, ctypes.c_int64
        L.orc_build.argtypes = [P, P, I64, P, P, ctypes.c_int, P, P, P, P, P, P]
        L.orc_build.restype = ctypes.c_int
        L.orc_trace_closest.argtypes = [P, P, P, P, I64, P, P, P, P]
        L.orc_trace_any.argtypes = [P, P, P, P, P, P, P, I64, P]
        L.orc_treelet_rounds.argtypes = [P, I64, ctypes.c_int]
        L.orc_morton.argtypes = [P, I64, P, P]
        L.orc_leaf_boxes.argtypes = [P, P, I64, P]
        L.orc_scene_bounds.argtypes = [P, I64, P]
        L.orc_num_threads.restype = ctypes.c_int
        _orc = L
    return _orc


def build(pos: np.ndarray, idx: np.ndarray, bounds=None, codes=None, rounds: int = 0) -> dict:
    """Oracle LBVH build.  codes: optional unsorted Morton codes to use instead of computing them."""
    pos = np.ascontiguousarray(pos, np.float32)
    idx = np.ascontiguousarray(idx, np.int32)
    n = idx.shape[0]
    out = {
        "codes": np.zeros(n, np.uint64),
        "sorted": np.zeros(n, np.uint64),
        "perm": np.zeros(n, np.int32),
        "merged": np.zeros(2 * n - 1, ONODE_DTYPE),
        "final": np.zeros(2 * n - 1, ONODE_DTYPE),
        "bounds": np.zeros(6, np.float32),
    }
    b = None if bounds is None else np.ascontiguousarray(bounds, np.float32)
    c = None if codes is None else np.ascontiguousarray(codes, np.uint64)
    st = oracle_lib().orc_build(_c(pos), _c(idx), n, _c(b), _c(c), int(rounds), _c(out["codes"]), _c(out["sorted"]),
                                _c(out["perm"]), _c(out["merged"]), _c(out["final"]), _c(out["bounds"]))
    if st != 0:
        raise ValueError(f"orc_build failed ({st})")
    return out


def morton(pos, idx, bounds) -> np.ndarray:
    n = idx.shape[0]
    box = np.zeros((n, 6), np.float32)
    pos = np.ascontiguousarray(pos, np.float32)
    idx = np.ascontiguousarray(idx, np.int32)
    bounds = np.ascontiguousarray(bounds, np.float32)
    oracle_lib().orc_leaf_boxes(_c(pos), _c(idx), n, _c(box))
    codes = np.zeros(n, np.uint64)
    oracle_lib().orc_morton(_c(box), n, _c(bounds), _c(codes))
    return codes


def treelet_rounds(nodes: np.ndarray, rounds: int) -> np.ndarray:
    out = np.ascontiguousarray(nodes.copy())
    oracle_lib().orc_treelet_rounds(_c(out), out.shape[0], int(rounds))
    return out


def rays6(rays8: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.concatenate([rays8[:, 0:3], rays8[:, 4:7]], axis=1).astype(np.float32))


# Every array handed to C is bound to a local name first: a temporary passed as
# `_c(np.ascontiguousarray(...))` would be freed before the foreign call reads it.
def trace_closest(nodes, pos, idx, rays8):
    n = rays8.shape[0]
    r6 = rays6(rays8)
    nodes = np.ascontiguousarray(nodes)
    pos = np.ascontiguousarray(pos, np.float32)
    idx = np.ascontiguousarray(idx, np.int32)
    prim = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    oracle_lib().orc_trace_closest(_c(nodes), _c(pos), _c(idx), _c(r6), n, _c(prim), _c(t), _c(u), _c(v))
    return prim, t, u, v


def trace_any(nodes, pos, idx, rays8, limit=None, excl=None, mesh_ids=None):
    n = rays8.shape[0]
    r6 = rays6(rays8)
    nodes = np.ascontiguousarray(nodes)
    pos = np.ascontiguousarray(pos, np.float32)
    idx = np.ascontiguousarray(idx, np.int32)
    occ = np.zeros(n, np.uint8)
    lim = None if limit is None else np.ascontiguousarray(limit, np.float32)
    ex = None if excl is None else np.ascontiguousarray(excl, np.int32)
    mi = None if mesh_ids is None else np.ascontiguousarray(mesh_ids, np.int32)
    oracle_lib().orc_trace_any(_c(nodes), _c(pos), _c(idx), _c(mi), _c(r6), _c(lim), _c(ex), n, _c(occ))
    return occ


def num_threads() -> int:
    return int(oracle_lib().orc_num_threads())


# ----------------------------------------------------------------- reference harness
def ref_available() -> bool:
    return _build.REF_LIB.exists()


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not _build.REF_LIB.exists():
            raise FileNotFoundError(f"{_build.REF_LIB} not built (needs the reference sources)")
        L = ctypes.CDLL(str(_build.REF_LIB))
        P, I = ctypes.c_void_p, ctypes.c_int
        L.ref_build.argtypes = [P, I, P, P, I, I, P, I, P, P, P, P, P, P, P, ctypes.POINTER(P)]
        L.ref_build.restype = I
        L.ref_export_nodes.argtypes = [P, P]
        L.ref_tree_depth.argtypes = [P]
        L.ref_load_nodes.argtypes = [P, P, I]
        L.ref_trace_closest.argtypes = [P, P, I, I, P, P, P]
        L.ref_trace_any.argtypes = [P, P, P, P, I, I, P, P]
        L.ref_free.argtypes = [P]
        _ref = L
    return _ref


REF_NODE_OUT = np.dtype(
    [("bmin", "<f4", (3,)), ("bmax", "<f4", (3,)), ("begin", "<i4"), ("end", "<i4"), ("left", "<i4"),
     ("right", "<i4"), ("is_leaf", "<i4")]
)


class RefScene:
    """The reference's own BVH build (BVH/BVH.cu:317-370, replayed stage by stage) on the GPU."""

    def __init__(self, pos, idx, mesh_ids=None, bounds=None, rounds=0, id_mode=1, dump=True):
        L = ref_lib()
        pos = np.ascontiguousarray(pos, np.float32)
        idx = np.ascontiguousarray(idx, np.int32)
        n = idx.shape[0]
        mesh = np.zeros(n, np.int32) if mesh_ids is None else np.ascontiguousarray(mesh_ids, np.int32)
        self.n = n
        self.codes = np.zeros(n, np.uint64) if dump else None
        self.sorted = np.zeros(n, np.uint64) if dump else None
        self.perm = np.zeros(n, np.int32) if dump else None
        self.merged = np.zeros(2 * n - 1, ONODE_DTYPE) if dump else None
        self.final_r = np.zeros(2 * n - 1, ONODE_DTYPE) if dump else None
        self.bounds = np.zeros(6, np.float32)
        self.stage_ms = np.zeros(8, np.float32)
        b = None if bounds is None else np.ascontiguousarray(bounds, np.float32)
        h = ctypes.c_void_p()
        st = L.ref_build(_c(pos), pos.shape[0], _c(idx), _c(mesh), n, int(id_mode), _c(b), int(rounds),
                         _c(self.codes), _c(self.sorted), _c(self.perm), _c(self.merged), _c(self.final_r),
                         _c(self.bounds), _c(self.stage_ms), ctypes.byref(h))
        if st != 0:
            raise RuntimeError(f"ref_build failed ({st})")
        self.h = h
        self.depth = L.ref_tree_depth(h)

    def nodes(self) -> np.ndarray:
        out = np.zeros(2 * self.n - 1, REF_NODE_OUT)
        ref_lib().ref_export_nodes(self.h, _c(out))
        return out

    def load_nodes(self, nodes):
        """Run the reference's traversal on `nodes` (any dtype with box, prim range, children, leaf flag)."""
        out = np.zeros(len(nodes), REF_NODE_OUT)
        for f in ("bmin", "bmax", "left", "right", "is_leaf"):
            out[f] = nodes[f]
        out["begin"] = nodes["begin"] if "begin" in nodes.dtype.names else nodes["prim_begin"]
        out["end"] = nodes["end"] if "end" in nodes.dtype.names else nodes["prim_end"]
        st = ref_lib().ref_load_nodes(self.h, _c(out), len(out))
        if st != 0:
            raise RuntimeError(f"ref_load_nodes failed ({st})")
        self.depth = ref_lib().ref_tree_depth(self.h)

    def trace_closest(self, rays8, reps=1):
        n = rays8.shape[0]
        prim = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        ms = np.zeros(1, np.float32)
        r6 = rays6(rays8)
        st = ref_lib().ref_trace_closest(self.h, _c(r6), n, int(reps), _c(prim), _c(t), _c(ms))
        if st != 0:
            raise RuntimeError(f"ref_trace_closest refused or failed ({st}); depth={self.depth}")
        return prim, t, float(ms[0])

    def trace_any(self, rays8, limit=None, excl=None, reps=1):
        n = rays8.shape[0]
        occ = np.zeros(n, np.uint8)
        ms = np.zeros(1, np.float32)
        lim = None if limit is None else np.ascontiguousarray(limit, np.float32)
        ex = None if excl is None else np.ascontiguousarray(excl, np.int32)
        r6 = rays6(rays8)
        st = ref_lib().ref_trace_any(self.h, _c(r6), _c(lim), _c(ex), n, int(reps), _c(occ), _c(ms))
        if st != 0:
            raise RuntimeError(f"ref_trace_any refused or failed ({st}); depth={self.depth}")
        return occ, float(ms[0])

    def free(self):
        if self.h:
            ref_lib().ref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------- path-tracing oracle
OMESH_DTYPE = np.dtype([("first_tri", "<i4"), ("tri_count", "<i4"), ("has_normals", "<i4"), ("reverse", "<i4"),
                        ("material", "<i4"), ("light", "<i4"), ("area", "<f4"), ("shape", "<i4"),
                        ("sphere", "<f4", (4,))])
OMAT_DTYPE = np.dtype([("type", "<i4"), ("kd", "<f4", (3,)), ("ks", "<f4", (3,)), ("kr", "<f4", (3,)),
                       ("kt", "<f4", (3,)), ("alpha_u", "<f4"), ("alpha_v", "<f4"), ("eta", "<f4"),
                       ("mirror_kr", "<f4"), ("f0", "<f4", (3,)), ("has_f0", "<i4"), ("kd_tex", "<i4")])
OLIGHT_DTYPE = np.dtype([("L", "<f4", (3,)), ("mesh", "<i4"), ("kind", "<i4"), ("tex", "<i4"), ("w2l", "<f4", (9,))])
OTEX_DTYPE = np.dtype([("width", "<i4"), ("height", "<i4"), ("rgba", "<u8"), ("rgbaf", "<u8")])
MATERIAL_TYPES = {"matte": 0, "mirror": 1, "substrate": 2, "metal": 3, "glass": 4, "plastic": 5}


def _pt_lib():
    L = oracle_lib()
    if not hasattr(L, "_pt_ready"):
        P, I, I64, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float
        L.orc_render_path.argtypes = [P, P, P, P, P, P, I, P, P, I, P, F, I, I, I, I, F, F, I64, I64, P, P, I, P, P, I]
        L.orc_render_path.restype = I
        L.orc_roughness_to_alpha.argtypes = [F]
        L.orc_roughness_to_alpha.restype = F
        L.orc_halton_tables.argtypes = [P, P, P]
        L.orc_halton_tables.restype = I64
        L.orc_load_gamma_table.argtypes = [P]
        L.orc_load_gamma_table.restype = None
        L._pt_ready = True
    return L


def roughness_to_alpha(r: float) -> float:
    return float(_pt_lib().orc_roughness_to_alpha(float(r)))


def load_gamma_table() -> np.ndarray:
    """uint8 [256]: a .png colour byte after the load-time inverse sRGB curve."""
    out = np.zeros(256, np.uint8)
    _pt_lib().orc_load_gamma_table(out.ctypes.data)
    return out


def material_record(mat, texture_index: dict | None = None) -> np.void:
    """A material as the reference's parser builds it (Materials/*.h createFromParams):
    a tuple is a matte Kd; a dict names "type" and the pbrt parameters ("Kd_texture": the
    name of a scene texture)."""
    m = np.zeros((), OMAT_DTYPE)
    m["kd_tex"] = -1
    if isinstance(mat, dict) and mat.get("Kd_texture") is not None:
        m["kd_tex"] = (texture_index or {})[mat["Kd_texture"]]
    if not isinstance(mat, dict):
        mat = {"type": "matte", "Kd": mat}
    t = mat["type"]
    m["type"] = MATERIAL_TYPES[t]
    m["eta"] = 1.5
    m["mirror_kr"] = 0.9
    if t == "matte":
        m["kd"] = mat.get("Kd", (1, 1, 1))
    elif t == "plastic":
        m["kd"] = mat.get("Kd", (0.25, 0.25, 0.25))
        m["ks"] = mat.get("Ks", (0.25, 0.25, 0.25))
        r = float(mat.get("roughness", 0.1))
        a = roughness_to_alpha(r) if mat.get("remaproughness", True) else r
        m["alpha_u"] = m["alpha_v"] = a
    elif t == "glass":
        m["kr"] = mat.get("Kr", (1, 1, 1))
        m["kt"] = mat.get("Kt", (1, 1, 1))
        m["eta"] = mat.get("eta", 1.5)
        r = float(mat.get("roughness", 0.0))
        if r != 0.0:
            a = roughness_to_alpha(r) if mat.get("remaproughness", True) else r
            m["alpha_u"] = m["alpha_v"] = a
    elif t == "metal":
        m["has_f0"] = 1
        f0 = np.array([0.955, 0.638, 0.538], np.float32)
        if "eta" in mat and "k" in mat:  # |((eta - 1) + ik) / ((eta + 1) + ik)|^2, complex<float> as the parser
            for c in range(3):
                z = np.complex64(complex(mat["eta"][c], mat["k"][c]))
                one = np.complex64(1)
                f0[c] = np.float32(abs(((z - one) / (z + one)) ** 2))
        m["f0"] = f0
        r = float(mat.get("roughness", 0.1))
        a = roughness_to_alpha(r) if mat.get("remaproughness", True) else r
        m["alpha_u"] = m["alpha_v"] = a
    elif t == "substrate":
        m["kd"] = mat.get("Kd", (0.5, 0.5, 0.5))
        m["ks"] = mat.get("Ks", (0.5, 0.5, 0.5))
        r = float(mat.get("roughness", 0.1))
        a = roughness_to_alpha(r) if mat.get("remaproughness", True) else r
        m["alpha_u"] = m["alpha_v"] = a
    elif t == "mirror":
        m["mirror_kr"] = mat.get("Kr", 0.9)
    return m


def look_at_c2w(eye, look, up) -> np.ndarray:
    """Camera-to-world of pbrt's LookAt as the reference builds it (glm::lookAtLH then
    inverse, SceneLoading/Parsing.cu:196-204); column-major 16 floats."""
    e, c, u = (np.asarray(x, np.float64) for x in (eye, look, up))
    f = c - e
    f /= np.linalg.norm(f)
    s = np.cross(u, f)
    s /= np.linalg.norm(s)
    uu = np.cross(f, s)
    V = np.eye(4)
    V[0, :3], V[1, :3], V[2, :3] = s, uu, f
    V[0, 3], V[1, 3], V[2, 3] = -s @ e, -uu @ e, -f @ e
    return np.linalg.inv(V).astype(np.float32).T.reshape(-1).copy()


def render_path(scene: dict, *, width: int, height: int, spp: int, max_depth: int, first: int = 0,
                count: int | None = None, filter_width: float = 1.0, integrator: str = "path"):
    """Oracle render of a scene dict (the format of cavalry_b200.scenes, camera from
    scene["camera"] else the config-1 view): returns the float film (sum [H,W,3], weight
    [H,W]) of camera samples [first, first + count).  integrator "directlighting" restates
    DirectLightingIntegrator.cu (one light sample per camera ray, no MIS)."""
    if integrator not in ("path", "directlighting"):
        raise ValueError(f"the oracle restates the path and direct-lighting integrators, not {integrator!r}")
    cam = dict(eye=(0.0, 0.0, -3.8), look=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), fov=40.0)
    cam.update(scene.get("camera", {}))
    eye, look, up, fov = cam["eye"], cam["look"], cam["up"], cam["fov"]
    pos = np.ascontiguousarray(scene["positions"], np.float32)
    idx = np.ascontiguousarray(scene["indices"], np.int32)
    tri_mesh = np.ascontiguousarray(scene["mesh_ids"], np.int32)
    nodes = build(pos, idx, rounds=0)["merged"]
    meshes = np.zeros(len(scene["meshes"]), OMESH_DTYPE)
    mats = np.zeros(len(scene["meshes"]), OMAT_DTYPE)
    # image textures in declaration order (named ones, then the environment's map), rows
    # flipped to the loader's bottom-up order
    images = [t["rgba"] for t in scene.get("textures", [])]
    tex_index = {t["name"]: k for k, t in enumerate(scene.get("textures", []))}
    env = scene.get("environment")
    lights = []
    w2l_id = (1, 0, 0, 0, 1, 0, 0, 0, 1)
    if env is not None:  # written first in the .pbrt, so light 0
        tex = -1
        if env.get("map") is not None:
            images.append(env["map"])
            tex = len(images) - 1
        lights.append((tuple(float(x) for x in env["L"]), -1, 1, tex, w2l_id))
    light_of = dict(scene.get("lights", []))
    shapes = scene.get("shapes", {})
    nrm = scene.get("normals")
    nrm = None if nrm is None else np.ascontiguousarray(nrm, np.float32)
    for k, (name, first_tri, n, mat) in enumerate(scene["meshes"]):
        meshes[k]["first_tri"], meshes[k]["tri_count"] = first_tri, n
        meshes[k]["material"] = k
        sh = shapes.get(k)
        if sh is not None and sh["type"] == "sphere":  # smooth normals; cone-sampled as a light
            meshes[k]["has_normals"] = 1
            meshes[k]["shape"] = 1
            c = np.asarray(sh["center"], np.float32)
            # TriangleMesh shapeParams: the transformed centre and |centre - transform(r, 0, 0)|
            e = (np.array([sh["radius"], 0, 0], np.float32) + c).astype(np.float32)
            meshes[k]["sphere"] = (c[0], c[1], c[2], np.float32(np.sqrt(np.float32(((c - e) ** 2).sum()))))
        elif sh is not None:
            meshes[k]["shape"] = 2
        mats[k] = material_record(mat, tex_index)
        L = light_of.get(k)
        if L is None and name == "light":
            L = scene.get("light_radiance", (17.0, 12.0, 4.0))
        if L is not None:
            meshes[k]["light"] = len(lights)
            lights.append(((float(L[0]), float(L[1]), float(L[2])), k, 0, -1, w2l_id))
        else:
            meshes[k]["light"] = -1
    light_arr = np.array(lights, OLIGHT_DTYPE)
    # 8-bit images flipped to the PNG loader's bottom-up rows; float (OpenEXR) images as stored,
    # RGBA as the EXR loader returns them (A = 1 when absent, one channel in all four)
    def float_rgba(im):
        f = np.asarray(im).astype(np.float32)
        if f.ndim == 2:
            f = f[..., None]
        if f.shape[2] == 1:
            f = np.repeat(f, 4, axis=2)
        elif f.shape[2] == 3:
            f = np.concatenate([f, np.ones(f.shape[:2] + (1,), np.float32)], axis=2)
        return np.ascontiguousarray(f)

    flipped = [float_rgba(im) if np.asarray(im).dtype.kind == "f" else np.ascontiguousarray(np.asarray(im, np.uint8)[::-1])
               for im in images]
    texs = np.zeros(max(len(flipped), 1), OTEX_DTYPE)
    for k, im in enumerate(flipped):
        texs[k]["width"], texs[k]["height"] = im.shape[1], im.shape[0]
        texs[k]["rgbaf" if im.dtype == np.float32 else "rgba"] = im.ctypes.data
    uvs = scene.get("uvs")
    uvs = None if uvs is None else np.ascontiguousarray(uvs, np.float32)
    c2w = look_at_c2w(eye, look, up)
    total = width * height * spp
    count = total - first if count is None else count
    fsum = np.zeros((height, width, 3), np.float32)
    fw = np.zeros((height, width), np.float32)
    st = _pt_lib().orc_render_path(_c(nodes), _c(pos), _c(idx), None if nrm is None else _c(nrm), _c(tri_mesh),
                                   _c(meshes), len(meshes),
                                   _c(mats), _c(light_arr), len(light_arr), _c(c2w), float(fov), width, height, spp,
                                   max_depth, filter_width, filter_width, int(first), int(count), _c(fsum), _c(fw),
                                   int(integrator == "directlighting"), None if uvs is None else _c(uvs), _c(texs),
                                   0 if env is not None else -1)
    del flipped
    if st != 0:
        raise RuntimeError(f"orc_render_path failed ({st})")
    return fsum, fw
