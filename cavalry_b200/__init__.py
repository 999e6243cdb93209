"""cavalry_b200: B200-native BVH build and ray queries behind Cavalry's BVH interface.

The CUDA library ``libcavalry_b200.so`` (sm_100a, built in-tree by
``python -m cavalry_b200.build_ext``) exports the C ABI of ``include/cavalry.h``.
This module binds it with ctypes and adds torch-tensor conveniences; torch only
supplies device memory and streams.  There is no CPU fallback: importing the
bindings fails loudly when the library is missing.

Reference interfaces mirrored (paths inside AmesingFlank/Cavalry):
  ``Context.build``      BVH::build(Triangle*, int, const AABB&, int)   BVH/BVH.cu:317
  ``Bvh.trace_closest``  BVH::intersect                                 BVH/BVH.h:23-107
  ``Bvh.trace_any``      BVH::testVisibility                            BVH/BVH.h:109-189
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

__all__ = ["CavError", "Context", "Bvh", "Scene", "SceneInfo", "Server", "lib", "parse_pbrt", "film_to_rgb8",
           "REF_NODE_DTYPE", "TRACE_EXACT", "TRACE_CULL_ON_POP", "SERVE_MERGED", "SERVE_SEQUENTIAL"]

_PKG = Path(__file__).resolve().parent
_LIB_PATH = _PKG / "libcavalry_b200.so"

TRACE_EXACT = 0
TRACE_CULL_ON_POP = 1
TRACE_FAST = 2
TRACE_REORDER = 4  # with either mode: trace a large batch in the Morton order of its ray origins

STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "CUDA error",
    3: "out of device memory",
    4: "device-side wait timed out",
    5: "traversal stack overflow",
    6: "not ready",
    7: "cancelled",
}

# cav_ref_node (include/cavalry.h), the reference's BVHNode fields (BVH/BVHNode.h:8-21)
REF_NODE_DTYPE = np.dtype(
    [("bmin", "<f4", (3,)), ("bmax", "<f4", (3,)), ("prim_begin", "<i4"), ("prim_end", "<i4"),
     ("left", "<i4"), ("right", "<i4"), ("is_leaf", "<i4")]
)
assert REF_NODE_DTYPE.itemsize == 44


class CavError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}")


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded CUDA library.  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing; build it with `python -m cavalry_b200.build_ext` "
            "(there is no CPU fallback)"
        )
    L = ctypes.CDLL(str(_LIB_PATH))
    P, I64, I32, U32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32
    sig = {
        "cav_version": ([], ctypes.c_int),
        "cav_ctx_create": ([ctypes.c_int, ctypes.POINTER(P)], ctypes.c_int),
        "cav_ctx_destroy": ([P], ctypes.c_int),
        "cav_last_error": ([P], ctypes.c_char_p),
        "cav_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "cav_sync_check": ([P, P], ctypes.c_int),
        "cav_bvh_build": ([P, P, I64, P, P, I64, P, ctypes.c_int, P, ctypes.POINTER(P)], ctypes.c_int),
        "cav_bvh_free": ([P], ctypes.c_int),
        "cav_bvh_num_triangles": ([P], I64),
        "cav_bvh_depth": ([P, P, P, ctypes.POINTER(I32)], ctypes.c_int),
        "cav_bvh_export_nodes": ([P, P, P, P], ctypes.c_int),
        "cav_bvh_export_stages": ([P, P, P, P, P, P], ctypes.c_int),
        "cav_bvh_stage_times": ([P, P, P], ctypes.c_int),
        "cav_trace_closest": ([P, P, P, I64, P, P, P, U32, P], ctypes.c_int),
        "cav_trace_any": ([P, P, P, P, P, I64, P, U32, P], ctypes.c_int),
        "cav_trace_closest_host": ([P, P, P, I64, P, P, P, U32], ctypes.c_int),
        "cav_trace_any_host": ([P, P, P, P, P, I64, P, U32], ctypes.c_int),
        "cav_set_trace_config": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "cav_set_trace_stack": ([P, ctypes.c_uint32, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "cav_ctx_set_limits": ([P, ctypes.c_double, I64], ctypes.c_int),
        "cav_ctx_inject": ([P, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "cav_server_cancel": ([P, I64], ctypes.c_int),
        "cav_trace_stats": ([P, P, P, I64, ctypes.c_int, P, P, U32, P, P], ctypes.c_int),
        "cav_scene_load_pbrt": ([P, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(P)],
                                ctypes.c_int),
        "cav_scene_free": ([P], ctypes.c_int),
        "cav_scene_info": ([P, P], ctypes.c_int),
        "cav_render_to_host": ([P, P, P, P, P, P], ctypes.c_int),
        "cav_render": ([P, P, P, P, P, P], ctypes.c_int),
        "cav_render_stats": ([P, P], ctypes.c_int),
        "cav_bvh_build_batch": ([P, ctypes.c_int, P, P, P, P, P, P, ctypes.c_int, P, P], ctypes.c_int),
        "cav_render_guided": ([P, P, P, P, P, P, P, P, P], ctypes.c_int),
        "cav_mlp_num_params": ([], ctypes.c_int),
        "cav_mlp_create": ([P, ctypes.c_uint64, ctypes.POINTER(P)], ctypes.c_int),
        "cav_mlp_free": ([P], ctypes.c_int),
        "cav_mlp_get_params": ([P, P], ctypes.c_int),
        "cav_mlp_set_params": ([P, P], ctypes.c_int),
        "cav_mlp_forward": ([P, P, ctypes.c_int64, P, P], ctypes.c_int),
        "cav_mlp_set_kernel": ([P, ctypes.c_int], ctypes.c_int),
        "cav_mlp_gradients": ([P, P, P, P, ctypes.c_int64, P, P], ctypes.c_int),
        "cav_mlp_train_step": ([P, P, P, P, ctypes.c_int64, ctypes.c_float, P], ctypes.c_int),
        "cav_mlp_last_loss": ([P, P], ctypes.c_int),
        "cav_mlp_mixture": ([P, P, ctypes.c_int64, P, P, P, P, P], ctypes.c_int),
        "cav_trace_autotune": ([P, P, P, ctypes.c_int64, ctypes.c_int, P, P, P, P], ctypes.c_int),
        "cav_bvh_has_fast_layout": ([P], ctypes.c_int),
        "cav_pbrt_load_triangles": ([ctypes.c_char_p, P, ctypes.c_int64, P, P, ctypes.c_int64, P, P, P,
                                     ctypes.c_int], ctypes.c_int),
        "cav_trace_autotune_flags": ([P, P, P, ctypes.c_int64, ctypes.c_int, P, P, U32, P, P], ctypes.c_int),
        "cav_load_texture_png": ([ctypes.c_char_p, P, ctypes.c_int64, P, P, P, ctypes.c_int], ctypes.c_int),
        "cav_load_texture_exr": ([ctypes.c_char_p, P, ctypes.c_int64, P, P, P, ctypes.c_int], ctypes.c_int),
        "cav_server_create": ([P, P, ctypes.POINTER(P)], ctypes.c_int),
        "cav_server_destroy": ([P], ctypes.c_int),
        "cav_server_submit_render": ([P, P, P, P, P, P], ctypes.c_int),
        "cav_server_submit_rays": ([P, P, ctypes.c_int, P, P, P, ctypes.c_int64, P, P, P, P, P], ctypes.c_int),
        "cav_server_submit_scene": ([P, P, P], ctypes.c_int),
        "cav_server_poll": ([P, ctypes.c_int64, P], ctypes.c_int),
        "cav_server_wait": ([P, ctypes.c_int64, ctypes.c_double, P], ctypes.c_int),
        "cav_server_stats": ([P, P], ctypes.c_int),
        "cav_scene_bvh": ([P], P),
        "cav_render_capture_rays": ([P, P, P, ctypes.c_int, P, ctypes.c_int64, P], ctypes.c_int),
        "cav_film_to_rgb8": ([P, P, ctypes.c_int, ctypes.c_int, P], ctypes.c_int),
        "cav_write_png": ([ctypes.c_char_p, P, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "cav_write_pfm": ([ctypes.c_char_p, P, P, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "cav_pbrt_parse_info": ([ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, P, P, P, ctypes.c_int], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _ptr(t) -> int | None:
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def _require_cuda(x, dtype, numel: int, name: str, device_index: int) -> None:
    """Raise ValueError unless `x` is a contiguous CUDA tensor of `dtype` on GPU `device_index`
    with at least `numel` elements: the kernels read or write that many through the raw
    pointer, so a smaller or mistyped buffer would be overrun on the device."""
    if not getattr(x, "is_cuda", False):
        raise ValueError(f"{name}: expected a CUDA tensor")
    if x.dtype != dtype:
        raise ValueError(f"{name}: expected dtype {dtype}, got {x.dtype}")
    if not x.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")
    if x.device.index != device_index:
        raise ValueError(f"{name}: on cuda:{x.device.index}, the context is on cuda:{device_index}")
    if x.numel() < numel:
        raise ValueError(f"{name}: {x.numel()} elements, at least {numel} needed")


def _require_host(x, dtype, numel: int, name: str) -> None:
    """Raise ValueError unless `x` is a C-contiguous numpy array or CPU torch tensor of numpy
    `dtype` with at least `numel` elements: the host-buffer entry points copy that many
    elements through the raw pointer (a CUDA tensor's pointer is not host memory)."""
    if isinstance(x, np.ndarray):
        ok_dtype, contiguous, size = x.dtype == np.dtype(dtype), x.flags["C_CONTIGUOUS"], x.size
    else:
        if getattr(x, "is_cuda", True):
            raise ValueError(f"{name}: expected a numpy array or a CPU tensor")
        import torch

        ok_dtype = x.dtype == torch.from_numpy(np.empty(0, dtype)).dtype
        contiguous, size = x.is_contiguous(), x.numel()
    if not ok_dtype:
        raise ValueError(f"{name}: expected dtype {np.dtype(dtype)}, got {x.dtype}")
    if not contiguous:
        raise ValueError(f"{name}: expected a contiguous array")
    if size < numel:
        raise ValueError(f"{name}: {size} elements, at least {numel} needed")


def _stream_ptr(stream) -> int | None:
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream or None


class Context:
    """A cav_ctx on one CUDA device."""

    def __init__(self, device: int = 0):
        self.device = device
        h = ctypes.c_void_p()
        st = lib().cav_ctx_create(device, ctypes.byref(h))
        if st != 0:
            raise CavError(st, "cav_ctx_create")
        self.handle = h

    def _check(self, st: int, what: str):
        if st != 0:
            msg = lib().cav_last_error(self.handle) or b""
            raise CavError(st, f"{what}: {msg.decode(errors='replace')}")

    def close(self):
        if self.handle:
            lib().cav_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync_check(self, stream=None):
        self._check(lib().cav_sync_check(self.handle, _stream_ptr(stream)), "cav_sync_check")

    def set_limits(self, sort_wait_s: float = 0.0, max_trace_steps: int = 0):
        """Bounds of the device-side waits (0: defaults, 2 s and 2^22 visits per ray)."""
        self._check(lib().cav_ctx_set_limits(self.handle, sort_wait_s, max_trace_steps), "cav_ctx_set_limits")

    def inject(self, what: int, count: int = 1):
        """Failure injection for tests (INJECT_SORT_STALL, INJECT_ALLOC_FAIL, INJECT_MLP_STALL,
        INJECT_NONE)."""
        self._check(lib().cav_ctx_inject(self.handle, what, count), "cav_ctx_inject")

    def set_trace_config(self, block_threads: int = 0, blocks_per_sm: int = 0, batch: int = 0):
        self._check(lib().cav_set_trace_config(self.handle, block_threads, blocks_per_sm, batch),
                    "cav_set_trace_config")

    def set_trace_stack(self, stack: int = 0, smem_stack: int = 0, flags: int = 0):
        """Traversal stack of the exact mode (flags=TRACE_EXACT): 64 or 128 entries (0 = 128),
        the first 16 in shared memory (smem_stack=16) or all in local memory (0); of the fast
        mode (flags=TRACE_FAST): stack 0, the first 8 node groups in shared memory or none."""
        self._check(lib().cav_set_trace_stack(self.handle, flags, stack, smem_stack), "cav_set_trace_stack")

    def build_batch(self, scenes, rounds: int = 0, stream=None) -> list:
        """Build many BVHs with one launch per LBVH stage: scenes = [(positions, indices) or
        (positions, indices, mesh_ids)] of CUDA tensors.  Returns one Bvh per scene."""
        K = len(scenes)
        P = ctypes.c_void_p
        pos = (P * K)(*[_ptr(sc[0]) for sc in scenes])
        idx = (P * K)(*[_ptr(sc[1]) for sc in scenes])
        mids = (P * K)(*[_ptr(sc[2]) if len(sc) > 2 else None for sc in scenes])
        nv = (ctypes.c_int64 * K)(*[sc[0].shape[0] for sc in scenes])
        nt = (ctypes.c_int64 * K)(*[sc[1].shape[0] for sc in scenes])
        outs = (P * K)()
        st = lib().cav_bvh_build_batch(self.handle, K, pos, nv, idx, mids, nt, None, rounds, _stream_ptr(stream), outs)
        self._check(st, "cav_bvh_build_batch")
        return [Bvh(self, outs[k], int(nt[k]), keep=tuple(scenes[k])) for k in range(K)]

    def load_pbrt(self, path: str, spp: int = -1, integrator: str | None = None, bvh_rounds: int = -1) -> Scene:
        """Load a .pbrt scene and build its BVH (the reference's --spp / --integrator / --bvh-opt-rounds)."""
        h = ctypes.c_void_p()
        st = lib().cav_scene_load_pbrt(self.handle, path.encode(), spp, integrator.encode() if integrator else None,
                                       bvh_rounds, ctypes.byref(h))
        self._check(st, "cav_scene_load_pbrt")
        return Scene(self, h)

    def build(self, positions, indices, mesh_ids=None, scene_bounds=None, rounds: int = 0, stream=None) -> "Bvh":
        """LBVH + ``rounds`` treelet rounds over device tensors.

        positions: float32 [V,3] CUDA; indices: int32 [T,3] CUDA; mesh_ids: int32 [T] CUDA or None;
        scene_bounds: 6 floats (min xyz, max xyz) or None (computed on the device).
        """
        import torch

        assert positions.is_cuda and positions.dtype == torch.float32 and positions.is_contiguous()
        assert indices.is_cuda and indices.dtype == torch.int32 and indices.is_contiguous()
        _require_cuda(positions, torch.float32, 0, "positions", self.device)  # counts: the library checks
        _require_cuda(indices, torch.int32, 0, "indices", self.device)
        if mesh_ids is not None:
            assert mesh_ids.is_cuda and mesh_ids.dtype == torch.int32 and mesh_ids.is_contiguous()
            _require_cuda(mesh_ids, torch.int32, indices.numel() // 3, "mesh_ids", self.device)
        nb = None
        if scene_bounds is not None:
            nb = np.ascontiguousarray(np.asarray(scene_bounds, dtype=np.float32).reshape(6))
        h = ctypes.c_void_p()
        st = lib().cav_bvh_build(
            self.handle, _ptr(positions), positions.numel() // 3, _ptr(indices), _ptr(mesh_ids),
            indices.numel() // 3, None if nb is None else nb.ctypes.data, int(rounds), _stream_ptr(stream),
            ctypes.byref(h),
        )
        self._check(st, "cav_bvh_build")
        return Bvh(self, h, indices.numel() // 3, keep=(positions, indices, mesh_ids))


class SceneInfo(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("spp", ctypes.c_int), ("max_depth", ctypes.c_int),
                ("triangles", ctypes.c_int64), ("meshes", ctypes.c_int), ("lights", ctypes.c_int),
                ("bvh_rounds", ctypes.c_int), ("integrator", ctypes.c_int)]


_INTEGRATORS = {None: 0, "path": -1, "rlpath": 1, "guided": 2, "directlighting": 3}
RENDER_GRAPH = 1
RENDER_FAST_TRACE = 2


class RenderOpts(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_int), ("max_depth", ctypes.c_int), ("integrator", ctypes.c_int),
                ("max_paths_in_flight", ctypes.c_int64), ("width", ctypes.c_int), ("height", ctypes.c_int),
                ("flags", ctypes.c_int), ("sample_begin", ctypes.c_int64), ("sample_end", ctypes.c_int64)]


def parse_pbrt(path: str, spp: int = -1, integrator: str | None = None) -> tuple[SceneInfo, np.ndarray]:
    """Host-only parse of a .pbrt file (no GPU): scene counts and the camera-to-world matrix."""
    info = SceneInfo()
    c2w = np.zeros(16, np.float32)
    err = ctypes.create_string_buffer(512)
    st = lib().cav_pbrt_parse_info(path.encode(), spp, integrator.encode() if integrator else None,
                                   ctypes.addressof(info), c2w.ctypes.data, ctypes.addressof(err), len(err))
    if st != 0:
        raise CavError(st, "cav_pbrt_parse_info: " + err.value.decode(errors="replace"))
    return info, c2w.reshape(4, 4).T


def load_texture_exr(path: str) -> np.ndarray:
    """Host-only: an OpenEXR texture as scene loading decodes it, [H, W, 4] float32 RGBA with
    rows in the file's order (no flip, no gamma) (no GPU)."""
    w, h = ctypes.c_int(), ctypes.c_int()
    err = ctypes.create_string_buffer(512)
    L = lib()
    st = L.cav_load_texture_exr(path.encode(), None, 0, ctypes.byref(w), ctypes.byref(h), ctypes.addressof(err),
                                len(err))
    if st != 0:
        raise CavError(st, "cav_load_texture_exr: " + err.value.decode(errors="replace"))
    out = np.zeros((h.value, w.value, 4), np.float32)
    st = L.cav_load_texture_exr(path.encode(), out.ctypes.data, out.size, ctypes.byref(w), ctypes.byref(h),
                                ctypes.addressof(err), len(err))
    if st != 0:
        raise CavError(st, "cav_load_texture_exr: " + err.value.decode(errors="replace"))
    return out


def load_texture_png(path: str) -> np.ndarray:
    """Host-only: a texture image as scene loading decodes it, [H, W, 4] uint8 with rows
    bottom-up and the colour channels through the inverse sRGB curve (no GPU)."""
    w, h = ctypes.c_int(), ctypes.c_int()
    err = ctypes.create_string_buffer(512)
    L = lib()
    st = L.cav_load_texture_png(path.encode(), None, 0, ctypes.byref(w), ctypes.byref(h), ctypes.addressof(err),
                                len(err))
    if st != 0:
        raise CavError(st, "cav_load_texture_png: " + err.value.decode(errors="replace"))
    out = np.zeros((h.value, w.value, 4), np.uint8)
    st = L.cav_load_texture_png(path.encode(), out.ctypes.data, out.nbytes, ctypes.byref(w), ctypes.byref(h),
                                ctypes.addressof(err), len(err))
    if st != 0:
        raise CavError(st, "cav_load_texture_png: " + err.value.decode(errors="replace"))
    return out


def load_pbrt_triangles(path: str) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Host-only parse of a .pbrt file to (positions [V,3] f32, indices [T,3] i32, mesh ids [T] i32)."""
    nv, nt = ctypes.c_int64(), ctypes.c_int64()
    err = ctypes.create_string_buffer(512)
    L = lib()
    st = L.cav_pbrt_load_triangles(path.encode(), None, 0, None, None, 0, ctypes.byref(nv), ctypes.byref(nt),
                                   ctypes.addressof(err), len(err))
    if st != 0:
        raise CavError(st, "cav_pbrt_load_triangles: " + err.value.decode(errors="replace"))
    pos = np.zeros((nv.value, 3), np.float32)
    idx = np.zeros((nt.value, 3), np.int32)
    mid = np.zeros(nt.value, np.int32)
    st = L.cav_pbrt_load_triangles(path.encode(), pos.ctypes.data, nv.value, idx.ctypes.data, mid.ctypes.data,
                                   nt.value, ctypes.byref(nv), ctypes.byref(nt), ctypes.addressof(err), len(err))
    if st != 0:
        raise CavError(st, "cav_pbrt_load_triangles: " + err.value.decode(errors="replace"))
    return pos, idx, mid


class RenderStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_int64), ("closest_rays", ctypes.c_int64), ("shadow_rays", ctypes.c_int64),
                ("bounces", ctypes.c_int), ("ms_total", ctypes.c_float), ("ms_closest", ctypes.c_float),
                ("ms_shade", ctypes.c_float), ("ms_any", ctypes.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GuideOpts(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_float), ("train_samples_per_pass", ctypes.c_int64),
                ("train_steps_per_pass", ctypes.c_int), ("train_batch", ctypes.c_int),
                ("learning_rate", ctypes.c_float), ("freeze", ctypes.c_int), ("seed", ctypes.c_uint64)]


class GuideStats(ctypes.Structure):
    _fields_ = [("passes", ctypes.c_int), ("train_samples", ctypes.c_int64), ("train_steps", ctypes.c_int64),
                ("last_loss", ctypes.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Scene:
    """A loaded .pbrt scene with its BVH (cav_scene)."""

    def __init__(self, ctx: "Context", handle):
        self.ctx = ctx
        self.handle = handle

    def info(self) -> SceneInfo:
        out = SceneInfo()
        self.ctx._check(lib().cav_scene_info(self.handle, ctypes.addressof(out)), "cav_scene_info")
        return out

    def render(self, spp: int = 0, max_depth: int = 0, max_paths_in_flight: int = 0, integrator: str | None = None,
               width: int = 0, height: int = 0, graph: bool = False, fast_trace: bool = False,
               sample_range: tuple[int, int] | None = None):
        """Render to host arrays; returns (film_sum [H,W,3], film_weight [H,W], ms).  integrator:
        None = the scene's, "path", "rlpath", "guided" or "directlighting"; width/height override
        the Film resolution; sample_range = (begin, end) renders only those camera samples
        (pixel-major numbering), whose films sum to the whole render's."""
        inf = self.info()
        W, H = (width, height) if width > 0 and height > 0 else (inf.width, inf.height)
        s = np.zeros((H, W, 3), np.float32)
        w = np.zeros((H, W), np.float32)
        ms = np.zeros(1, np.float32)
        b, e = sample_range if sample_range is not None else (0, 0)
        opts = RenderOpts(spp, max_depth, _INTEGRATORS[integrator], max_paths_in_flight, width, height,
                          (RENDER_GRAPH if graph else 0) | (RENDER_FAST_TRACE if fast_trace else 0), b, e)
        st = lib().cav_render_to_host(self.ctx.handle, self.handle, ctypes.addressof(opts), s.ctypes.data,
                                      w.ctypes.data, ms.ctypes.data)
        self.ctx._check(st, "cav_render_to_host")
        return s, w, float(ms[0])

    def render_into(self, film_sum, film_weight, spp: int = 0, max_depth: int = 0, max_paths_in_flight: int = 0,
                    stream=None, integrator: str | None = None, width: int = 0, height: int = 0, graph: bool = False,
                    fast_trace: bool = False, sample_range: tuple[int, int] | None = None):
        """Render into DEVICE films (pointers, or objects with data_ptr(): 3 + 1 floats per
        pixel), stream-ordered on `stream` (a pointer, an object with cuda_stream, or None)."""
        ptr = lambda x: x if isinstance(x, int) else x.data_ptr()  # noqa: E731
        st_ptr = None if stream is None else (stream if isinstance(stream, int) else stream.cuda_stream)
        b, e = sample_range if sample_range is not None else (0, 0)
        opts = RenderOpts(spp, max_depth, _INTEGRATORS[integrator], max_paths_in_flight, width, height,
                          (RENDER_GRAPH if graph else 0) | (RENDER_FAST_TRACE if fast_trace else 0), b, e)
        st = lib().cav_render(self.ctx.handle, self.handle, ctypes.addressof(opts), ptr(film_sum), ptr(film_weight),
                              st_ptr)
        self.ctx._check(st, "cav_render")

    def render_guided(self, spp: int = 0, max_depth: int = 0, width: int = 0, height: int = 0, mlp=None,
                      alpha: float = 0.5, freeze: bool = False, seed: int = 1, **train):
        """MLP-guided render into host arrays: (film_sum, film_weight, ms, stats dict)."""
        import torch

        inf = self.info()
        W, H = (width, height) if width > 0 and height > 0 else (inf.width, inf.height)
        fs = torch.zeros(H * W * 3, device=f"cuda:{self.ctx.device}")
        fw = torch.zeros(H * W, device=f"cuda:{self.ctx.device}")
        opts = RenderOpts(spp, max_depth, -1, 0, width, height, 0)
        g = GuideOpts(alpha, train.get("samples_per_pass", 0), train.get("steps_per_pass", 0), train.get("batch", 0),
                      train.get("lr", 0.0), int(freeze), seed)
        st_out = GuideStats()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        st = lib().cav_render_guided(self.ctx.handle, self.handle, ctypes.addressof(opts),
                                     mlp.handle if mlp is not None else None, ctypes.addressof(g), fs.data_ptr(),
                                     fw.data_ptr(), None, ctypes.addressof(st_out))
        b.record()
        self.ctx._check(st, "cav_render_guided")
        torch.cuda.synchronize()
        return (fs.view(H, W, 3).cpu().numpy(), fw.view(H, W).cpu().numpy(), a.elapsed_time(b), st_out.as_dict())

    def bvh(self) -> "Bvh":
        """The scene's BVH (owned by the scene; valid until the scene is freed)."""
        h = lib().cav_scene_bvh(self.handle)
        return Bvh(self.ctx, h, int(self.info().triangles), keep=(self,), owned=False)

    def stats(self) -> RenderStats:
        """Ray counts and device stage times of the last render (waits for it)."""
        out = RenderStats()
        self.ctx._check(lib().cav_render_stats(self.handle, ctypes.addressof(out)), "cav_render_stats")
        return out

    def capture_rays(self, depth: int, capacity: int = 1 << 22, spp: int = 0, max_depth: int = 0):
        """Extend-stage rays of bounce `depth` of the first chunk of paths, as a [k, 8] float32
        CUDA tensor (the 32-byte cav_ray records)."""
        import torch

        buf = torch.empty((capacity, 8), dtype=torch.float32, device=f"cuda:{self.ctx.device}")
        n = ctypes.c_int64(0)
        opts = RenderOpts(spp, max_depth, 0, capacity, 0, 0)
        st = lib().cav_render_capture_rays(self.ctx.handle, self.handle, ctypes.addressof(opts), depth,
                                           buf.data_ptr(), capacity, ctypes.byref(n))
        self.ctx._check(st, "cav_render_capture_rays")
        return buf[: n.value]

    def free(self):
        if self.handle:
            lib().cav_scene_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


SCENE_RENDER, SCENE_CLOSEST, SCENE_ANY = 0, 1, 2


class SceneJob(ctypes.Structure):
    _fields_ = [("pbrt_path", ctypes.c_char_p), ("kind", ctypes.c_int), ("bvh_rounds", ctypes.c_int),
                ("render", RenderOpts), ("host_sum", ctypes.c_void_p), ("host_weight", ctypes.c_void_p),
                ("host_rays", ctypes.c_void_p), ("host_limit", ctypes.c_void_p), ("host_excl", ctypes.c_void_p),
                ("n_rays", ctypes.c_int64), ("host_prim", ctypes.c_void_p), ("host_t", ctypes.c_void_p),
                ("host_uv", ctypes.c_void_p), ("host_occ", ctypes.c_void_p)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_int64), ("mode", ctypes.c_int), ("max_live_jobs", ctypes.c_int),
                ("max_paths_per_job", ctypes.c_int64), ("trace_flags", ctypes.c_uint32), ("lanes", ctypes.c_int),
                ("min_paths_per_slice", ctypes.c_int64), ("reject_over_budget", ctypes.c_int),
                ("loaders", ctypes.c_int), ("graph_max_paths", ctypes.c_int64)]


class JobStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int), ("t_submit", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_done", ctypes.c_double), ("bounces", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [("ticks", ctypes.c_int64), ("closest_launches", ctypes.c_int64), ("any_launches", ctypes.c_int64),
                ("max_segments", ctypes.c_int64), ("busy_s", ctypes.c_double), ("now_s", ctypes.c_double),
                ("pending", ctypes.c_int64), ("live", ctypes.c_int64), ("hbm_in_use", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


JOB_PENDING, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = 0, 1, 2, 3, 4
INJECT_NONE, INJECT_SORT_STALL, INJECT_ALLOC_FAIL, INJECT_MLP_STALL = 0, 1, 2, 3
SERVE_MERGED, SERVE_SEQUENTIAL = 0, 1


class Server:
    """A serving loop (cav_server): render and ray-query jobs merged into shared traversal
    launches.  Results land in the numpy arrays returned by the submit calls once
    :meth:`wait` reports the job done."""

    def __init__(self, ctx: "Context", hbm_budget_bytes: int = 80 << 30, mode: int = SERVE_MERGED,
                 max_live_jobs: int = 64, max_paths_per_job: int = 0, trace_flags: int = TRACE_EXACT, lanes: int = 0,
                 min_paths_per_slice: int = 0, reject_over_budget: bool = False, loaders: int = 0,
                 graph_max_paths: int = 0):
        self.ctx = ctx
        cfg = ServerConfig(hbm_budget_bytes, mode, max_live_jobs, max_paths_per_job, trace_flags, lanes,
                           min_paths_per_slice, int(reject_over_budget), loaders, graph_max_paths)
        h = ctypes.c_void_p()
        ctx._check(lib().cav_server_create(ctx.handle, ctypes.addressof(cfg), ctypes.byref(h)), "cav_server_create")
        self.handle = h
        self._keep: dict[int, tuple] = {}

    def submit_render(self, scene: "Scene", spp: int = 0, max_depth: int = 0, max_paths_in_flight: int = 0,
                      width: int = 0, height: int = 0):
        inf = scene.info()
        W, H = (width, height) if width > 0 and height > 0 else (inf.width, inf.height)
        fs = np.zeros((H, W, 3), np.float32)
        fw = np.zeros((H, W), np.float32)
        opts = RenderOpts(spp, max_depth, -1, max_paths_in_flight, width, height)
        job = ctypes.c_int64(0)
        st = lib().cav_server_submit_render(self.handle, scene.handle, ctypes.addressof(opts), fs.ctypes.data,
                                            fw.ctypes.data, ctypes.byref(job))
        self.ctx._check(st, "cav_server_submit_render")
        self._keep[job.value] = (scene, fs, fw, opts)
        return job.value, fs, fw

    def submit_rays(self, bvh: "Bvh", rays: np.ndarray, any_hit: bool = False, limit=None, excl=None):
        rays = np.ascontiguousarray(rays, np.float32)
        if rays.ndim != 2 or rays.shape[1] != 8:
            raise ValueError(f"rays: expected an [n, 8] array, got shape {rays.shape}")
        n = rays.shape[0]
        lim = None if limit is None else np.ascontiguousarray(limit, np.float32)
        ex = None if excl is None else np.ascontiguousarray(excl, np.int32)
        if lim is not None:
            _require_host(lim, np.float32, n, "limit")
        if ex is not None:
            _require_host(ex, np.int32, 2 * n, "excl")
        job = ctypes.c_int64(0)
        if any_hit:
            out = (np.zeros(n, np.uint8),)
            st = lib().cav_server_submit_rays(self.handle, bvh.handle, 1, rays.ctypes.data, _np_ptr(lim), _np_ptr(ex),
                                              n, None, None, None, out[0].ctypes.data, ctypes.byref(job))
        else:
            out = (np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros((n, 2), np.float32))
            st = lib().cav_server_submit_rays(self.handle, bvh.handle, 0, rays.ctypes.data, None, None, n,
                                              out[0].ctypes.data, out[1].ctypes.data, out[2].ctypes.data, None,
                                              ctypes.byref(job))
        self.ctx._check(st, "cav_server_submit_rays")
        self._keep[job.value] = (bvh, rays, lim, ex, out)
        return (job.value, *out)

    def submit_scene_render(self, pbrt_path: str, width: int, height: int, spp: int = 0, max_depth: int = 0,
                            bvh_rounds: int = -1, max_paths_in_flight: int = 0):
        """A render job that brings its own scene (cav_server_submit_scene): returns (job id,
        film_sum [H,W,3], film_weight [H,W]), filled once the job is done."""
        fs = np.zeros((height, width, 3), np.float32)
        fw = np.zeros((height, width), np.float32)
        spec = SceneJob(pbrt_path.encode(), SCENE_RENDER, bvh_rounds,
                        RenderOpts(spp, max_depth, -1, max_paths_in_flight, width, height), fs.ctypes.data,
                        fw.ctypes.data)
        job = ctypes.c_int64(0)
        st = lib().cav_server_submit_scene(self.handle, ctypes.addressof(spec), ctypes.byref(job))
        self.ctx._check(st, "cav_server_submit_scene")
        self._keep[job.value] = (spec, fs, fw)
        return job.value, fs, fw

    def submit_scene_rays(self, pbrt_path: str, rays: np.ndarray, any_hit: bool = False, limit=None, excl=None,
                          bvh_rounds: int = -1):
        """A ray-query job against its own scene's tree: returns (job id, *outputs) as submit_rays."""
        rays = np.ascontiguousarray(rays, np.float32)
        if rays.ndim != 2 or rays.shape[1] != 8:
            raise ValueError(f"rays: expected an [n, 8] array, got shape {rays.shape}")
        n = rays.shape[0]
        lim = None if limit is None else np.ascontiguousarray(limit, np.float32)
        ex = None if excl is None else np.ascontiguousarray(excl, np.int32)
        if lim is not None:
            _require_host(lim, np.float32, n, "limit")
        if ex is not None:
            _require_host(ex, np.int32, 2 * n, "excl")
        if any_hit:
            out = (np.zeros(n, np.uint8),)
            spec = SceneJob(pbrt_path.encode(), SCENE_ANY, bvh_rounds, RenderOpts(), None, None, rays.ctypes.data,
                            _np_ptr(lim), _np_ptr(ex), n, None, None, None, out[0].ctypes.data)
        else:
            out = (np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros((n, 2), np.float32))
            spec = SceneJob(pbrt_path.encode(), SCENE_CLOSEST, bvh_rounds, RenderOpts(), None, None, rays.ctypes.data,
                            None, None, n, out[0].ctypes.data, out[1].ctypes.data, out[2].ctypes.data, None)
        job = ctypes.c_int64(0)
        st = lib().cav_server_submit_scene(self.handle, ctypes.addressof(spec), ctypes.byref(job))
        self.ctx._check(st, "cav_server_submit_scene")
        self._keep[job.value] = (spec, rays, lim, ex, out)
        return (job.value, *out)

    def wait(self, job: int, timeout_s: float = -1.0) -> JobStatus:
        """Waits for a job; returns its status (state JOB_DONE or JOB_CANCELLED), raises
        TimeoutError when it is still running after timeout_s and CavError when it failed."""
        out = JobStatus()
        st = lib().cav_server_wait(self.handle, job, timeout_s, ctypes.addressof(out))
        if st == 4 and out.state not in (JOB_DONE, JOB_FAILED, JOB_CANCELLED):
            raise TimeoutError(f"job {job} not done after {timeout_s} s")
        if st != 7:  # CAV_ERR_CANCELLED: the status says so
            self.ctx._check(st, f"job {job}")
        return out

    def cancel(self, job: int):
        """Cancel a pending or running job (cav_server_cancel); wait() then reports JOB_CANCELLED."""
        self.ctx._check(lib().cav_server_cancel(self.handle, job), "cav_server_cancel")

    def poll(self, job: int) -> JobStatus:
        out = JobStatus()
        self.ctx._check(lib().cav_server_poll(self.handle, job, ctypes.addressof(out)), "cav_server_poll")
        return out

    def release(self, job: int):
        """Drop the host arrays kept alive for a finished job."""
        self._keep.pop(job, None)

    def stats(self) -> ServerStats:
        out = ServerStats()
        self.ctx._check(lib().cav_server_stats(self.handle, ctypes.addressof(out)), "cav_server_stats")
        return out

    def close(self):
        if self.handle:
            lib().cav_server_destroy(self.handle)
            self.handle = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


MLP_KERNEL_TCGEN05 = 0  # cav_mlp_set_kernel: 128-sample tiles on tcgen05, accumulators in TMEM
MLP_KERNEL_MMA_SYNC = 1  # 16-sample warp tiles with mma.sync


class Mlp:
    """The learned directional proposal (cav_mlp): 5 inputs in [0, 1] -> 8-lobe vMF mixture.
    `kernel` picks the forward-pass kernel (MLP_KERNEL_TCGEN05 by default)."""

    def __init__(self, ctx: "Context", seed: int = 1, kernel: int = MLP_KERNEL_TCGEN05):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx._check(lib().cav_mlp_create(ctx.handle, seed, ctypes.byref(h)), "cav_mlp_create")
        self.handle = h
        self.n_params = lib().cav_mlp_num_params()
        self.set_kernel(kernel)

    def set_kernel(self, kernel: int):
        self.ctx._check(lib().cav_mlp_set_kernel(self.handle, kernel), "cav_mlp_set_kernel")
        self.kernel = kernel

    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        self.ctx._check(lib().cav_mlp_get_params(self.handle, p.ctypes.data), "cav_mlp_get_params")
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        self.ctx._check(lib().cav_mlp_set_params(self.handle, p.ctypes.data), "cav_mlp_set_params")

    def forward(self, x):
        import torch

        out = torch.empty((x.shape[0], 32), dtype=torch.float32, device=x.device)
        self.ctx._check(lib().cav_mlp_forward(self.handle, _ptr(x), x.shape[0], _ptr(out), None), "cav_mlp_forward")
        return out

    def gradients(self, x, dirs, w):
        g = np.zeros(self.n_params, np.float32)
        loss = np.zeros(1, np.float32)
        st = lib().cav_mlp_gradients(self.handle, _ptr(x), _ptr(dirs), _ptr(w), x.shape[0], g.ctypes.data,
                                     loss.ctypes.data)
        self.ctx._check(st, "cav_mlp_gradients")
        return g, float(loss[0])

    def train_step(self, x, dirs, w, lr: float = 1e-3, stream=None):
        st = lib().cav_mlp_train_step(self.handle, _ptr(x), _ptr(dirs), _ptr(w), x.shape[0], lr, _stream_ptr(stream))
        self.ctx._check(st, "cav_mlp_train_step")

    def last_loss(self) -> float:
        v = np.zeros(1, np.float32)
        self.ctx._check(lib().cav_mlp_last_loss(self.handle, v.ctypes.data), "cav_mlp_last_loss")
        return float(v[0])

    def pdf(self, out, dirs):
        import torch

        p = torch.empty(out.shape[0], dtype=torch.float32, device=out.device)
        st = lib().cav_mlp_mixture(self.ctx.handle, _ptr(out), out.shape[0], _ptr(dirs), _ptr(p), None, None, None)
        self.ctx._check(st, "cav_mlp_mixture")
        return p

    def sample(self, out, u):
        import torch

        d = torch.empty((out.shape[0], 3), dtype=torch.float32, device=out.device)
        st = lib().cav_mlp_mixture(self.ctx.handle, _ptr(out), out.shape[0], None, None, _ptr(u), _ptr(d), None)
        self.ctx._check(st, "cav_mlp_mixture")
        return d

    def free(self):
        if self.handle:
            lib().cav_mlp_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _np_ptr(a):
    return None if a is None else a.ctypes.data


def film_to_rgb8(film_sum: np.ndarray, film_weight: np.ndarray) -> np.ndarray:
    h, w = film_weight.shape
    out = np.zeros((h, w, 3), np.uint8)
    s = np.ascontiguousarray(film_sum, np.float32)
    wt = np.ascontiguousarray(film_weight, np.float32)
    lib().cav_film_to_rgb8(s.ctypes.data, wt.ctypes.data, w, h, out.ctypes.data)
    return out


class TraceConfig(ctypes.Structure):
    _fields_ = [("block_threads", ctypes.c_int), ("blocks_per_sm", ctypes.c_int), ("batch", ctypes.c_int),
                ("stack", ctypes.c_int), ("ms", ctypes.c_float), ("smem_stack", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Bvh:
    """A built BVH (cav_bvh).  Device memory is released by :meth:`free`."""

    def __init__(self, ctx: Context, handle, n: int, keep=(), owned: bool = True):
        self.ctx = ctx
        self.handle = handle
        self.n = n
        self._keep = keep
        self._owned = owned

    def free(self):
        if self.handle and self._owned:
            lib().cav_bvh_free(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def export_nodes(self, stream=None) -> np.ndarray:
        out = np.zeros(2 * self.n - 1, dtype=REF_NODE_DTYPE)
        self.ctx._check(lib().cav_bvh_export_nodes(self.ctx.handle, self.handle, _stream_ptr(stream), out.ctypes.data),
                        "cav_bvh_export_nodes")
        return out

    def export_stages(self, stream=None):
        mu = np.zeros(self.n, np.uint64)
        ms = np.zeros(self.n, np.uint64)
        pr = np.zeros(self.n, np.int32)
        self.ctx._check(lib().cav_bvh_export_stages(self.ctx.handle, self.handle, _stream_ptr(stream), mu.ctypes.data,
                                                    ms.ctypes.data, pr.ctypes.data), "cav_bvh_export_stages")
        return mu, ms, pr

    def depth(self, stream=None) -> int:
        d = ctypes.c_int32()
        self.ctx._check(lib().cav_bvh_depth(self.ctx.handle, self.handle, _stream_ptr(stream), ctypes.byref(d)),
                        "cav_bvh_depth")
        return d.value

    def stage_times(self) -> list[float]:
        ms = np.zeros(6, np.float32)
        self.ctx._check(lib().cav_bvh_stage_times(self.ctx.handle, self.handle, ms.ctypes.data), "cav_bvh_stage_times")
        return [float(x) for x in ms]

    def autotune(self, rays, any_hit: bool = False, limit=None, excl=None, flags: int = TRACE_EXACT,
                 stream=None) -> dict:
        """Pick and install the fastest traversal launch shape for this tree on a CUDA ray sample,
        for the exact mode or (flags=TRACE_FAST) the compressed 8-wide mode."""
        import torch

        n = rays.shape[0]
        _require_cuda(rays, torch.float32, 8 * n, "rays", self.ctx.device)
        if limit is not None:
            _require_cuda(limit, torch.float32, n, "limit", self.ctx.device)
        if excl is not None:
            _require_cuda(excl, torch.int32, 2 * n, "excl", self.ctx.device)
        out = TraceConfig()
        st = lib().cav_trace_autotune_flags(self.ctx.handle, self.handle, _ptr(rays), rays.shape[0], int(any_hit),
                                            _ptr(limit), _ptr(excl), flags, _stream_ptr(stream),
                                            ctypes.addressof(out))
        self.ctx._check(st, "cav_trace_autotune_flags")
        return out.as_dict()

    def has_fast_layout(self) -> bool:
        """Whether the compressed 8-wide view of TRACE_FAST has been built for this tree."""
        return bool(lib().cav_bvh_has_fast_layout(self.handle))

    def trace_closest(self, rays, flags: int = TRACE_EXACT, stream=None, out=None):
        """rays: float32 [n,8] CUDA (o.xyz, tmin, d.xyz, tmax).  Returns (prim int32, t float32, uv float32 [n,2])."""
        import torch

        assert rays.is_cuda and rays.dtype == torch.float32 and rays.is_contiguous() and rays.shape[-1] == 8
        n = rays.shape[0]
        dev = self.ctx.device
        _require_cuda(rays, torch.float32, 8 * n, "rays", dev)
        if out is None:
            prim = torch.empty(n, dtype=torch.int32, device=rays.device)
            t = torch.empty(n, dtype=torch.float32, device=rays.device)
            uv = torch.empty((n, 2), dtype=torch.float32, device=rays.device)
        else:
            prim, t, uv = out
            _require_cuda(prim, torch.int32, n, "out prim", dev)
            if t is not None:
                _require_cuda(t, torch.float32, n, "out t", dev)
            if uv is not None:
                _require_cuda(uv, torch.float32, 2 * n, "out uv", dev)
        st = lib().cav_trace_closest(self.ctx.handle, self.handle, _ptr(rays), n, _ptr(prim), _ptr(t), _ptr(uv),
                                     int(flags), _stream_ptr(stream))
        self.ctx._check(st, "cav_trace_closest")
        return prim, t, uv

    def trace_any(self, rays, limit=None, excl=None, flags: int = TRACE_EXACT, stream=None, out=None):
        """Any hit.  limit: float32 [n] or None; excl: int32 [n,2] (source, target mesh) or None."""
        import torch

        assert rays.is_cuda and rays.dtype == torch.float32 and rays.is_contiguous() and rays.shape[-1] == 8
        n = rays.shape[0]
        dev = self.ctx.device
        _require_cuda(rays, torch.float32, 8 * n, "rays", dev)
        if limit is not None:
            _require_cuda(limit, torch.float32, n, "limit", dev)
        if excl is not None:
            _require_cuda(excl, torch.int32, 2 * n, "excl", dev)
        occ = out if out is not None else torch.empty(n, dtype=torch.uint8, device=rays.device)
        _require_cuda(occ, torch.uint8, n, "out", dev)
        st = lib().cav_trace_any(self.ctx.handle, self.handle, _ptr(rays), _ptr(limit), _ptr(excl), n, _ptr(occ),
                                 int(flags), _stream_ptr(stream))
        self.ctx._check(st, "cav_trace_any")
        return occ

    def trace_stats(self, rays, any_hit: bool = False, limit=None, excl=None, flags: int = TRACE_EXACT, stream=None):
        """(node records fetched, triangles tested) totals of one instrumented traversal."""
        out = np.zeros(2, np.uint64)
        st = lib().cav_trace_stats(self.ctx.handle, self.handle, _ptr(rays), rays.shape[0], int(any_hit), _ptr(limit),
                                   _ptr(excl), int(flags), _stream_ptr(stream), out.ctypes.data)
        self.ctx._check(st, "cav_trace_stats")
        return int(out[0]), int(out[1])

    def trace_closest_host(self, rays: np.ndarray, flags: int = TRACE_EXACT, out=None):
        """Host-buffer variant (numpy in and out; pinned torch CPU tensors also accepted)."""
        n = rays.shape[0]
        _require_host(rays, np.float32, 8 * n, "rays")
        if out is None:
            prim = np.empty(n, np.int32)
            t = np.empty(n, np.float32)
            uv = np.empty((n, 2), np.float32)
        else:
            prim, t, uv = out
            _require_host(prim, np.int32, n, "out prim")
            if t is not None:
                _require_host(t, np.float32, n, "out t")
            if uv is not None:
                _require_host(uv, np.float32, 2 * n, "out uv")
        st = lib().cav_trace_closest_host(self.ctx.handle, self.handle, _ptr(rays), n, _ptr(prim), _ptr(t), _ptr(uv),
                                          int(flags))
        self.ctx._check(st, "cav_trace_closest_host")
        return prim, t, uv

    def trace_any_host(self, rays, limit=None, excl=None, flags: int = TRACE_EXACT, out=None):
        n = rays.shape[0]
        _require_host(rays, np.float32, 8 * n, "rays")
        if limit is not None:
            _require_host(limit, np.float32, n, "limit")
        if excl is not None:
            _require_host(excl, np.int32, 2 * n, "excl")
        occ = out if out is not None else np.empty(n, np.uint8)
        _require_host(occ, np.uint8, n, "out")
        st = lib().cav_trace_any_host(self.ctx.handle, self.handle, _ptr(rays), _ptr(limit), _ptr(excl), n, _ptr(occ),
                                      int(flags))
        self.ctx._check(st, "cav_trace_any_host")
        return occ
