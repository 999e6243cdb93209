import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN_DIR = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


def golden_files():
    """BVH fixtures (the render fixture render_ref.npz has its own tests)."""
    return sorted(p for p in GOLDEN_DIR.glob("*.npz") if not p.name.startswith("render_"))


def load_golden(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def cuda_ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    import cavalry_b200 as cav

    ctx = cav.Context(0)
    yield ctx
    ctx.close()


def nodes_equal(mine, ref, what=""):
    """Bit-exact comparison of final node arrays on the fields the reference defines:
    leaf flag and box for every node, primitive for leaves, children for internal nodes
    (internal prim ranges are uninitialised in the reference, BVH/Optimization.cu:396-432)."""
    assert len(mine) == len(ref), what
    leaf_m = mine["is_leaf"].astype(bool)
    leaf_r = ref["is_leaf"].astype(bool)
    bad = np.nonzero(leaf_m != leaf_r)[0]
    assert bad.size == 0, f"{what}: leaf flags differ at {bad[:10]}"
    bm = mine["bmin"].view(np.uint32) != ref["bmin"].view(np.uint32)
    bM = mine["bmax"].view(np.uint32) != ref["bmax"].view(np.uint32)
    bad = np.nonzero(bm.any(1) | bM.any(1))[0]
    assert bad.size == 0, f"{what}: boxes differ at {bad[:10]}"
    pm = mine["prim_begin"] if "prim_begin" in mine.dtype.names else mine["begin"]
    pr = ref["prim_begin"] if "prim_begin" in ref.dtype.names else ref["begin"]
    bad = np.nonzero(leaf_m & (pm != pr))[0]
    assert bad.size == 0, f"{what}: leaf primitives differ at {bad[:10]}"
    inner = ~leaf_m
    bad = np.nonzero(inner & ((mine["left"] != ref["left"]) | (mine["right"] != ref["right"])))[0]
    assert bad.size == 0, f"{what}: children differ at {bad[:10]}"


def _prim(a):
    return a["prim_begin"] if "prim_begin" in a.dtype.names else a["begin"]


def race_affected(ref):
    """(sites, affected) masks over a reference LBVH node array: a site is an internal node
    whose stored box is not the union of its children's stored boxes (the unfenced sibling
    read of computeBounds, BVH/BVH.cu:224-248, picked up a zero-filled box); affected adds
    every ancestor of a site."""
    count = len(ref)
    leaf = ref["is_leaf"].astype(bool)
    inner = np.nonzero(~leaf)[0]
    L, R = ref["left"][inner], ref["right"][inner]
    umin = np.minimum(ref["bmin"][L], ref["bmin"][R])
    umax = np.maximum(ref["bmax"][L], ref["bmax"][R])
    site = np.zeros(count, bool)
    site[inner] = ((umin.view(np.uint32) != ref["bmin"][inner].view(np.uint32)).any(1)
                   | (umax.view(np.uint32) != ref["bmax"][inner].view(np.uint32)).any(1))
    parent = np.full(count, -1, np.int64)
    parent[L] = inner
    parent[R] = inner
    affected = site.copy()
    frontier = np.nonzero(site)[0]
    while frontier.size:
        p = parent[frontier]
        p = np.unique(p[p >= 0])
        p = p[~affected[p]]
        affected[p] = True
        frontier = p
    return site, affected


def lbvh_matches_reference(mine, ref, correct, what=""):
    """LBVH parity with the reference's own build.  Topology, leaf primitives and leaf boxes
    are bit-exact; internal boxes are bit-exact at every node the reference's refit race
    did not touch.  At a race site each coordinate of the reference's box is explained by
    one child read back as the zero-filled record (min(0, .) / max(0, .) of the other
    child); above a site the reference propagated that value.  Ours equals the race-free
    union (`correct`, the oracle's recomputation on the same topology) everywhere.
    Returns the number of race sites found in the reference."""
    assert len(mine) == len(ref) == len(correct), what
    leaf = ref["is_leaf"].astype(bool)
    assert np.array_equal(mine["is_leaf"].astype(bool), leaf), f"{what}: leaf flags differ"
    assert np.array_equal(_prim(mine)[leaf], _prim(ref)[leaf]), f"{what}: leaf primitives differ"
    inner = ~leaf
    assert np.array_equal(mine["left"][inner], ref["left"][inner]), f"{what}: left children differ"
    assert np.array_equal(mine["right"][inner], ref["right"][inner]), f"{what}: right children differ"
    site, affected = race_affected(ref)
    same = ~affected
    for f in ("bmin", "bmax"):
        bad = np.nonzero(same & (mine[f].view(np.uint32) != ref[f].view(np.uint32)).any(1))[0]
        assert bad.size == 0, f"{what}: {f} differs at unraced nodes {bad[:10]}"
    s = np.nonzero(site)[0]
    L, R = ref["left"][s], ref["right"][s]
    z = np.float32(0)
    okmin = ((ref["bmin"][s] == np.minimum(ref["bmin"][L], ref["bmin"][R]))
             | (ref["bmin"][s] == np.minimum(z, ref["bmin"][L])) | (ref["bmin"][s] == np.minimum(z, ref["bmin"][R])))
    okmax = ((ref["bmax"][s] == np.maximum(ref["bmax"][L], ref["bmax"][R]))
             | (ref["bmax"][s] == np.maximum(z, ref["bmax"][L])) | (ref["bmax"][s] == np.maximum(z, ref["bmax"][R])))
    bad = s[~(okmin.all(1) & okmax.all(1))]
    assert bad.size == 0, f"{what}: unexplained reference boxes at {bad[:10]}"
    for f in ("bmin", "bmax"):
        assert np.array_equal(mine[f].view(np.uint32), correct[f].view(np.uint32)), f"{what}: {f} not race-free union"
    return int(site.sum())
