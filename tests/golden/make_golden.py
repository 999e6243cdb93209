"""Generate the golden fixtures in tests/golden/ by running the REFERENCE's own CUDA code.

    python tests/golden/make_golden.py [OUT_DIR]

Needs a GPU and ``oracle/_ref/libcavref.so`` (the reference's BVH/BVH.cu and
BVH/Optimization.cu compiled verbatim by ``oracle/build_ref.sh``).  For every case the
reference replays the LBVH part of BVH::build stage by stage (BVH/BVH.cu:317-352); its
verbatim BVH::intersect / BVH::testVisibility (BVH/BVH.h:23-189) then traces rays over

* the reference's LBVH topology with race-free boxes (the reference's computeBounds,
  BVH/BVH.cu:217-259, reads sibling boxes without a fence and on the B200 sometimes
  unions a child's zero-filled box; the oracle recomputes the boxes from the same
  topology), and
* that tree after 3 treelet rounds computed by the oracle.  The reference's own
  treelet kernel is never run: it raised an illegal memory access on the B200
  (optimizeBVHImpl, 34-triangle room, first run of this script).

Keys of each fixture (inputs are stored too, so tests never regenerate them):

  pos, idx, mesh_ids              inputs of the build
  bounds                          scene bounds (host fold of Core/Scene.cu:131-135)
  codes, sorted, perm             reference Morton codes, sorted codes, sort order
  merged_ref                      reference node records after mergeNodesArray (as computed, races included)
  merged                          the same topology with race-free boxes/areas/costs (oracle)
  final3                          `merged` after 3 treelet rounds (oracle)
  rays, c_prim, c_t               closest-hit rays (n x 8) and the reference's results on `merged`
  srays, s_limit, s_excl, s_occ   any-hit rays, limits, excluded meshes, reference results on `merged`
  c3_prim, c3_t, s3_occ           the reference's results on `final3` (-3 / 3 when `final3` is
                                  deeper than the reference's 64-entry traversal stack allows)
  depth                           depth of the reference's tree
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cavalry_b200 import scenes  # noqa: E402
from oracle import pyoracle as po  # noqa: E402


def duplicate_soup(n: int):
    pos, idx = scenes.soup(1, seed=99)
    pos = np.tile(pos, (n, 1))
    idx = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    return pos, idx


def flat_soup(n: int, seed: int):
    pos, idx = scenes.soup(n, seed=seed)
    pos = pos.copy()
    pos[:, 2] = 0.5  # zero scene extent along z
    return pos, idx


def cases():
    room = scenes.mini_room()
    n34 = 34
    pos34 = room["positions"]
    idx34 = room["indices"][:n34]
    mesh34 = room["mesh_ids"][:n34]
    yield "room34", pos34, idx34, mesh34, 0, 2048
    yield "room36", room["positions"], room["indices"], room["mesh_ids"], 0, 2048
    p, i = scenes.soup(2, seed=3)
    yield "soup2", p, i, None, 0, 256
    p, i = scenes.soup(1000, seed=11)
    yield "soup1k", p, i, None, 0, 4096
    p, i = scenes.soup(4097, seed=13)
    yield "soup4097", p, i, None, 0, 4096
    p, i = scenes.soup(8000, seed=12)
    yield "soup8k", p, i, None, 0, 8192
    p, i = duplicate_soup(300)
    yield "dup300", p, i, None, 0, 1024
    p, i = flat_soup(2000, seed=14)
    yield "flat2k", p, i, None, 0, 2048


def room_shadow_rays(pos, idx, mesh, m, seed):
    """Shadow rays between random points on triangles and the light (last mesh), with the
    reference's source/target mesh exclusion."""
    rng = np.random.default_rng(seed)
    n = idx.shape[0]
    light_mesh = int(mesh.max())
    light_tris = np.nonzero(mesh == light_mesh)[0]
    src_t = rng.integers(0, n, m)
    dst_t = light_tris[rng.integers(0, len(light_tris), m)]

    def sample(t):
        a, b = rng.uniform(0, 1, (2, len(t)))
        sa = np.sqrt(a)
        w0, w1, w2 = 1 - sa, sa * (1 - b), sa * b
        v = pos[idx[t]].astype(np.float64)
        return w0[:, None] * v[:, 0] + w1[:, None] * v[:, 1] + w2[:, None] * v[:, 2]

    o = sample(src_t).astype(np.float32)
    p = sample(dst_t).astype(np.float32)
    v = (p - o).astype(np.float32)
    dist = np.sqrt((v.astype(np.float64) ** 2).sum(1)).astype(np.float32)
    dist = np.maximum(dist, np.float32(1e-6))
    d = (v / dist[:, None]).astype(np.float32)
    excl = np.stack([mesh[src_t], mesh[dst_t]], axis=1).astype(np.int32)
    return scenes.make_rays(o, d), dist, excl


def main(out_dir: Path):
    out_dir.mkdir(parents=True, exist_ok=True)
    for name, pos, idx, mesh, _rounds, m in cases():
        n = idx.shape[0]
        mesh_arr = np.zeros(n, np.int32) if mesh is None else np.asarray(mesh, np.int32)
        ref = po.RefScene(pos, idx, mesh_ids=mesh_arr, rounds=0, id_mode=1, dump=True)
        o = po.build(pos, idx, codes=ref.codes, rounds=0)
        for f in ("left", "right", "is_leaf"):
            assert np.array_equal(o["merged"][f], ref.merged[f]), f"{name}: oracle topology differs ({f})"
        rays = scenes.closest_rays(m, seed=100 + n)
        if name.startswith("room"):
            # rays from inside the room towards random directions
            rng = np.random.default_rng(7)
            org = rng.uniform(-0.9, 0.9, (m, 3)).astype(np.float32)
            rays = scenes.make_rays(org, scenes._unit_vectors(rng, m).astype(np.float32))
            srays, slim, sexcl = room_shadow_rays(pos, idx, mesh_arr, m, seed=8)
        else:
            srays, slim = scenes.shadow_rays(m, seed=200 + n)
            sexcl = np.full((m, 2), -1, np.int32)
        ref.load_nodes(o["merged"])
        c_prim, c_t, _ = ref.trace_closest(rays)
        s_occ, _ = ref.trace_any(srays, limit=slim, excl=sexcl)
        final3 = po.treelet_rounds(o["merged"], 3)
        ref.load_nodes(final3)
        if ref.depth <= 62:
            c3_prim, c3_t, _ = ref.trace_closest(rays)
            s3_occ, _ = ref.trace_any(srays, limit=slim, excl=sexcl)
        else:
            # deeper than the reference's fixed 64-entry traversal stack (BVH/BVH.h:41):
            # the reference cannot trace this tree safely, so no reference results are stored
            c3_prim = np.full(m, -3, np.int32)
            c3_t = np.zeros(m, np.float32)
            s3_occ = np.full(m, 3, np.uint8)
        np.savez_compressed(
            out_dir / f"{name}.npz", pos=pos, idx=idx, mesh_ids=mesh_arr, bounds=ref.bounds, codes=ref.codes,
            sorted=ref.sorted, perm=ref.perm, merged_ref=ref.merged, merged=o["merged"], final3=final3,
            rays=rays, c_prim=c_prim, c_t=c_t, srays=srays, s_limit=slim, s_excl=sexcl, s_occ=s_occ,
            c3_prim=c3_prim, c3_t=c3_t, s3_occ=s3_occ, depth=np.int32(ref.depth),
        )
        print(f"{name}: n={n} depth={ref.depth} lbvh_cost={o['merged'][0]['cost']:.6g} "
              f"r3_cost={final3[0]['cost']:.6g} hits={(c_prim >= 0).mean():.3f} occluded={s_occ.mean():.3f}")
        ref.free()


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
