"""Test infrastructure: builds the C oracle and (when the reference sources exist) the
reference harness.

    python -m oracle.build [REFERENCE_ROOT]

* ``oracle/_build/libcavoracle.so`` from ``cav_oracle.c`` and ``pt_oracle.c`` (gcc; -ffp-contract=off so
  that only the explicit fmaf/fma calls contract, OpenMP for the timed CPU baseline).
* ``oracle/_ref/libcavref.so`` from the reference's own BVH sources via
  ``build_ref.sh`` (nvcc, sm_100a).  The reference tree is given as an argument or by the
  ``CAVALRY_REFERENCE`` environment variable; without one (or when it is absent) the step
  is skipped and an earlier build, if any, is kept.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
ORACLE_LIB = BUILD / "libcavoracle.so"
REF_LIB = HERE / "_ref" / "libcavref.so"


def build_oracle(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = [HERE / "cav_oracle.c", HERE / "pt_oracle.c"]
    if not force and ORACLE_LIB.exists() and ORACLE_LIB.stat().st_mtime >= max(p.stat().st_mtime for p in srcs):
        return ORACLE_LIB
    tmp = ORACLE_LIB.with_suffix(".tmp.so")
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           "-o", str(tmp), *map(str, srcs), "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def build_ref(reference_root: str | os.PathLike | None = None, force: bool = False) -> Path | None:
    root = reference_root or os.environ.get("CAVALRY_REFERENCE")
    if not root or not (Path(root) / "BVH" / "BVH.cu").exists():
        return REF_LIB if REF_LIB.exists() else None
    deps = [HERE / "ref_harness.cu", HERE / "build_ref.sh", *sorted((HERE / "ref_shim").rglob("*.h"))]
    if not force and REF_LIB.exists() and REF_LIB.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return REF_LIB
    subprocess.run(["bash", str(HERE / "build_ref.sh"), str(root)], check=True)
    return REF_LIB


if __name__ == "__main__":
    import sys

    print(build_oracle())
    print(build_ref(sys.argv[1] if len(sys.argv) > 1 else None))
