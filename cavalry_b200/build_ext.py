"""Build the cavalry_b200 CUDA library in-tree for sm_100a.

    python -m cavalry_b200.build_ext          # builds cavalry_b200/libcavalry_b200.so

Each ``csrc/*.cu`` file is compiled with the reference's numerics flags
(``-use_fast_math``, Cavalry's CMakeLists.txt:5) for ``sm_100a`` and linked into one
shared library with a plain C ABI (``include/cavalry.h``).  Objects go to
``cavalry_b200/_build`` (not committed); the ``.so`` sits next to this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcavalry_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "-use_fast_math",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O3",
    "-I",
    str(ROOT / "include"),
]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _compile(src: Path, extra: list[str]) -> Path:
    obj = BUILD / (src.stem + src.suffix.replace(".", "_") + ".o")
    deps = [src, *CSRC.glob("*.cuh"), *CSRC.glob("*.h"), ROOT / "include" / "cavalry.h"]
    if obj.exists() and obj.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return obj
    if src.suffix == ".cpp":  # host C++ (the .pbrt loader): plain g++ through nvcc
        cmd = [nvcc(), "-std=c++17", "-O2", "-Xcompiler", "-fPIC,-O2", "-I", str(ROOT / "include"), "-x", "c++",
               "-c", str(src), "-o", str(obj)]
    else:
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra or []), srcs))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lz"]  # zlib: PNG textures
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    if verbose:
        print(f"built {LIB}")
    return LIB


CLI_SRC = PKG / "cli" / "cavalry_main.cpp"
CLI = PKG / "cavalry"


def build_cli(verbose: bool = False) -> Path:
    """The `cavalry` command-line renderer, linked against the in-tree library."""
    lib = build(verbose=verbose)
    if CLI.exists() and CLI.stat().st_mtime >= max(CLI_SRC.stat().st_mtime, lib.stat().st_mtime):
        return CLI
    cmd = ["g++", "-std=c++17", "-O2", "-o", str(CLI), str(CLI_SRC), "-L", str(PKG), "-lcavalry_b200",
           "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"CLI link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {CLI}")
    return CLI


def ptxas_report() -> str:
    """Register/spill/shared-memory report of every kernel (ptxas -v)."""
    out = []
    for src in sorted(CSRC.glob("*.cu")):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-Xptxas", "-v", "-c", str(src), "-o", os.devnull]
        r = subprocess.run(cmd, capture_output=True, text=True)
        out.append(f"== {src.name}\n{r.stderr}")
    return "\n".join(out)


if __name__ == "__main__":
    if "--ptxas" in sys.argv:
        print(ptxas_report())
    else:
        build(verbose=True)
        build_cli(verbose=True)
