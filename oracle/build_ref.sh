#!/usr/bin/env bash
# Test infrastructure: builds the reference's own BVH code into oracle/_ref/libcavref.so.
#
# No reference source is copied.  A symlink farm under oracle/_ref/src points at the
# reference files where they lie, except Core/TriangleMesh.h and
# Core/IntersectionResult.h, which point at the narrow shims in oracle/ref_shim
# (the real headers pull in the scene/material/variant layers that the BVH path never
# touches).  BVH/BVH.cu and BVH/Optimization.cu are compiled verbatim, with the
# reference's numerics flags (CMakeLists.txt:5: -use_fast_math), for sm_100a.
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT
set -euo pipefail
REF="${1:?usage: oracle/build_ref.sh REFERENCE_ROOT}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
SRC="$OUT/src"

if [ ! -f "$REF/BVH/BVH.cu" ]; then
    echo "build_ref: reference not found at $REF; skipping" >&2
    exit 0
fi

rm -rf "$SRC"
mkdir -p "$SRC/BVH" "$SRC/Utils" "$SRC/Core" "$SRC/harness"
for f in BVH.cu BVH.h BVHNode.h Optimization.cu Optimization.h SAH.h; do
    ln -s "$REF/BVH/$f" "$SRC/BVH/$f"
done
for f in GpuCommons.h MathsCommons.h Utils.h Timer.h Array.h; do
    ln -s "$REF/Utils/$f" "$SRC/Utils/$f"
done
for f in BoundingBox.h Triangle.h Ray.h VisibilityTest.h; do
    ln -s "$REF/Core/$f" "$SRC/Core/$f"
done
ln -s "$HERE/ref_shim/Core/TriangleMesh.h" "$SRC/Core/TriangleMesh.h"
ln -s "$HERE/ref_shim/Core/IntersectionResult.h" "$SRC/Core/IntersectionResult.h"
ln -s "$HERE/ref_harness.cu" "$SRC/harness/ref_harness.cu"

NVCC="${NVCC:-nvcc}"
"$NVCC" -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -use_fast_math --extended-lambda \
    -w -I "$REF/Dependencies/include" -Xcompiler -fPIC -shared \
    -o "$OUT/libcavref.so" "$SRC/harness/ref_harness.cu"
echo "build_ref: wrote $OUT/libcavref.so"
