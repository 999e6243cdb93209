#!/usr/bin/env bash
# Test infrastructure: builds the reference renderer (the whole Cavalry executable) into
# oracle/_ref/cavalry_ref, for render-parity fixtures of the wavefront integrators.
#
# The reference targets MSVC.  Six compile-only fixes are needed for nvcc + GCC; they
# are applied with sed to a scratch copy OUTSIDE this repository (nothing of the
# reference is copied into the repo) and change no behaviour:
#   1. Utils/Variant.h: `variant :: variant<typename Ts...>` -> `variant::variant<Ts...>`,
#      and drop the explicit `template<>` in front of the copy constructor;
#   2. `is_base_of<X, typename T>` -> `is_base_of<X, T>` in the *Object.h visitors;
#   3. Dependencies/include/variant/variant.h: std::declval<...>() of the visitor's
#      return-type deductions as lvalue references (`&`);
#   4. Core/Scene.h: drop `mutable` from two pointer members;
#   5. Utils/TaskQueue.h: include <thrust/sort.h> and <thrust/execution_policy.h>;
#   6. main.cu: `auto& result =` -> `auto result =` (binds a temporary).
# Build flags follow CMakeLists.txt:5 (-use_fast_math --extended-lambda -std=c++17) for
# sm_100a.  The renderer must always be run with --bvh-opt-rounds 0: its treelet kernel
# faulted on the B200 (see oracle/ref_harness.cu).
#
# Usage: CAV_REF_WORK=SCRATCH_DIR oracle/build_ref_full.sh REFERENCE_ROOT
# SCRATCH_DIR receives the patched copy and the objects; it must lie outside this repository.
set -euo pipefail
REF="${1:?usage: CAV_REF_WORK=SCRATCH_DIR oracle/build_ref_full.sh REFERENCE_ROOT}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
WORK="${CAV_REF_WORK:?set CAV_REF_WORK to a scratch directory outside the repository}"
case "$(cd "$(dirname "$WORK")" && pwd)/" in
    "$(cd "$HERE/.." && pwd)/"*) echo "build_ref_full: CAV_REF_WORK must lie outside the repository" >&2; exit 2 ;;
esac
if [ ! -f "$REF/main.cu" ]; then
    echo "build_ref_full: reference not found at $REF; skipping" >&2
    exit 0
fi
rm -rf "$WORK"
mkdir -p "$WORK" "$OUT"
cp -r "$REF"/. "$WORK/src"
S="$WORK/src"
sed -i 's/variant :: variant<typename Ts\.\.\.>/variant::variant<Ts...>/' "$S/Utils/Variant.h"
sed -i '/^\s*template<>\s*$/d' "$S/Utils/Variant.h"
for f in SceneLoading/Lexing.h Cameras/CameraObject.h BSDFs/BSDFObject.h Samplers/SamplerObject.h \
         Lights/LightObject.h Filters/FilterObject.h Materials/MaterialObject.h; do
    sed -i 's/is_base_of<\([A-Za-z_]*\), *typename T>/is_base_of<\1, T>/g' "$S/$f"
done
V="$S/Dependencies/include/variant/variant.h"
sed -i 's/std::declval<H>()/std::declval<H\&>()/g' "$V"
sed -i 's/std::declval<typename unwrapped<typename S::head_type>::type>()/std::declval<typename unwrapped<typename S::head_type>::type\&>()/g' "$V"
sed -i 's/std::declval<typename Variant::cons_type::head_type>()/std::declval<typename Variant::cons_type::head_type\&>()/g' "$V"
sed -i 's/Primitive\* mutable primitives/Primitive* primitives/; s/LightObject\* mutable lights/LightObject* lights/' "$S/Core/Scene.h"
sed -i '0,/#pragma once/s//#pragma once\n#include <thrust\/sort.h>\n#include <thrust\/execution_policy.h>/' "$S/Utils/TaskQueue.h"
sed -i 's/auto& result = setup.renderer.render/auto result = setup.renderer.render/' "$S/main.cu"

NVCC="${NVCC:-nvcc}"
mkdir -p "$WORK/obj"
cd "$S"
find . -name '*.cu' -not -path './Dependencies/*' | sort > "$WORK/sources.txt"
xargs -P "${CAV_REF_JOBS:-8}" -I{} sh -c \
    "\"$NVCC\" -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -use_fast_math --extended-lambda -w \
     -I Dependencies/include -I Core -I . -c '{}' -o \"$WORK/obj/\$(echo '{}' | tr '/.' '__').o\"" \
    < "$WORK/sources.txt"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -o "$OUT/cavalry_ref" "$WORK"/obj/*.o -lcurand
echo "build_ref_full: wrote $OUT/cavalry_ref"
