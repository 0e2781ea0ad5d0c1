#!/usr/bin/env bash
# Build the reference-backed oracle binary oracle/_ref/ref_harness from the
# reference's own sources (test infrastructure only).  The reference tree is
# copied to a scratch directory, given the mechanical GCC-compatibility edits
# of patch_ref_src.sh, compiled together with ref_harness.cpp, and the scratch
# copy is deleted.  Only the binary lands in oracle/_ref/ (git-ignored).
#   REF_ROOT (default /root/reference) -- where the reference checkout lives.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_ROOT="${REF_ROOT:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF_ROOT/src" ]; then
    echo "reference sources not found at $REF_ROOT; oracle/_ref not rebuilt" >&2
    exit 0
fi
mkdir -p "$OUT"
SCRATCH="$(mktemp -d /tmp/lsg_ref_src.XXXXXX)"
trap 'rm -rf "$SCRATCH"' EXIT
"$HERE/patch_ref_src.sh" "$REF_ROOT" "$SCRATCH/ref"
# -O2 (g++ 13 at -O3 miscompiles the reference's restrict-qualified CSR
# builders, e.g. the even-even-even restriction portrait), no -march=native:
# the binary also runs on the GPU hosts, whose CPU
# model differs from the build container's.  No -ffast-math (IEEE FP64).
g++ -std=c++17 -O2 -fopenmp -fpermissive -w \
    -include "$HERE/ref_compat.h" -DCONFIG_PATH=\"/tmp\" \
    -I"$SCRATCH/ref/src" \
    "$HERE/ref_harness.cpp" "$SCRATCH/ref/src/Base/profiler.cpp" \
    -o "$OUT/ref_harness"
echo "built $OUT/ref_harness"

# The drop-in build: the same harness with PoissonDiscreteEquation's solver
# ladder given the one branch a maintainer adds for the B200 library
# (include/lsstag_b200_adapter.hpp): -DLS_STAG_USE_B200 selects
# B200MGFGMRES, which calls liblsstag_b200.so through the C ABI.  Built only
# when the library has been built (make -C ls-stag-3d_parallel_b200).
REPO="$(cd "$HERE/.." && pwd)"
LIBDIR="$REPO/ls-stag-3d_parallel_b200/lib"
if [ -f "$LIBDIR/liblsstag_b200.so" ]; then
    python3 - "$SCRATCH/ref/src/DiscreteEquations/poisson_discrete_equation.h" <<'PY'
import sys
p = sys.argv[1]
s = open(p, encoding='utf-8', errors='surrogateescape').read()
inc = '// ================================================================== SYNOPSIS'
i = s.index(inc)
s = s[:i] + '#ifdef LS_STAG_USE_B200\n#include "lsstag_b200_adapter.hpp"\n#endif\n' + s[i:]
ladder = '#ifdef LS_STAG_USE_CUDA'
first = s.index(ladder)
second = s.index(ladder, first + 1)          # the solver member's ladder
s = s[:second] + '#if defined(LS_STAG_USE_B200)\n    B200MGFGMRES solver;\n#elif defined(LS_STAG_USE_CUDA)' + \
    s[second + len(ladder):]
open(p, 'w', encoding='utf-8', errors='surrogateescape').write(s)
PY
    g++ -std=c++17 -O2 -fopenmp -fpermissive -w -DLS_STAG_USE_B200 \
        -include "$HERE/ref_compat.h" -DCONFIG_PATH=\"/tmp\" \
        -I"$SCRATCH/ref/src" -I"$REPO/include" \
        "$HERE/ref_harness.cpp" "$SCRATCH/ref/src/Base/profiler.cpp" \
        -L"$LIBDIR" -llsstag_b200 -Wl,-rpath,'$ORIGIN/../../ls-stag-3d_parallel_b200/lib' \
        -o "$OUT/ref_harness_b200"
    echo "built $OUT/ref_harness_b200"
fi
