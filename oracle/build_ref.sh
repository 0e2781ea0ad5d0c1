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
