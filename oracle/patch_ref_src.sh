#!/usr/bin/env bash
# Copy the reference's src/ tree into a scratch directory and apply the
# mechanical GCC-compatibility edits it needs (it was written for MSVC, which
# does not do two-phase name lookup).  The copy is build scratch for the
# oracle binary only: it is never committed and the product never uses it.
#   $1 = reference root (contains src/), $2 = destination directory
# Edits (all semantic no-ops):
#   array.h:36, mesh_function.h:64, coord_mesh_function.h:113
#       -> `using Base::member;` for members of dependent base classes
#   coarse_grids_hierarchy.h:75  min(...)  -> std::min(...)
#   loads_calculator.h:1386      sprintf_s -> provided by ref_compat.h
set -euo pipefail
REF="$1"; DST="$2"
rm -rf "$DST"; mkdir -p "$DST"
cp -r "$REF/src" "$DST/src"
chmod -R u+w "$DST/src"
M="$DST/src/Base/MeshFunctions"
python3 - "$M" "$DST/src/Base/CoarseGrid/coarse_grids_hierarchy.h" <<'PY'
import sys, re
mdir, cgh = sys.argv[1], sys.argv[2]
def inject(path, header, base):
    s = open(path, encoding='utf-8', errors='surrogateescape').read()
    i = s.index(header)
    j = s.index('{', i) + 1
    using = ''.join(f' using {base}::{m};' for m in ('size', 'Vector', 'capasity', 'getCopy'))
    s = s[:j] + using + s[j:]
    open(path, 'w', encoding='utf-8', errors='surrogateescape').write(s)
inject(f'{mdir}/array.h', 'struct ArrayCPU : ArrayInterface<ElemType>', 'ArrayInterface<ElemType>')
inject(f'{mdir}/mesh_function.h', 'struct MeshFunction : Array<ElemType>', 'Array<ElemType>')
inject(f'{mdir}/coord_mesh_function.h', 'struct CoordMeshFunction : Array<coord<ElemType>>', 'Array<coord<ElemType>>')
s = open(cgh, encoding='utf-8', errors='surrogateescape').read()
s = s.replace('min(min(m_A->m_N, m_A->m_M), m_A->m_K)', 'std::min(std::min(m_A->m_N, m_A->m_M), m_A->m_K)')
open(cgh, 'w', encoding='utf-8', errors='surrogateescape').write(s)
PY
