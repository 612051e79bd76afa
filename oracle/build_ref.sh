#!/usr/bin/env bash
# Builds the unmodified Vship reference (CUDA backend) from its own sources, in place
# under /root/reference, into oracle/_ref/libvship_ref.so for sm_100a.  Same recipe as the
# reference's Makefile "buildcuda" target (Makefile:42-43) with the architecture pinned.
# The library is only a checker and a timing baseline: the product never links it.
set -euo pipefail
REF=${VSHIP_REFERENCE_ROOT:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/VshipLib.cpp" ]; then
    echo "reference sources not found at $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
if [ "$OUT/libvship_ref.so" -nt "$REF/src/VshipLib.cpp" ] && [ "$OUT/libvship_ref.so" -nt "$0" ]; then
    exit 0
fi
nvcc -x cu "$REF/src/VshipLib.cpp" -O3 -std=c++17 -I "$REF/include" \
    -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fPIC \
    -Xlinker -Bsymbolic -o "$OUT/libvship_ref.so.tmp"
mv "$OUT/libvship_ref.so.tmp" "$OUT/libvship_ref.so"
echo "built $OUT/libvship_ref.so"
