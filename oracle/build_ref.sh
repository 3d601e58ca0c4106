#!/bin/bash
# Build the reference CPU solvers from their own sources, where they lie, into
# oracle/_ref/ (git-ignored).  Used only as a checker and as the timed CPU
# baseline; nothing in the product links these binaries.
#
#   oracle/_ref/lbm3d-perm         LMB3d/lbm3d-perm.cpp with its own flags (LMB3d/make_perm.sh:15)
#   oracle/_ref/lbm3d-perm-tau0.8  the same source with the one TAU constant
#                                  (LMB3d/lbm3d-perm.cpp:112) set to 0.8, edited
#                                  on the fly in a pipe (no copy is written)
#   oracle/_ref/lbm2d-perm         LMB2d/main.cpp + LMB2d/lbm.cpp, -O3 as in
#                                  LMB2d/make_perm.sh:7, against oracle/stub/Magick++.h
#                                  (.dat/.ppm input only)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${REF:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/LMB3d/lbm3d-perm.cpp" ]; then
    echo "reference sources not found under $REF; skipping the reference build" >&2
    exit 0
fi
mkdir -p "$OUT"
FLAGS3D="-O3 -march=broadwell -ffast-math"
g++ $FLAGS3D -o "$OUT/lbm3d-perm.new" "$REF/LMB3d/lbm3d-perm.cpp"
mv -f "$OUT/lbm3d-perm.new" "$OUT/lbm3d-perm"

PAT='^static const double TAU     = 1\.0;'
if [ "$(grep -c "$PAT" "$REF/LMB3d/lbm3d-perm.cpp")" != "1" ]; then
    echo "TAU line not found exactly once; cannot build the tau=0.8 variant" >&2
    exit 1
fi
sed "s/$PAT/static const double TAU     = 0.8;/" "$REF/LMB3d/lbm3d-perm.cpp" \
    | g++ $FLAGS3D -x c++ - -o "$OUT/lbm3d-perm-tau0.8.new"
mv -f "$OUT/lbm3d-perm-tau0.8.new" "$OUT/lbm3d-perm-tau0.8"

g++ -O3 -I"$HERE/stub" -o "$OUT/lbm2d-perm.new" "$REF/LMB2d/main.cpp" "$REF/LMB2d/lbm.cpp"
mv -f "$OUT/lbm2d-perm.new" "$OUT/lbm2d-perm"
echo "built reference solvers in $OUT"
