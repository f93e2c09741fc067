#!/usr/bin/env bash
# Builds the reference implementation (FTSPolySol) from its own sources, where
# they lie, into oracle/_ref/ -- test infrastructure only (a checker and the
# reference arm of bench.py), never part of the product.
#
#   oracle/_ref/main         the unmodified reference executable (its Makefile
#                            recipe: nvcc -O3 -std=c++17 <arch> *.cu -lcufft -lcurand)
#   oracle/_ref/ref_harness  the reference's sources minus main.cu, linked with
#                            oracle/ref_harness.cu (golden-vector dumps, timing)
#
# Usage: oracle/build_ref.sh [REFERENCE_DIR]
#   REFERENCE_DIR defaults to $FTSP_REFERENCE_DIR, else to a directory named
#   "reference" beside the repository.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${FTSP_REFERENCE_DIR:-$HERE/../../reference}}"
OUT="$HERE/_ref"
ARCH="-gencode arch=compute_100a,code=sm_100a"
FLAGS="-O3 -std=c++17"
if [ ! -f "$REF/complexLangevin.cu" ]; then
    echo "build_ref: reference sources not found in $REF" >&2
    exit 1
fi
mkdir -p "$OUT/obj"
pids=()
for src in "$REF"/*.cu; do
    base="$(basename "$src" .cu)"
    obj="$OUT/obj/$base.o"
    if [ ! -f "$obj" ] || [ "$src" -nt "$obj" ]; then
        nvcc $FLAGS $ARCH -I"$REF" -c "$src" -o "$obj" &
        pids+=($!)
    fi
done
hobj="$OUT/obj/ref_harness.o"
if [ ! -f "$hobj" ] || [ "$HERE/ref_harness.cu" -nt "$hobj" ]; then
    nvcc $FLAGS $ARCH -I"$REF" -c "$HERE/ref_harness.cu" -o "$hobj" &
    pids+=($!)
fi
for p in "${pids[@]}"; do wait "$p"; done
objs=()
for src in "$REF"/*.cu; do
    base="$(basename "$src" .cu)"
    [ "$base" = "main" ] && continue
    objs+=("$OUT/obj/$base.o")
done
nvcc $FLAGS $ARCH -o "$OUT/main" "${objs[@]}" "$OUT/obj/main.o" -lcufft -lcurand
nvcc $FLAGS $ARCH -o "$OUT/ref_harness" "${objs[@]}" "$hobj" -lcufft -lcurand
echo "build_ref: built $OUT/main and $OUT/ref_harness"
