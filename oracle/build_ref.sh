#!/usr/bin/env bash
# Builds the reference (ParallelPopGen 3P, read-only at $REF; default: a checkout named `reference`
# beside this repository) into oracle/_ref/ for use as a test oracle.  Compiles the reference's own sources where they lie, with its own flags
# (examples/*/makefile: -O3 --use_fast_math, relocatable device code).  The reference's legacy
# __shfl/__ballot calls only compile for a pre-Volta virtual architecture, so the PTX target is
# compute_60 and ptxas lowers it to sm_100a machine code.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${REF:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
if [ ! -d "$REF/3P" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
CODE="--generate-code arch=compute_60,code=sm_100a"
FLAGS="-O3 --use_fast_math -rdc=true -Wno-deprecated-gpu-targets -w -I $REF/3P"
set -x
"$NVCC" $CODE $FLAGS -c "$REF/3P/_internal/shared.cu" -o "$OUT/shared.o"
"$NVCC" $CODE $FLAGS -c "$REF/3P/_internal/go_fish_impl.cu" -o "$OUT/go_fish_impl.o"
"$NVCC" $CODE $FLAGS -c "$REF/3P/_internal/spectrum.cu" -o "$OUT/spectrum.o"
"$NVCC" $CODE $FLAGS -c "$HERE/ref_driver.cu" -o "$OUT/ref_driver.o"
"$NVCC" $CODE -Wno-deprecated-gpu-targets "$OUT/ref_driver.o" "$OUT/shared.o" "$OUT/go_fish_impl.o" "$OUT/spectrum.o" -o "$OUT/ref_driver"
