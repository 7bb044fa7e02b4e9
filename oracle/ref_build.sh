#!/usr/bin/env bash
# Builds the reference's own CUDA launchers — redi/redi_kernel.cu
# (`redi_cuda_launch_`) and redi/opt_kernel.cu (`redi_opt_launch`) — from the
# reference sources where they lie, into oracle/_ref/libredi_refcuda.so.
# Test infrastructure only: used on a B200 to generate the golden vectors that
# pin the CPU oracle (tests/golden/make_golden.py).
#
# Built exactly as the reference's Makefile builds them (redi/Makefile:57-63:
# -O3, -I../common, -DMODEL_NZ_STACK_MAX=128 -DWITH_CUDA) except for two flags:
# the target is sm_100a, and FMA contraction is off (-fmad=false) so the
# result is the IEEE sequence of the source, comparable bit for bit.
set -euo pipefail
REF="${REDI_REFERENCE_DIR:-/root/reference}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
if [[ ! -f "$REF/redi/redi_kernel.cu" ]]; then
  echo "ref_build.sh: reference sources not found under $REF; skipping" >&2
  exit 0
fi
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
mkdir -p "$OUT"
FLAGS=(-O3 -gencode arch=compute_100a,code=sm_100a -fmad=false -I"$REF/common" -I"$REF/redi"
       --compiler-options -fPIC -DMODEL_NZ_STACK_MAX=128 -DWITH_CUDA)
LIB="$OUT/libredi_refcuda.so"
# The same launchers built with the reference's own flags only (FMA contraction
# on, as its Makefile builds them), for timing the reference on this GPU
# (oracle/time_reference_cuda.py); not used for parity.
NATIVE="$OUT/libredi_refcuda_native.so"
if [[ -f "$LIB" && -f "$NATIVE" && "$LIB" -nt "$REF/redi/redi_kernel.cu" && "$LIB" -nt "$REF/redi/opt_kernel.cu" \
      && "$LIB" -nt "$0" && "$NATIVE" -nt "$0" ]]; then
  exit 0
fi
"$NVCC" "${FLAGS[@]}" -c "$REF/redi/redi_kernel.cu" -o "$OUT/redi_kernel.o"
"$NVCC" "${FLAGS[@]}" -c "$REF/redi/opt_kernel.cu" -o "$OUT/opt_kernel.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$LIB" "$OUT/redi_kernel.o" "$OUT/opt_kernel.o"
echo "built $LIB"
NFLAGS=(-O3 -gencode arch=compute_100a,code=sm_100a -I"$REF/common" -I"$REF/redi"
        --compiler-options -fPIC -DMODEL_NZ_STACK_MAX=128 -DWITH_CUDA)
"$NVCC" "${NFLAGS[@]}" -c "$REF/redi/redi_kernel.cu" -o "$OUT/redi_kernel_native.o"
"$NVCC" "${NFLAGS[@]}" -c "$REF/redi/opt_kernel.cu" -o "$OUT/opt_kernel_native.o"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -shared -o "$NATIVE" "$OUT/redi_kernel_native.o" "$OUT/opt_kernel_native.o"
echo "built $NATIVE"
