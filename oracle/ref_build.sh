#!/usr/bin/env bash
# Builds the reference's own CUDA launchers from the reference sources where
# they lie, into oracle/_ref/. Test infrastructure only: used on a B200 to
# generate the golden vectors that pin the CPU oracles (tests/golden/) and to
# time the reference's CUDA beside this repository's kernels.
#
#   libredi_refcuda.so   redi/redi_kernel.cu (`redi_cuda_launch_`) and
#                        redi/opt_kernel.cu (`redi_opt_launch`)
#   libmeke_refcuda.so   meke/meke_kernel.cu (`meke_cuda_launch`) and
#                        meke/opt_kernel.cu (`meke_opt_launch`)
#   libale_refcuda.so    ale_remap/ale_kernel.cu (`ale_remap_cuda`) and
#                        ale_remap/opt_kernel.cu (`ale_remap_opt`)
#
# Built as the reference's Makefiles build them (redi/Makefile:57-63: -O3,
# -I../common, -DMODEL_NZ_STACK_MAX=128 -DWITH_CUDA; meke/Makefile CUFLAGS:
# -O3, -I../common -I.; ale_remap/Makefile CUFLAGS: -O3, -I../common,
# -DMODEL_NZ_STACK_MAX=128) except for two flags: the target is sm_100a, and FMA
# contraction is off (-fmad=false) so the result is the IEEE sequence of the
# source, comparable bit for bit. The *_native.so twins keep the reference's
# own flags (FMA contraction on) and are used only for timing.
#
# The reference checkout is $REDI_REFERENCE_DIR, or else a directory named
# `reference` beside this repository's root.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${REDI_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
OUT="$HERE/_ref"
if [[ ! -f "$REF/redi/redi_kernel.cu" ]]; then
  echo "ref_build.sh: reference sources not found under $REF; skipping" >&2
  exit 0
fi
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
ARCH=(-gencode arch=compute_100a,code=sm_100a)
mkdir -p "$OUT"

# build_pair <name> <srcdir> <extra flags...> -- <sources...>
build_pair() {
  local name="$1" dir="$2"; shift 2
  local extra=()
  while [[ "$1" != "--" ]]; do extra+=("$1"); shift; done
  shift
  local srcs=("$@")
  local lib="$OUT/lib${name}_refcuda.so" native="$OUT/lib${name}_refcuda_native.so"
  local fresh=1
  for s in "${srcs[@]}"; do
    [[ -f "$lib" && -f "$native" && "$lib" -nt "$dir/$s" && "$lib" -nt "$0" && "$native" -nt "$0" ]] || fresh=0
  done
  [[ $fresh == 1 ]] && return 0
  local objs=() nobjs=()
  for s in "${srcs[@]}"; do
    local b="${s%.cu}"
    "$NVCC" -O3 "${ARCH[@]}" -fmad=false -I"$REF/common" -I"$dir" --compiler-options -fPIC "${extra[@]}" \
      -c "$dir/$s" -o "$OUT/${name}_${b}.o"
    "$NVCC" -O3 "${ARCH[@]}" -I"$REF/common" -I"$dir" --compiler-options -fPIC "${extra[@]}" \
      -c "$dir/$s" -o "$OUT/${name}_${b}_native.o"
    objs+=("$OUT/${name}_${b}.o"); nobjs+=("$OUT/${name}_${b}_native.o")
  done
  "$NVCC" "${ARCH[@]}" -shared -o "$lib" "${objs[@]}"
  "$NVCC" "${ARCH[@]}" -shared -o "$native" "${nobjs[@]}"
  echo "built $lib $native"
}

build_pair redi "$REF/redi" -DMODEL_NZ_STACK_MAX=128 -DWITH_CUDA -- redi_kernel.cu opt_kernel.cu
if [[ -f "$REF/meke/meke_kernel.cu" ]]; then
  build_pair meke "$REF/meke" -- meke_kernel.cu opt_kernel.cu
fi
if [[ -f "$REF/ale_remap/ale_kernel.cu" ]]; then
  build_pair ale "$REF/ale_remap" -DMODEL_NZ_STACK_MAX=128 -- ale_kernel.cu opt_kernel.cu
fi

# The reference's CUDA transcriptions of eos_specvol_derivs (WRIGHT_97 and
# LINEAR), one per model that carries one, run through oracle/ref_eos_harness.cu
# (built with each model's own size definitions, FMA contraction off).
build_eos() {
  local name="$1" dir="$2" macro="$3" src="$4"; shift 4
  local lib="$OUT/libeos_${name}_refcuda.so"
  if [[ -f "$lib" && "$lib" -nt "$dir/$src" && "$lib" -nt "$HERE/ref_eos_harness.cu" && "$lib" -nt "$0" ]]; then
    return 0
  fi
  "$NVCC" -O3 "${ARCH[@]}" -fmad=false -I"$REF/common" -I"$dir" --compiler-options -fPIC "$@" -D"$macro" \
    -shared "$HERE/ref_eos_harness.cu" -o "$lib"
  echo "built $lib"
}
if [[ -f "$REF/epbl/epbl_kernel.cu" ]]; then
  build_eos epbl "$REF/epbl" REF_EOS_EPBL epbl_kernel.cu \
    -DMODEL_NZ_STACK_MAX=128 -DEPBL_LB_THREADS=128 -DEPBL_LB_BLOCKS_PER_SM=4
fi
if [[ -f "$REF/kappa_shear/ks_kernel.cu" ]]; then
  build_eos ks "$REF/kappa_shear" REF_EOS_KS ks_kernel.cu -DMODEL_NZ_STACK_MAX=128 -DKS_FULL_COPY
fi
