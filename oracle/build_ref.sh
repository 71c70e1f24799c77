#!/usr/bin/env bash
# Compile the reference's own CUDA operator kernels (GPU-IMPACT-CT src/*_launcher.cu, which
# #include their *_kernel.cu) from the reference tree, unchanged, into oracle/_ref/libref_kernels.so.
# Test infrastructure only: the GPU pin tests run them on the same inputs as the oracle to pin
# the oracle's restatement to the reference's implementation.  Nothing is copied into this repo.
#   usage: oracle/build_ref.sh path/to/GPU-IMPACT-CT   (or IMPACT_REFERENCE_ROOT in the environment)
set -euo pipefail
REF="${1:-${IMPACT_REFERENCE_ROOT:-}}"
[ -n "$REF" ] || { echo "usage: $0 path/to/GPU-IMPACT-CT (or set IMPACT_REFERENCE_ROOT)"; exit 2; }
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
SRC="$REF/src"
[ -d "$SRC" ] || { echo "reference tree not found at $REF; skipping"; exit 0; }
mkdir -p "$OUT/obj"
NVCC="${NVCC:-nvcc}"
CCBIN=""
[ -x /usr/bin/g++ ] && CCBIN="-ccbin /usr/bin/g++"
# jor_kernel_launcher.cu is left out on purpose: its kernel updates rel in place (a data race
# between neighbouring threads), so its values are not a reproducible pin.
LAUNCHERS="gradient_kernel_launcher.cu divergence_kernel_launcher.cu divergence2_kernel_launcher.cu
helmholtz_explicit_kernel_launcher.cu Nonlinear_upwind_kernel_launcher.cu
interpolate2_pre_vel_kernel_launcher.cu interpolate2_vel_pre_kernel_launcher.cu axpby_kernel_launcher.cu
jacobi_kernel_launcher.cu product_dg_relax_kernel_launcher.cu set_pressure_BC_kernel_launcher.cu
get_ghost_launcher.cu"
OBJS=""
for f in $LAUNCHERS; do
  o="$OUT/obj/${f%.cu}.o"
  if [ ! -f "$o" ] || [ "$SRC/$f" -nt "$o" ]; then
    $NVCC $CCBIN -gencode arch=compute_100a,code=sm_100a -O3 -Xcompiler -fPIC -w -I"$SRC" -c "$SRC/$f" -o "$o"
  fi
  OBJS="$OBJS $o"
done
$NVCC $CCBIN -gencode arch=compute_100a,code=sm_100a -shared -cudart static -o "$OUT/libref_kernels.so" $OBJS
echo "$OUT/libref_kernels.so"
