#!/usr/bin/env bash
# Builds the reference program (mGPUKDE_tiled) from its own, unmodified
# sources where they lie, into oracle/_ref/mgkde_ref.  Test infrastructure:
# the binary pins the FP64 oracle (tests/golden/make_golden.py), is the timed
# "reference" CPU baseline (its OpenMP path, skip_gpu_parallel=1), and its
# own CUDA path (skip_omp_parallel=1, mode 1, h_option -1: the edge-weight and
# tile-density kernels, read for bounds before it first ran) is the bench's
# second comparator on the GPU.
#
# What it takes to compile the Windows/GDAL sources on Linux, without editing
# them:
#   -I oracle/ref_shim     windows.h (GlobalMemoryStatusEx) and a small GDAL
#                          stand-in built on csrc/tiff_io.hpp
#   -include cfloat/climits  DBL_MAX, FLT_MAX, ULLONG_MAX used without includes
#   -Dfalse=0              kde_cuda_kdtr_tiled.cu:568 passes `false` for a
#                          float* argument (accepted by MSVC only)
#   -D_FORTIFY_SOURCE=0    kde_cuda_kdtr_tiled.cu:2055-2057 strcpy()s the
#                          projection into a buffer one byte short
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REPO="$(dirname "$HERE")"
SRC="${REFERENCE_ROOT:-/root/reference}"
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -f "$SRC/kde_cuda_kdtr_tiled.cu" ]; then
  echo "reference sources not found under $SRC" >&2
  exit 2
fi
nvcc -std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a \
  -Xcompiler -fopenmp -Xcompiler -fpermissive \
  -Xcompiler -U_FORTIFY_SOURCE -Xcompiler -D_FORTIFY_SOURCE=0 \
  -Dfalse=0 -include cfloat -include climits \
  -I "$HERE/ref_shim" -I "$REPO/mgpukde_tiled_b200/csrc" -I "$SRC" \
  "$SRC/kde_cuda_kdtr_tiled.cu" "$SRC/KDtree.cu" "$SRC/CUDA_KDtree.cu" \
  -o "$OUT/mgkde_ref" -lgomp -w
echo "$OUT/mgkde_ref"
