#!/bin/bash
# Compiles the reference's own CUDA sources, where they lie under $REF_ROOT
# (default /root/reference, the read-only mount of the reference tree), with the test-only harnesses of oracle/ref_harness into
# oracle/_ref/ (git-ignored; the built .so files are copied with the
# working tree to the GPU machine).  Used only to produce golden vectors of the reference and
# to time the reference's own GPU loop (oracle/ref_gpu_timing.py).
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_ROOT="${REF_ROOT:-/root/reference}"
REF="$REF_ROOT/code/cuda"
OUT="$HERE/_ref"
[ -d "$REF" ] || { echo "reference tree not mounted; nothing to build"; exit 0; }
mkdir -p "$OUT"
FLAGS="-std=c++14 -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -shared -w"
HYB="$REF/SG-tSNE-HYB/sgtsnepi/src"
nvcc $FLAGS -I"$HYB/cuda" -I"$HYB" -o "$OUT/libref_hyb.so" "$HERE/ref_harness/ref_hyb.cu" \
  "$HYB/cuda/Frep.cu" "$HYB/cuda/nuconv.cu" "$HYB/cuda/gridding.cu" \
  "$HYB/cuda/non_periodic_convF.cu" "$HYB/cuda/non_periodic_convD.cu" -lcufft
CU="$REF/SG-tSNE-CUDA/src"
nvcc $FLAGS -I"$CU" -o "$OUT/libref_cu.so" "$HERE/ref_harness/ref_cu.cu" \
  "$CU/pq.cu" "$CU/Frep.cu" "$CU/nuconv.cu" "$CU/gridding.cu" \
  "$CU/non_periodic_convF.cu" "$CU/non_periodic_convD.cu" "$CU/utils.cu" \
  "$CU/gradient_descend.cu" "$CU/compute_error.cu" "$CU/perplexity_search.cu" -lcufft -lcublas
# the lambda bisection kernel: graph_rescaling.cu alone, with a shim for the
# four legacy cuSPARSE routines of its (unused) symmetrisation code
nvcc $FLAGS -I"$CU" -include "$HERE/ref_harness/cusparse_legacy_shim.h" \
  -o "$OUT/libref_rescale.so" "$HERE/ref_harness/ref_rescale.cu" "$CU/graph_rescaling.cu" -lcusparse
echo "built $OUT/libref_hyb.so $OUT/libref_cu.so $OUT/libref_rescale.so"
