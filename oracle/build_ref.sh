#!/bin/sh
# Builds, from the reference's own sources where they lie, into oracle/_ref/
# only (checkers, never part of the product):
#   ref_gar_helpers  oracle/ref_gar_helpers.cu against the reference's GAR
#                    filter headers (pins oracle/gar.py's restated helpers);
#   ref_gar_match    oracle/ref_gar_match_main.cu with the reference's
#                    core/task/gpu_task/kernel/kernel_gar_match.cu (its GPU
#                    GARMatch kernels; run by tests/test_gar_ref_gpu.py).
# Needs the reference sources (not present on GPU boxes; the built programs
# travel with the repository snapshot) and nvcc; exits 0 without them.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${MG_REFERENCE_DIR:-/root/reference}
[ -d "$REF/core" ] || exit 0
command -v nvcc >/dev/null 2>&1 || exit 0
mkdir -p "$HERE/_ref"
nvcc -std=c++17 -O1 -gencode arch=compute_100a,code=sm_100a -diag-suppress 20012 -I "$REF" -o "$HERE/_ref/ref_gar_helpers" "$HERE/ref_gar_helpers.cu"
nvcc -std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a -diag-suppress 20012,20013,550,177 -I "$REF" -o "$HERE/_ref/ref_gar_match" "$HERE/ref_gar_match_main.cu" "$REF/core/task/gpu_task/kernel/kernel_gar_match.cu"
