#!/bin/sh
# Builds oracle/_ref/ref_gar_helpers: a host program of this repository
# (oracle/ref_gar_helpers.cu) compiled against the reference's own headers
# where they lie, for pinning the GAR oracle's restated helpers.  Output goes
# only to oracle/_ref/.  Needs the reference sources (not present on GPU
# boxes) and nvcc; exits 0 without them.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${MG_REFERENCE_DIR:-/root/reference}
[ -d "$REF/core" ] || exit 0
command -v nvcc >/dev/null 2>&1 || exit 0
mkdir -p "$HERE/_ref"
nvcc -std=c++17 -O1 -gencode arch=compute_100a,code=sm_100a -diag-suppress 20012 -I "$REF" -o "$HERE/_ref/ref_gar_helpers" "$HERE/ref_gar_helpers.cu"
