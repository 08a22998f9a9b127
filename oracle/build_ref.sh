#!/usr/bin/env bash
# Compiles satidev/gct's own host-callable sources, where they lie under the reference tree, with
# the harness oracle/ref_host.cu into oracle/_ref/libgct_ref_host.so (TEST INFRASTRUCTURE ONLY).
#
# Only translation units that build without the reference's missing Eigen submodule are used:
#   src/cpp/recon/ramp_filter.cpp, src/cpp/recon/proj_filt_kernel.cpp, src/cpp/geom/rotation_geom.cpp
# and the header-only __host__ __device__ functions included by ref_host.cu. Nothing is copied
# out of the reference tree; outputs go to oracle/_ref/ only.
set -euo pipefail
REF="${GCT_REFERENCE_DIR:-/root/reference}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
    echo "build_ref.sh: reference tree not found at $REF" >&2
    exit 1
fi
mkdir -p "$OUT"
NVCC="${NVCC:-nvcc}"
FLAGS=(-std=c++20 -O2 --expt-relaxed-constexpr -Xcompiler -fPIC -I "$REF/src" -gencode arch=compute_100a,code=sm_100a)
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_host.cu" -o "$OUT/ref_host.o"
for src in cpp/recon/ramp_filter.cpp cpp/recon/proj_filt_kernel.cpp cpp/geom/rotation_geom.cpp; do
    g++ -std=c++20 -O2 -fPIC -I "$REF/src" -c "$REF/src/$src" -o "$OUT/$(basename "$src" .cpp).o"
done
"$NVCC" -shared -o "$OUT/libgct_ref_host.so" "$OUT/ref_host.o" "$OUT/ramp_filter.o" "$OUT/proj_filt_kernel.o" \
    "$OUT/rotation_geom.o" -lcudart
echo "$OUT/libgct_ref_host.so"
