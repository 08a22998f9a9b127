#!/usr/bin/env bash
# Builds satidev/gct's own code, compiled from its sources where they lie under the reference tree,
# into oracle/_ref/ (TEST INFRASTRUCTURE ONLY; nothing is copied out of the reference tree):
#
#   libgct_ref_host.so  the reference's host-callable functions (ramp taps, rotation analysis,
#                       Parker and cosine weights, projMapping, voxel positions) behind the C
#                       entry points of oracle/ref_host.cu, for the golden vectors and CPU tests;
#   ref_fdk             the reference's CUDA FDK (GCT::Recon::CUDA::reconstruct and everything it
#                       calls) for sm_100a, driven by oracle/ref_fdk_main.cu, for the GPU parity
#                       tests against the reference itself;
#   libgct_ref_io.so    the reference's array-file readers and writers (src/cpp/io) behind the C
#                       entry points of oracle/ref_io.cpp, for the IO golden files;
#   ref_wrappers        the reference's reconstruct() overloads on its own types, defined by this
#                       repository's include/gct_recon_wrappers.hpp over gct_b200/libgct_fdk.so
#                       (built first), driven by oracle/ref_wrappers_main.cpp.
#
# The reference's Eigen submodule is empty in its tree. The translation units used here compile
# without it except for declarations in src/cpp/geom/projection_matrix.h, which
# oracle/eigen_api/ satisfies with a minimal matrix API (the matrices built with it are never read
# by a kernel). The Eigen-dependent sources (geom_math.cpp, eigen_utils.cpp, projection_matrix.cpp,
# proj_geom_cb_factory.cpp) are not compiled; ref_fdk_main.cu defines the two functions of theirs
# the FDK links against.
#
# The reference tree is GCT_REFERENCE_DIR, else the read-only checkout this recipe was written for.
# With --if-present the recipe exits 0 without building when that tree is absent (a machine that
# only runs the prebuilt files).
set -euo pipefail
REF="${GCT_REFERENCE_DIR:-/root/reference}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
    if [ "${1:-}" = "--if-present" ]; then
        exit 0
    fi
    echo "build_ref.sh: reference tree not found at $REF (set GCT_REFERENCE_DIR)" >&2
    exit 1
fi
mkdir -p "$OUT"
NVCC="${NVCC:-nvcc}"
ARCH=(-gencode arch=compute_100a,code=sm_100a)
FLAGS=(-std=c++20 -O2 --expt-relaxed-constexpr --expt-extended-lambda -Xcompiler -fPIC -w -I "$REF/src"
       -I "$HERE/eigen_api" "${ARCH[@]}")

# host functions library
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_host.cu" -o "$OUT/ref_host.o"
CPP=(cpp/recon/ramp_filter.cpp cpp/recon/proj_filt_kernel.cpp cpp/geom/rotation_geom.cpp
     cpp/data/proj_meta_info.cpp cpp/geom/vec_wcs.cpp)
for src in "${CPP[@]}"; do
    g++ -std=c++20 -O2 -fPIC -w -I "$REF/src" -c "$REF/src/$src" -o "$OUT/$(basename "$src" .cpp).o" &
done
wait
"$NVCC" "${ARCH[@]}" -shared -o "$OUT/libgct_ref_host.so" "$OUT/ref_host.o" "$OUT/ramp_filter.o" \
    "$OUT/proj_filt_kernel.o" "$OUT/rotation_geom.o" -lcudart

# the reference's CUDA FDK
CU=(cuda/recon/recon_wrappers.cu cuda/geom/ct_geom_dev.cu cuda/recon/parker_weighting.cu
    cuda/recon/ramp_filtering_fft.cu cuda/utils/check_error.cu cuda/utils/cuda_config.cu)
pids=()
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_fdk_main.cu" -o "$OUT/ref_fdk_main.o" & pids+=($!)
for src in "${CU[@]}"; do
    "$NVCC" "${FLAGS[@]}" -c "$REF/src/$src" -o "$OUT/ref_$(basename "$src" .cu).o" & pids+=($!)
done
for p in "${pids[@]}"; do wait "$p"; done
"$NVCC" "${ARCH[@]}" -o "$OUT/ref_fdk" "$OUT/ref_fdk_main.o" "$OUT"/ref_recon_wrappers.o "$OUT"/ref_ct_geom_dev.o \
    "$OUT"/ref_parker_weighting.o "$OUT"/ref_ramp_filtering_fft.o "$OUT"/ref_check_error.o "$OUT"/ref_cuda_config.o \
    "$OUT/ramp_filter.o" "$OUT/proj_filt_kernel.o" "$OUT/rotation_geom.o" "$OUT/proj_meta_info.o" "$OUT/vec_wcs.o" \
    -lcufft -lcudart
# the reference's array-file readers and writers
IO=(cpp/io/file_reader/meta_img_reader.cpp cpp/io/file_reader/array_file_reader.cpp
    cpp/io/file_reader/den_file_reader.cpp cpp/io/file_reader/raw_data_file_reader.cpp cpp/io/file_utils.cpp
    cpp/io/string_utils.cpp cpp/io/file_writer/meta_img_file_writer.cpp)
g++ -std=c++20 -O2 -fPIC -w -I "$REF/src" -shared -o "$OUT/libgct_ref_io.so" "$HERE/ref_io.cpp" \
    "${IO[@]/#/$REF/src/}"
# the drop-in overloads on the reference's types, over this repository's library
REPO="$(cd "$HERE/.." && pwd)"
g++ -std=c++20 -O2 -w -I "$REF/src" -I "$REPO/include" -I "$HERE" -o "$OUT/ref_wrappers" "$HERE/ref_wrappers_main.cpp" \
    "$OUT/rotation_geom.o" "$OUT/vec_wcs.o" "$OUT/proj_meta_info.o" -L "$REPO/gct_b200" -lgct_fdk \
    -Wl,-rpath,'$ORIGIN/../../gct_b200'
echo "$OUT/libgct_ref_host.so $OUT/ref_fdk $OUT/libgct_ref_io.so $OUT/ref_wrappers"
