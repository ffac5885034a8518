#!/usr/bin/env bash
# Builds oracle/_ref/libhadros_ref.so (and the reference's two cache
# executables and its GPU executable): the reference's own hot-path sources,
# compiled where they lie (read-only, unmodified) with the reference Makefile's
# flags (-O3 -std=c++17 -fopenmp, no -march), plus oracle/ref_driver.cpp.
# Test infrastructure only; outputs go to oracle/_ref/ (git-ignored).
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
# REFERENCE_ROOT defaults to $HADROS_REFERENCE_ROOT, else /root/reference.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref="${1:-${HADROS_REFERENCE_ROOT:-/root/reference}}"
out="$here/_ref"
if [ ! -d "$ref/src" ]; then
    echo "build_ref: no reference sources at $ref; skipping" >&2
    exit 0
fi
mkdir -p "$out"
# where the sources were found, for tests that run the reference's own scripts
printf '%s\n' "$ref" > "$out/REFERENCE_ROOT"
srcs=""
for f in kerr_metric kerr_geodesic kerr_camera sigma_table torus_profile \
         radiative_transfer mev_neutrino_physics; do
    srcs="$srcs $ref/src/$f.cpp"
done
g++ -O3 -std=c++17 -fopenmp -fPIC -shared -I"$ref/include" \
    -o "$out/libhadros_ref.so" $srcs "$here/ref_driver.cpp"
# the reference's own cache writer and cache reader executables (file-format
# compatibility tests)
for app in compute_kerr_geodesics compute_kerr_image_from_cache; do
    g++ -O3 -std=c++17 -fopenmp -I"$ref/include" -o "$out/$app" $srcs "$ref/apps/$app.cpp"
done
# the reference's own GPU executable (a single .cu, reference flags plus the
# B200 target), for the reference-CUDA leg of bench.py
if command -v nvcc >/dev/null 2>&1 || [ -x /usr/local/cuda/bin/nvcc ]; then
    NVCC="$(command -v nvcc || echo /usr/local/cuda/bin/nvcc)"
    "$NVCC" -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a \
        -o "$out/compute_kerr_image_cuda" "$ref/apps/compute_kerr_image_cuda.cu"
fi
echo "built $out/libhadros_ref.so and reference cache executables"
