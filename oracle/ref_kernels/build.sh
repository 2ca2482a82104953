#!/bin/bash
# Builds the reference's own CUDA kernels (test-only checker) from the reference
# sources in place.  Output goes to oracle/_ref/ only (git-ignored; it travels
# with the repository snapshot to the GPU machine).  The reference's meson build
# is not used.
#   libref_kernels.so   cast, beamformer, detector and channelizer kernels
#                       (+ cuFFT), compiled as ordinary host + device code once a
#                       blade_config.hh defines the three version macros the
#                       headers expect;
#   ref_*.cubin         polarizer, gather (accumulate) and permutation kernels,
#                       device code only (ref_device_only.cu explains why), one
#                       kernel per cubin.
# The reference checkout is $BLADE_REFERENCE, else a `reference` directory beside
# this repository.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/../_ref"
REF="${BLADE_REFERENCE:-$HERE/../../../reference}"
if [ ! -d "$REF/src/modules" ]; then
    echo "reference sources not found (set BLADE_REFERENCE): $REF" >&2
    exit 1
fi
mkdir -p "$OUT/include"
cat > "$OUT/include/blade_config.hh" <<'CFG'
#define BLADE_VERSION_STR "reference"
#define BLADE_COMMIT_STR "reference"
#define BLADE_BUILD_TYPE "release"
CFG
FLAGS=(-std=c++20 --expt-relaxed-constexpr -O2 -gencode arch=compute_100a,code=sm_100a -w
       -I "$REF" -I "$REF/include" -I "$OUT/include" -I "$HERE")
nvcc "${FLAGS[@]}" -Xcompiler -fPIC -shared "$HERE/ref_kernels.cu" -o "$OUT/libref_kernels.so" -lcufft
names=(polarizer_cf32 polarizer_cf16 gather_cf32 permutation_cf32)
for i in 1 2 3 4; do
    nvcc "${FLAGS[@]}" -cubin -DREF_PICK=$i "$HERE/ref_device_only.cu" -o "$OUT/ref_${names[$((i - 1))]}.cubin"
done
echo "$OUT/libref_kernels.so"
