#!/bin/bash
# Builds the reference's own CUDA kernels (test-only checker) from the reference
# sources in place: /root/reference/src/modules/{cast,beamformer,detector,
# channelizer}/*.cu.  Output goes to oracle/_ref/ only (git-ignored; it travels
# with the repository snapshot to the GPU machine).  The reference's meson build is
# not used: the four kernel files compile directly with nvcc once a
# blade_config.hh defines the three version macros the headers expect.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/../_ref"
REF="${BLADE_REFERENCE:-/root/reference}"
mkdir -p "$OUT/include"
cat > "$OUT/include/blade_config.hh" <<'CFG'
#define BLADE_VERSION_STR "reference"
#define BLADE_COMMIT_STR "reference"
#define BLADE_BUILD_TYPE "release"
CFG
nvcc -std=c++20 --expt-relaxed-constexpr -O2 -gencode arch=compute_100a,code=sm_100a \
    -Xcompiler -fPIC -shared -w \
    -I "$REF" -I "$REF/include" -I "$OUT/include" -I "$HERE" \
    "$HERE/ref_kernels.cu" -o "$OUT/libref_kernels.so" -lcufft
echo "$OUT/libref_kernels.so"
