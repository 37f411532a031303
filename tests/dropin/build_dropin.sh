#!/usr/bin/env bash
# Builds the reference's own test programs and its heat-diffusion-2d example, UNMODIFIED from the
# reference tree, against this repository's include/ tree and libxkb200.so -- the drop-in check of
# the C and C++ source APIs. Outputs go to tests/dropin/_bin/ (git-ignored; the binaries travel
# with the repository to GPU machines, where tests/test_dropin_gpu.py runs them). The reference
# tree is only read, and only here.
#
# Usage: tests/dropin/build_dropin.sh REFERENCE_ROOT   (or XK_REFERENCE_ROOT in the environment)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REPO="$(cd "$HERE/../.." && pwd)"
REF="${1:-${XK_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
    echo "usage: $0 REFERENCE_ROOT (or set XK_REFERENCE_ROOT)" >&2
    exit 2
fi
if [ ! -d "$REF/tests" ] || [ ! -d "$REF/examples/heat-diffusion-2d" ]; then
    echo "build_dropin.sh: reference tree not found at $REF; skipping" >&2
    exit 0
fi
OUT="$HERE/_bin"
mkdir -p "$OUT"
CUDA="${CUDA_HOME:-/usr/local/cuda}"
LIBDIR="$REPO/xkaapi_b200"
# the binaries find libxkb200.so relative to themselves, wherever the repository is copied
RPATH='-Wl,-rpath,$ORIGIN/../../../xkaapi_b200'
CXXFLAGS="-std=c++20 -O2 -I$REPO/include -I$CUDA/include"

for t in task-dependency task-dependency-interval task-dependency-interval-matrix task-dependency-handle task-format-host \
         init deinit sync task-format task-gpu-empty memory-register-async-legacy memory-register-assisted \
         memory-register-assisted-unregister; do
    g++ $CXXFLAGS -o "$OUT/$t" "$REF/tests/$t.cc" -L"$LIBDIR" -lxkb200 "$RPATH"
done
gcc -std=c11 -O2 -I"$REPO/include" -o "$OUT/task-with-access" "$REF/tests/api/c/task-with-access.c" -L"$LIBDIR" -lxkb200 "$RPATH"

HEAT="$REF/examples/heat-diffusion-2d"
"$CUDA/bin/nvcc" -gencode arch=compute_100a,code=sm_100a -O2 -I"$HEAT/include" -c "$HEAT/src/kernels/diffusion.cu" -o "$OUT/diffusion.o"
g++ $CXXFLAGS -I"$HEAT/include" -c "$HEAT/src/main.cc" -o "$OUT/heat-main.o"
g++ -o "$OUT/heat-diffusion-2d" "$OUT/heat-main.o" "$OUT/diffusion.o" -L"$LIBDIR" -lxkb200 -L"$CUDA/lib64" -lcudart \
    -L"$CUDA/lib64/stubs" -lcuda "$RPATH"
rm -f "$OUT/diffusion.o" "$OUT/heat-main.o"
echo "built the reference's tests and heat example into $OUT"
