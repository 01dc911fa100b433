#!/usr/bin/env bash
# Build the UNMODIFIED reference C++ core (src/bindings.cpp and its headers, read
# in place from the reference checkout) into the host CPU oracle, using the
# SYCL / mdspan shims in oracle/shim/.  Outputs go to oracle/_ref/ only:
#   oracle/_ref/fp64/cpp_core<EXT>   (egg::real = double)
#   oracle/_ref/fp32/cpp_core<EXT>   (egg::real = float, -DEGG_REAL_IS_FP32=1)
#   oracle/_ref/fp64snap/cpp_core<EXT> (fp64, parallel loops run serially with the
#                                     shared-node refreshes before the ghost fills)
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or set EGG_REFERENCE_ROOT)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${EGG_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
  echo "usage: build_ref.sh REFERENCE_ROOT (or set EGG_REFERENCE_ROOT)" >&2
  exit 2
fi
if [ ! -f "$REF/src/bindings.cpp" ]; then
  echo "build_ref.sh: reference sources not found under $REF" >&2
  exit 2
fi
PY="${PYTHON:-python}"
PYINC="$($PY -c 'import sysconfig;print(sysconfig.get_paths()["include"])')"
PBINC="$($PY -c 'import pybind11;print(pybind11.get_include())')"
EXT="$($PY -c 'import sysconfig;print(sysconfig.get_config_var("EXT_SUFFIX"))')"
# -ffp-contract=off keeps the oracle's fp64 arithmetic unfused; -march=x86-64-v3
# (AVX2/FMA) so the binary also runs on the GPU hosts' CPUs.
FLAGS=(-std=c++23 -O3 -march=x86-64-v3 -ffp-contract=off -fopenmp -shared -fPIC -w
       -I"$HERE/shim" -I"$REF/src" -I"$PYINC" -I"$PBINC")
mkdir -p "$HERE/_ref/fp64" "$HERE/_ref/fp32" "$HERE/_ref/fp64snap"
g++ "${FLAGS[@]}" "$REF/src/bindings.cpp" -o "$HERE/_ref/fp64/cpp_core$EXT" &
p1=$!
g++ "${FLAGS[@]}" -DEGG_REAL_IS_FP32=1 "$REF/src/bindings.cpp" -o "$HERE/_ref/fp32/cpp_core$EXT" &
p2=$!
# serial, race-free ordering of the shim's parallel loops (see oracle/shim/sycl/sycl.hpp)
g++ "${FLAGS[@]}" -DEGG_SHIM_SNAPSHOT=1 "$REF/src/bindings.cpp" -o "$HERE/_ref/fp64snap/cpp_core$EXT" &
p3=$!
wait $p1
wait $p2
wait $p3
echo "built $HERE/_ref/{fp64,fp32,fp64snap}/cpp_core$EXT"
