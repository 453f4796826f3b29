#!/usr/bin/env bash
# Compiles the one part of the reference path that builds from its own
# sources: the header-only RNG include/XoshiroCpp.hpp, driven by
# oracle/ref_xoshiro_main.cpp. Output: oracle/_ref/xoshiro_golden.
# The rest of the reference needs lattice_lib, FFTW3, HDF5, argparse and
# Eigen, none of which exist here, so it is not built.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref="${PYRO_REFERENCE_DIR:-/root/reference}"
mkdir -p "$here/_ref"
if [ ! -f "$ref/include/XoshiroCpp.hpp" ]; then
  echo "reference tree not present at $ref; nothing to build" >&2
  exit 0
fi
${CXX:-g++} -O2 -std=c++20 -I"$ref/include" "$here/ref_xoshiro_main.cpp" -o "$here/_ref/xoshiro_golden"
echo "built $here/_ref/xoshiro_golden"
