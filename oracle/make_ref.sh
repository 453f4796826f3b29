#!/usr/bin/env bash
# Compiles the parts of the reference path that build from their own sources,
# where they lie in the reference tree (given as $1 or PYRO_REFERENCE_DIR),
# into oracle/_ref/ (git-ignored; the outputs travel with the repository):
#  * _ref/xoshiro_golden: the header-only RNG include/XoshiroCpp.hpp, driven by
#    oracle/ref_xoshiro_main.cpp;
#  * _ref/libref_mc.so: the reference's own Monte Carlo code, src/MC.cpp,
#    compiled unchanged with oracle/ref_mc_main.cpp (C entry points) against
#    the stand-ins in oracle/ref_shim/ for what MC.cpp includes but this image
#    lacks (lattice_lib's Supercell and vector types, HDF5 and json
#    declarations, the FFTW-backed ssf_manager). -O3 without -march, like the
#    oracle and the reference's release build.
# The rest of the reference (its drivers, ssf_manager, Luttinger-Tisza) needs
# argparse, FFTW3, HDF5 and Eigen, none of which exist here, so it is not built.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref="${1:-${PYRO_REFERENCE_DIR:-}}"
if [ -z "$ref" ]; then
  echo "usage: make_ref.sh <reference tree>  (or set PYRO_REFERENCE_DIR)" >&2
  exit 2
fi
mkdir -p "$here/_ref"
if [ ! -f "$ref/include/XoshiroCpp.hpp" ]; then
  echo "reference tree not present at $ref; nothing to build" >&2
  exit 0
fi
CXX="${CXX:-g++}"
"$CXX" -O2 -std=c++20 -I"$ref/include" "$here/ref_xoshiro_main.cpp" -o "$here/_ref/xoshiro_golden"
echo "built $here/_ref/xoshiro_golden"
if [ -f "$ref/src/MC.cpp" ]; then
  tmp="$here/_ref/obj"
  mkdir -p "$tmp"
  flags=(-O3 -std=c++20 -fPIC -I"$here/ref_shim" -I"$ref/include")
  "$CXX" "${flags[@]}" -c "$ref/src/MC.cpp" -o "$tmp/MC.o"
  "$CXX" "${flags[@]}" -c "$here/ref_mc_main.cpp" -o "$tmp/ref_mc_main.o"
  "$CXX" -shared -o "$here/_ref/libref_mc.so" "$tmp/ref_mc_main.o" "$tmp/MC.o"
  echo "built $here/_ref/libref_mc.so"
fi
