#!/usr/bin/env bash
# Builds the reference VVM step (AB2 + WATER + KESSLER_MICROPHY) from its own
# sources, where they lie under the reference checkout, into
# oracle/_ref/libvvmref.so: a serial build (no -fopenmp). The reference's
# OpenMP loops share loop temporaries between threads (e.g. src/Advection.cpp:26,
# src/Buoyancy.cpp:12-18), so only the serial build is a valid oracle; this
# image also ships no libgomp, so an OpenMP build does not link here.
#
# Test infrastructure only. No reference source is written to disk: each
# translation unit reaches g++ on stdin as
#     oracle/ref_config.hpp                    (flags in place of src/Config.hpp)
#   + src/Declare.hpp without its `#include "Config.hpp"`
#   + src/<unit>.cpp without its `#include "Declare.hpp"`
# with two lines dropped on the way, both of which name members that exist
# only in builds this oracle does not use:
#   src/Init.cpp:260        model.pb_lev_all[...]             (P3 only)
#   src/AddForcing.cpp:20   model.radiation_heating_rate[...] (RRTMGP only)
# Eigen is the copy vendored with the reference (include/Eigen, 3.3.91).
#
# usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
# With REF_VARIANT=tropical it builds oracle/_ref/libvvmref_tropical.so from
# oracle/ref_config_tropical.hpp instead (sounding file and Q1/Q2 forcing on),
# reading the reference's own input/init.txt.
set -euo pipefail
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
SRC="$REF/src"
if [ ! -f "$SRC/Declare.hpp" ]; then
    echo "build_ref.sh: reference sources not found under $REF" >&2
    exit 1
fi
CONFIG="$HERE/ref_config.hpp"
LIB=libvvmref.so
OBJ="$OUT/obj"
EXTRA=""
if [ "${REF_VARIANT:-}" = tropical ]; then
    CONFIG="$HERE/ref_config_tropical.hpp"
    LIB=libvvmref_tropical.so
    OBJ="$OUT/obj_tropical"
    EXTRA="-DREF_INIT_PATH=\"$REF/input/init.txt\""
fi
mkdir -p "$OBJ"
CXX=${CXX:-g++}
FLAGS="-std=c++17 -O3 -fPIC -w -I$REF/include -I$SRC $EXTRA"
UNITS="Advection Boundary Buoyancy MicroPhysics Turbulent NumericalProcess PoissonSolver Iteration AddForcing Init"

emit_unit() {  # $1 = path of the .cpp to append after the shared header
    cat "$CONFIG"
    sed '/#include "Config.hpp"/d' "$SRC/Declare.hpp"
    sed -e '/#include "Declare.hpp"/d' -e '/pb_lev_all/d' -e '/radiation_heating_rate/d' "$1"
}

pids=""
for u in $UNITS ref_harness; do
    if [ "$u" = ref_harness ]; then f="$HERE/ref_harness.cpp"; else f="$SRC/$u.cpp"; fi
    ( emit_unit "$f" | $CXX $FLAGS -x c++ -c - -o "$OBJ/$u.o" ) &
    pids="$pids $!"
done
for p in $pids; do wait "$p"; done
objs=""
for u in $UNITS ref_harness; do objs="$objs $OBJ/$u.o"; done
# link the shared libstdc++ explicitly: with a static copy inside the .so,
# std::cout is never constructed when the host process has no libstdc++ loaded
$CXX -shared -o "$OUT/$LIB" $objs -l:libstdc++.so.6
echo "built $OUT/$LIB"
