#!/usr/bin/env bash
# Builds the reference VVM step (AB2 + WATER + KESSLER_MICROPHY) from its own
# sources, where they lie under the reference checkout, into
# oracle/_ref/libvvmref.so: a serial build (no -fopenmp). The reference's
# OpenMP loops share loop temporaries between threads (e.g. src/Advection.cpp:26,
# src/Buoyancy.cpp:12-18), so only the serial build is a valid oracle.
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
# reading the reference's own input/init.txt. With REF_VARIANT=stream it
# builds oracle/_ref/libvvmref_stream.so from oracle/ref_config_stream.hpp
# (the streamfunction formulation, STREAMFUNCTION; POISSONPARAM = 0). With
# REF_VARIANT=dropin it builds oracle/_ref/libvvmref_dropin.so: the model as a
# maintainer would build it with GPU_STEP, i.e. every unit as above except
# that TimeMarching comes from the committed binding
# 2d-vector-vorticity-model_b200/integration/Iteration_GPU.cpp, linked
# against libvvmgpu.so (built first). src/Iteration.cpp is compiled with its
# TimeMarching renamed (-DTimeMarching=TimeMarching_cpu), which is what the
# maintainer's `#ifndef GPU_STEP` around it achieves.
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
elif [ "${REF_VARIANT:-}" = stream ]; then
    CONFIG="$HERE/ref_config_stream.hpp"
    LIB=libvvmref_stream.so
    OBJ="$OUT/obj_stream"
    EXTRA="-DPOISSONPARAM=0.0"
elif [ "${REF_VARIANT:-}" = dropin ]; then
    LIB=libvvmref_dropin.so
    OBJ="$OUT/obj_dropin"
    EXTRA="-DGPU_STEP -I$HERE/../include"
fi
mkdir -p "$OBJ"
CXX=${CXX:-g++}
FLAGS="-std=c++17 -O3 -fPIC -w -I$REF/include -I$SRC $EXTRA"
UNITS="Advection Boundary Buoyancy MicroPhysics Turbulent NumericalProcess PoissonSolver Iteration AddForcing Init"

# The streamfunction routine (src/PoissonSolver.cpp:124-177) has three more
# compile errors, all in its own lines, mended on the way to g++ for that
# variant only: it names `dx` without `model.` (line 133) and calls the halo
# routines with the field alone, without nx and nz (lines 168, 179, 180).
STREAM_FIX=()
if [ "${REF_VARIANT:-}" = stream ]; then
    STREAM_FIX=(-e 's/zetap\[i\]\[k\] \* dx \* dx;/zetap[i][k] * model.dx * model.dx;/'
                -e 's/BoundaryProcess2D_\(westdown\|center\)(model\.\(psi\|u\|w\));/BoundaryProcess2D_\1(model.\2, model.nx, model.nz);/')
fi

emit_unit() {  # $1 = path of the .cpp to append after the shared header
    cat "$CONFIG"
    sed '/#include "Config.hpp"/d' "$SRC/Declare.hpp"
    sed -e '/#include "Declare.hpp"/d' -e '/pb_lev_all/d' -e '/radiation_heating_rate/d' "${STREAM_FIX[@]}" "$1"
}

ALL="$UNITS ref_harness"
LINK=""
if [ "${REF_VARIANT:-}" = dropin ]; then
    ALL="$ALL Iteration_GPU"
    GPULIB="$HERE/../2d-vector-vorticity-model_b200/lib"
    LINK="-L$GPULIB -lvvmgpu -Wl,-rpath,\$ORIGIN/../../2d-vector-vorticity-model_b200/lib"
fi
pids=""
for u in $ALL; do
    uflags=""
    case "$u" in
        ref_harness) f="$HERE/ref_harness.cpp" ;;
        Iteration_GPU) f="$HERE/../2d-vector-vorticity-model_b200/integration/Iteration_GPU.cpp" ;;
        Iteration) f="$SRC/$u.cpp"
                   if [ "${REF_VARIANT:-}" = dropin ]; then uflags="-DTimeMarching=TimeMarching_cpu"; fi ;;
        *) f="$SRC/$u.cpp" ;;
    esac
    ( emit_unit "$f" | $CXX $FLAGS $uflags -x c++ -c - -o "$OBJ/$u.o" ) &
    pids="$pids $!"
done
for p in $pids; do wait "$p"; done
objs=""
for u in $ALL; do objs="$objs $OBJ/$u.o"; done
# link the shared libstdc++ explicitly: with a static copy inside the .so,
# std::cout is never constructed when the host process has no libstdc++ loaded
$CXX -shared -o "$OUT/$LIB" $objs $LINK -l:libstdc++.so.6
echo "built $OUT/$LIB"
