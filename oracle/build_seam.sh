#!/usr/bin/env bash
# Build the reference's OWN, unmodified MhdSolver2D (src/physics/mhd/
# mhd_solver.cpp and the numerics registry it dispatches through) over this
# project's CUDA kernels: the per-kernel seam of kernels.hpp defined by
# oracle/seam/mhd_kernels_b200.cpp over include/quasar_mhd_launch.h, and the
# device runtime of device.hpp by oracle/seam/device_cuda.cpp.  Output:
# oracle/_ref/libquasar_mhd_seam.so, with the same qref_* C entry points as
# the CPU build (oracle/ref_capi.cpp).  Test infrastructure only: the GPU tests
# use it to check that the reference's driver runs unchanged on this backend.
# The reference sources are compiled where they lie; nothing is copied.
#
#   REF=/path/to/quasar oracle/build_seam.sh     (after quasar_b200/build.py)
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(cd "$HERE/.." && pwd)
if [ -z "${REF:-}" ]; then
  echo "$(basename "$0"): set REF to the quasar source tree" >&2
  exit 2
fi
CUDA=${CUDA_HOME:-/usr/local/cuda}
OUT=$HERE/_ref
OBJ=$OUT/obj_seam
LIB=$ROOT/quasar_b200/_lib
if [ ! -d "$REF/src/physics/mhd" ]; then
  echo "build_seam: reference tree not found at $REF" >&2
  exit 2
fi
if [ ! -f "$LIB/libquasar_mhd_b200.so" ]; then
  echo "build_seam: build quasar_b200 first ($LIB/libquasar_mhd_b200.so missing)" >&2
  exit 2
fi
mkdir -p "$OBJ"
# -fno-gnu-unique and the export map keep the reference's registry singletons
# private to this library: the CPU build of the reference (libquasar_mhd_ref.so)
# registers the same factory names, and a process may load both
FLAGS="-std=c++20 -O2 -fPIC -fopenmp -ffp-contract=off -fno-gnu-unique -w -I$REF/include -I$REF/src"
HOSTSRC="src/physics/mhd/mhd_solver.cpp src/numerics/flux_reconstruction.cpp
 src/numerics/hlld_riemann.cpp src/numerics/ct_scheme.cpp
 src/numerics/ssprk_integrator.cpp src/numerics/positivity_limiter.cpp
 src/physics/mhd/mhd_boundary.cpp src/numerics/radial_tables.cpp
 src/numerics/mhd_background_profile.cpp src/physics/mhd/initial_conditions.cpp
 src/numerics/mhd_state.cpp"
pids=()
for f in $HOSTSRC; do
  g++ $FLAGS -c "$REF/$f" -o "$OBJ/h_$(basename "$f" .cpp).o" & pids+=($!)
done
for f in device_cuda mhd_kernels_b200; do
  g++ $FLAGS -I"$ROOT/include" -I"$CUDA/include" -c "$HERE/seam/$f.cpp" -o "$OBJ/s_$f.o" &
  pids+=($!)
done
g++ $FLAGS -c "$HERE/ref_capi.cpp" -o "$OBJ/ref_capi.o" & pids+=($!)
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
if [ $rc -ne 0 ]; then echo "build_seam: compile failed" >&2; exit 1; fi
g++ -shared -fopenmp -Wl,--no-undefined -Wl,--version-script="$HERE/seam/exports.map" "$OBJ"/*.o -o "$OUT/libquasar_mhd_seam.so" \
    -L"$LIB" -lquasar_mhd_b200 -L"$CUDA/lib64" -lcudart \
    -Wl,-rpath,'$ORIGIN/../../quasar_b200/_lib' -Wl,-rpath,"$CUDA/lib64"
echo "built $OUT/libquasar_mhd_seam.so"
