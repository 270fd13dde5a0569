#!/usr/bin/env bash
# Build the reference's OWN MHD hot path for the host CPU into
# oracle/_ref/libquasar_mhd_ref.so (test infrastructure: parity oracle and the
# timed CPU baseline).  The reference sources are compiled where they lie,
# unmodified, with the HIP->CPU shim in oracle/shim; nothing is copied.
#
#   REF=/path/to/quasar oracle/build_ref.sh
#
# Sources: src/backend/hip/mhd/*.hip (as C++), src/physics/mhd/mhd_solver.cpp,
# the numerics registry .cpp files and the MHD boundary registry.  Flags follow
# the reference's own fp-contract=off rule for the scaled-arithmetic modules
# (scaled_arithmetic.hpp:22-23); x86-64 g++ emits no FMA contraction anyway.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
if [ -z "${REF:-}" ]; then
  echo "$(basename "$0"): set REF to the quasar source tree" >&2
  exit 2
fi
OUT=$HERE/_ref
OBJ=$OUT/obj
if [ ! -d "$REF/src/backend/hip/mhd" ]; then
  echo "build_ref: reference tree not found at $REF" >&2
  exit 2
fi
mkdir -p "$OBJ"
FLAGS="-std=c++20 -O2 -fPIC -fopenmp -ffp-contract=off -U_FORTIFY_SOURCE -D_FORTIFY_SOURCE=0 -w -I$REF/include -I$REF/src"
KERNELS="mhd_reconstruct mhd_riemann mhd_ct mhd_update mhd_reduce mhd_split_energy
 mhd_initial_conditions mhd_collocation mhd_cell_sums mhd_boundary_hip
 mhd_background_validate mhd_background_build mhd_background_momentum
 mhd_cylindrical_momentum mhd_halo"
HOSTSRC="src/physics/mhd/mhd_solver.cpp src/numerics/flux_reconstruction.cpp
 src/numerics/hlld_riemann.cpp src/numerics/ct_scheme.cpp
 src/numerics/ssprk_integrator.cpp src/numerics/positivity_limiter.cpp
 src/physics/mhd/mhd_boundary.cpp src/numerics/radial_tables.cpp
 src/numerics/mhd_background_profile.cpp src/physics/mhd/initial_conditions.cpp
 src/numerics/mhd_state.cpp"
pids=()
for k in $KERNELS; do
  g++ $FLAGS -x c++ -include "$HERE/shim/hip/hip_runtime.h" -I"$HERE/shim" \
      -c "$REF/src/backend/hip/mhd/$k.hip" -o "$OBJ/k_$k.o" & pids+=($!)
done
for f in $HOSTSRC; do
  g++ $FLAGS -c "$REF/$f" -o "$OBJ/h_$(basename "$f" .cpp).o" & pids+=($!)
done
g++ $FLAGS -c "$HERE/ref_backend.cpp" -o "$OBJ/ref_backend.o" & pids+=($!)
g++ $FLAGS -include "$HERE/shim/hip/hip_runtime.h" -I"$HERE/shim" \
    -c "$HERE/ref_capi.cpp" -o "$OBJ/ref_capi.o" & pids+=($!)
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
if [ $rc -ne 0 ]; then echo "build_ref: compile failed" >&2; exit 1; fi
g++ -shared -fopenmp "$OBJ"/*.o -o "$OUT/libquasar_mhd_ref.so"
echo "built $OUT/libquasar_mhd_ref.so"
