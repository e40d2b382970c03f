#!/usr/bin/env bash
# Builds the reference's own CPU hot-path code (Vlasiator, GPL-2.0-or-later)
# into oracle/_ref/ as a parity oracle and CPU baseline.  Nothing from the
# reference is copied into this repository: the reference sources are
# symlinked from where they lie into a build tree under oracle/_ref/src, the
# few headers that pull in MPI / dccrg / phiprof are replaced by the small
# stand-ins in oracle/ref_shim, and only the shared objects are written.
#
#   oracle/_ref/libvlasov_ref_sp.so  : FP32 VDF (Realf=float, Real=double), VECL=16, PPM
#   oracle/_ref/libvlasov_ref_dp.so  : all-FP64 (Realf=double), VECL=8, PPM
#   oracle/_ref/libvlasov_ref_sp_pqm.so, libvlasov_ref_sp_plm.so : FP32, PQM / PLM acceleration
#   oracle/_ref/libvlasov_ref_sp_dropin.so : the FP32 build plus the C++ drop-in layer
#                                           (include/vlgpu.hpp) over libvlgpu.so, for its tests
#
# Usage: oracle/build_ref.sh [reference_root]   (default $VLASIATOR_REF, else /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${VLASIATOR_REF:-/root/reference}}"
OUT="$HERE/_ref"
SRC="$OUT/src"
if [ ! -f "$REF/vlasovsolver/cpu_acc_map.cpp" ]; then
  echo "build_ref: reference tree not found at $REF" >&2
  exit 3
fi
rm -rf "$SRC"
mkdir -p "$SRC/vlasovsolver" "$SRC/spatial_cells" "$SRC/arch" "$SRC/sysinc"
for f in cpu_acc_map.cpp cpu_acc_map.hpp cpu_acc_sort_blocks.cpp cpu_acc_sort_blocks.hpp \
         cpu_acc_load_blocks.cpp cpu_acc_load_blocks.hpp cpu_1d_plm.hpp cpu_1d_ppm.hpp \
         cpu_1d_pqm.hpp cpu_1d_ppm_nonuniform.hpp cpu_face_estimates.hpp cpu_slope_limiters.hpp \
         vec.h vectorclass_fallback.h arch_moments.h cpu_trans_map_amr.hpp cpu_trans_pencils.hpp; do
  ln -s "$REF/vlasovsolver/$f" "$SRC/vlasovsolver/$f"
done
for f in velocity_mesh_cpu.h velocity_block_container.h; do
  ln -s "$REF/spatial_cells/$f" "$SRC/spatial_cells/$f"
done
for f in common.h definitions.h open_bucket_hashtable.h velocity_mesh_parameters.h velocity_mesh_parameters.cpp memoryallocation.h; do
  ln -s "$REF/$f" "$SRC/$f"
done
for f in arch_device_api.h arch_device_host.h; do
  ln -s "$REF/arch/$f" "$SRC/arch/$f"
done
# translation: the uniform-grid part of cpu_trans_map_amr.cpp (propagatePencil,
# copy_trans_block_data_amr, trans_map_1d_amr; lines 1-443), without the MPI
# remote-contribution functions that follow
sed -n '1,443p' "$REF/vlasovsolver/cpu_trans_map_amr.cpp" > "$SRC/vlasovsolver/cpu_trans_map_amr_part.cpp"
# block adjustment: the content test and block add/remove of SpatialCell
# (adjust_velocity_blocks, compute_block_has_content,
# update_velocity_block_content_lists, updateSparseMinValue; spatial_cell_cpu.cpp
# lines 179-273, 290-316, 675-688, 699-727) and the grid-level drivers of
# block_adjust_cpu.cpp (lines 28-119), compiled as members of the stand-in cell
{
  printf '#include <iostream>\n#include <unordered_set>\n#include <vector>\n'
  printf '#include "spatial_cells/spatial_cell_wrapper.hpp"\n#include "object_wrapper.h"\n'
  printf 'using namespace std;\nnamespace spatial_cell {\n'
  sed -n '179,273p;290,316p;675,688p;699,727p' "$REF/spatial_cells/spatial_cell_cpu.cpp"
  printf '}  // namespace spatial_cell\n'
  sed -n '28,119p' "$REF/spatial_cells/block_adjust_cpu.cpp"
} > "$SRC/spatial_cells/block_adjust_part.cpp"
# the r-space time-step reduction reduce_vlasov_dt (arch_dt.cpp, the whole
# file); its source names std types unqualified
{
  printf '#include <algorithm>\n#include <limits>\n#include <vector>\nusing namespace std;\n'
  cat "$REF/vlasovsolver/arch_dt.cpp"
} > "$SRC/vlasovsolver/arch_dt_part.cpp"
# the initial condition's phase-space densities, MaxwellianPhaseSpaceDensity
# and TriMaxwellianPhaseSpaceDensity (projects/project.h lines 34-73, inline
# functions), without the Project class and the field-solver headers around them
mkdir -p "$SRC/projects"
{
  printf '#include <cmath>\n#include "common.h"\nnamespace projects {\n'
  sed -n '34,73p' "$REF/projects/project.h"
  printf '}  // namespace projects\n'
} > "$SRC/projects/project_density_part.h"
cp "$HERE/ref_shim/grid.h" "$SRC/grid.h"
cp "$HERE/ref_shim/object_wrapper.h" "$SRC/object_wrapper.h"
cp "$HERE/ref_shim/spatial_cells/spatial_cell_wrapper.hpp" "$SRC/spatial_cells/spatial_cell_wrapper.hpp"
cp "$HERE/ref_shim/sysinc/"*.hpp "$SRC/sysinc/"
cp "$HERE/ref_harness.cpp" "$SRC/ref_harness.cpp"

CXX="${REF_CXX:-/usr/bin/g++}"
COMMON=(-std=c++20 -O3 -march=x86-64-v3 -ffp-contract=off -fopenmp -fPIC -shared
        -DDP -DTRANS_SEMILAG_PPM -DVEC_FALLBACK_GENERIC
        -I"$SRC" -I"$SRC/sysinc" -w)
SRCS=("$SRC/ref_harness.cpp" "$SRC/vlasovsolver/cpu_acc_map.cpp"
      "$SRC/vlasovsolver/cpu_acc_sort_blocks.cpp" "$SRC/vlasovsolver/cpu_acc_load_blocks.cpp"
      "$SRC/velocity_mesh_parameters.cpp" "$SRC/vlasovsolver/cpu_trans_map_amr_part.cpp"
      "$SRC/spatial_cells/block_adjust_part.cpp" "$SRC/vlasovsolver/arch_dt_part.cpp")
# the oracle's own FP64 geometry restatement (the reference's needs Eigen)
CC="${REF_CC:-/usr/bin/gcc}"
"$CC" -O2 -std=c11 -fPIC -ffp-contract=off -c "$HERE/vlasov_oracle.c" -o "$OUT/orc_geometry_sp.o"
"$CC" -O2 -std=c11 -fPIC -ffp-contract=off -DORC_DOUBLE -c "$HERE/vlasov_oracle.c" -o "$OUT/orc_geometry_dp.o"
rm -f "$OUT"/libvlasov_ref_*.so
pids=()
"$CXX" "${COMMON[@]}" -DACC_SEMILAG_PPM -DSPF -DVECL=16 "${SRCS[@]}" "$OUT/orc_geometry_sp.o" \
  -o "$OUT/libvlasov_ref_sp.so" & pids+=($!)
"$CXX" "${COMMON[@]}" -DACC_SEMILAG_PPM -DDPF -DVECL=8 "${SRCS[@]}" "$OUT/orc_geometry_dp.o" \
  -o "$OUT/libvlasov_ref_dp.so" & pids+=($!)
# the other acceleration reconstructions of the reference (PQM is its
# Makefile default, PLM the lowest order), FP32 VDF
"$CXX" "${COMMON[@]}" -DACC_SEMILAG_PQM -DSPF -DVECL=16 "${SRCS[@]}" "$OUT/orc_geometry_sp.o" \
  -o "$OUT/libvlasov_ref_sp_pqm.so" & pids+=($!)
"$CXX" "${COMMON[@]}" -DACC_SEMILAG_PLM -DSPF -DVECL=16 "${SRCS[@]}" "$OUT/orc_geometry_sp.o" \
  -o "$OUT/libvlasov_ref_sp_plm.so" & pids+=($!)
# the C++ drop-in layer (include/vlgpu.hpp) instantiated with the stand-in
# cell beside the reference's own map_1d, linked against libvlgpu.so
LIBVLGPU="$HERE/../vlasiator_b200/libvlgpu.so"
cp "$HERE/dropin_harness.cpp" "$SRC/dropin_harness.cpp"
if [ -f "$LIBVLGPU" ]; then
  "$CXX" "${COMMON[@]}" -DACC_SEMILAG_PPM -DSPF -DVECL=16 -I"$HERE/../include" "${SRCS[@]}" "$SRC/dropin_harness.cpp" \
    "$OUT/orc_geometry_sp.o" -L"$HERE/../vlasiator_b200" -lvlgpu -Wl,-rpath,'$ORIGIN/../../vlasiator_b200' \
    -o "$OUT/libvlasov_ref_sp_dropin.so" & pids+=($!)
fi
fail=0
for p in "${pids[@]}"; do wait "$p" || fail=1; done
if [ "$fail" -ne 0 ]; then echo "build_ref: a compilation failed" >&2; exit 4; fi
for f in sp dp sp_pqm sp_plm; do test -f "$OUT/libvlasov_ref_$f.so"; done
echo "build_ref: built $OUT/libvlasov_ref_{sp,dp,sp_pqm,sp_plm}.so"
