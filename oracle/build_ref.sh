#!/bin/sh
# Compile the reference leaves the oracle is pinned to, from their own
# sources, into oracle/_ref/libref.so (git-ignored; it travels with the tree).
#   src_charm_driver/utility/para_grp_parse.C   flip_data_set, get_chareG_line_prms
#   src_mathlib/lst_sort_clean.C                sort_commence
#   src_piny_physics_v1.0/abinito_physics/cp_orthog/cp_lowdin.C   get_iter_Tmat
#   src_piny_physics_v1.0/abinito_physics/cp_nonlocal/cp_ees_nonlocal.C  EES non-local
#   src_piny_physics_v1.0/interface/cp_ewald/set_cp_ewald.C  get_bspline_wght1d,
#                                                           init_nonlocal_ees
#   src_piny_physics_v1.0/abinito_physics/cp_xc_fnctl/cp_becke.C, cp_grad_rho_ctrl.C,
#                         cp_pz_lda.C   becke_gcx_lda, lyp_gcc, CP_getGGAFunctional,
#                                       CP_exc_calc
#   src_piny_physics_v1.0/abinito_physics/cp_nonlocal/cp_struct_fact.C, cp_nlmat.C,
#                         cp_nl_energy_forc.C   the structure-factor nonlocal (l = 0)
#   src_piny_physics_v1.0/abinito_physics/cp_ions/cp_rspace_ion.C   CP_getionforce
#   src_piny_physics_v1.0/abinito_physics/cp_integrate/cp_isokin.C, cp_dynamics.C
#                         initCPNHC, cp_isoNHC_update, CP_integrate_dyn
#   src_piny_physics_v1.0/classical_physics/integrate/integration_drivers.C
#                         integrate_nvt_2nd_half / _1st_half (massive atom NHC)
#   src_piny_physics_v1.0/abinito_physics/cp_nonlocal/cp_eke.C   CP_eke_calc
#   src_piny_physics_v1.0/abinito_physics/cp_local/cp_hart_ext.C CP_hart_eext_calc
#   src_charm_driver/fft_slab_ctrl/fftCache.C   FFTcache::expandGSpace, packGSpace:
#       the rest of that file needs Charm++, so the two member functions are
#       cut from it (sed, by their first and last lines) into _ref/fftcache_pack.C
#       behind the class stand-in ref_shim/fftcache_shim.h
# The shims in oracle/ref_shim stand in for the Charm++/PINY headers, and
# oracle/ref_mathlib.c for the Fortran GENMATMUL.  Test infrastructure only.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${OPENATOM_REF:-/root/reference}
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -d "$REF/src_charm_driver" ]; then
  echo "reference tree not found at $REF; keeping any prebuilt $OUT/libref.so" >&2
  exit 0
fi
gcc -O2 -fPIC -c "$HERE/ref_mathlib.c" -o "$OUT/ref_mathlib.o"
# the EES sources read the PINY singletons (CP::get() under CHARM_ON) and the
# PINY constants/macros (SIMP_NINT as every platform standard_include.h sets)
PINY="$REF/src_piny_physics_v1.0"
EESFLAGS="-O2 -fPIC -w -DCHARM_ON -DSIMP_NINT -include $HERE/ref_shim/ees_shim.h \
  -include $PINY/include/class_defs/piny_constants.h -I $HERE/ref_shim -I $HERE/ref_shim/sub \
  -I $REF -I $REF/src_charm_driver/utility -I $PINY/include/class_defs -I $REF/include"
for f in "$PINY/abinito_physics/cp_nonlocal/cp_ees_nonlocal.C" \
         "$PINY/interface/cp_ewald/set_cp_ewald.C" "$HERE/ref_ees.cpp" \
         "$PINY/abinito_physics/cp_xc_fnctl/cp_becke.C" \
         "$PINY/abinito_physics/cp_xc_fnctl/cp_grad_rho_ctrl.C" \
         "$PINY/abinito_physics/cp_xc_fnctl/cp_pz_lda.C" "$HERE/ref_xc.cpp" \
         "$PINY/abinito_physics/cp_nonlocal/cp_struct_fact.C" \
         "$PINY/abinito_physics/cp_nonlocal/cp_nlmat.C" \
         "$PINY/abinito_physics/cp_nonlocal/cp_nl_energy_forc.C" "$HERE/ref_sf.cpp" \
         "$PINY/abinito_physics/cp_ions/cp_rspace_ion.C" "$HERE/ref_ion.cpp" \
         "$PINY/abinito_physics/cp_integrate/cp_isokin.C" \
         "$PINY/abinito_physics/cp_integrate/cp_dynamics.C" "$HERE/ref_isokin.cpp" \
         "$PINY/classical_physics/integrate/integration_drivers.C" "$HERE/ref_atomnhc.cpp" \
         "$PINY/abinito_physics/cp_nonlocal/cp_eke.C" \
         "$PINY/abinito_physics/cp_local/cp_hart_ext.C" "$HERE/ref_local.cpp"; do
  g++ $EESFLAGS -c "$f" -o "$OUT/$(basename "$f" | sed 's/\.[Cc]p*$//').o"
done
{
  echo '#include "fftcache_shim.h"'
  sed -n '/^void FFTcache::expandGSpace/,/^}\/\/end routine/p' \
    "$REF/src_charm_driver/fft_slab_ctrl/fftCache.C"
  sed -n '/^void FFTcache::packGSpace/,/^}\/\/end routine/p' \
    "$REF/src_charm_driver/fft_slab_ctrl/fftCache.C"
} > "$OUT/fftcache_pack.C"
g++ -O2 -fPIC -w -include "$HERE/ref_shim/ees_shim.h" -I "$HERE/ref_shim" -I "$REF/include" \
  -c "$OUT/fftcache_pack.C" \
  -o "$OUT/fftcache_pack.o"
g++ -O2 -fPIC -shared -w -o "$OUT/libref.so" \
  -I "$HERE/ref_shim" -I "$HERE/ref_shim/sub" -I "$REF" \
  -I "$REF/src_charm_driver/utility" -I "$REF/src_piny_physics_v1.0/include/class_defs" \
  "$REF/src_charm_driver/utility/para_grp_parse.C" \
  "$REF/src_mathlib/lst_sort_clean.C" \
  "$REF/src_piny_physics_v1.0/abinito_physics/cp_orthog/cp_lowdin.C" \
  "$HERE/ref_driver.cpp" "$OUT/ref_mathlib.o" \
  "$OUT/cp_ees_nonlocal.o" "$OUT/set_cp_ewald.o" "$OUT/ref_ees.o" \
  "$OUT/cp_becke.o" "$OUT/cp_grad_rho_ctrl.o" "$OUT/cp_pz_lda.o" "$OUT/ref_xc.o" \
  "$OUT/cp_struct_fact.o" "$OUT/cp_nlmat.o" "$OUT/cp_nl_energy_forc.o" "$OUT/ref_sf.o" \
  "$OUT/cp_rspace_ion.o" "$OUT/ref_ion.o" \
  "$OUT/cp_isokin.o" "$OUT/cp_dynamics.o" "$OUT/ref_isokin.o" \
  "$OUT/integration_drivers.o" "$OUT/ref_atomnhc.o" \
  "$OUT/cp_eke.o" "$OUT/cp_hart_ext.o" "$OUT/ref_local.o" "$OUT/fftcache_pack.o"
echo "$OUT/libref.so"
