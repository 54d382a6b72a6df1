// C entry point around the reference's real-space ion-ion routine
// CPRSPACEION::CP_getionforce (cp_ions/cp_rspace_ion.C:25-250), compiled by
// build_ref.sh from its own source; fills the PINY singletons it reads for a
// fully periodic (iperd = 3) cell without the Grimme term.  Test
// infrastructure only: oracle/ions.py is pinned to this.
#include <vector>
#include "standard_include.h"
#include "ckcomplex.h"
#include "../../include/Atoms.h"
#include "allclass_gen.h"
#include "allclass_mdatoms.h"
#include "allclass_cp.h"
#include "CP_OPERATIONS/class_cprspaceion.h"

MDATOMS readonly_mdatoms;

extern "C" {

// f[natm][3] += real-space Ewald forces; out = {pot_ewd_rs, vself, vbgr}
void ref_ionforce(int natm, const double* xyz, const double* q, const double* hmat,
                  const double* hmati, double vol, double alp_ewd, double ecut, double* f,
                  double* out) {
  GENERAL_DATA* gd = GENERAL_DATA::get();
  MDATOMS* md = MDATOMS::get();
  for (int k = 0; k < 9; ++k) {
    gd->gencell.hmat[k + 1] = hmat[k];
    gd->gencell.hmati[k + 1] = hmati[k];
  }
  gd->gencell.vol = vol;
  gd->gencell.iperd = 3;
  gd->genewald.alp_ewd = alp_ewd;
  gd->genewald.ecut = ecut;
  md->mdclatoms_info.natm_tot = natm;
  md->mdclatoms_info.cp_grimme = 0;
  std::vector<double> x(natm), y(natm), z(natm), qq(q, q + natm), fx(natm), fy(natm), fz(natm);
  for (int i = 0; i < natm; ++i) {
    x[i] = xyz[3 * i];
    y[i] = xyz[3 * i + 1];
    z[i] = xyz[3 * i + 2];
    fx[i] = f[3 * i];
    fy[i] = f[3 * i + 1];
    fz[i] = f[3 * i + 2];
  }
  FastAtoms fa;
  fa.natm = natm;
  fa.x = x.data();
  fa.y = y.data();
  fa.z = z.data();
  fa.q = qq.data();
  fa.fx = fx.data();
  fa.fy = fy.data();
  fa.fz = fz.data();
  PSSCRATCH ps;
  double pot = 0.0, vself = 0.0, vbgr = 0.0, corr = 0.0, potg = 0.0;
  CPRSPACEION::CP_getionforce(natm, &fa, 0, 1, &pot, &vself, &vbgr, &corr, &ps, &potg);
  for (int i = 0; i < natm; ++i) {
    f[3 * i] = fx[i];
    f[3 * i + 1] = fy[i];
    f[3 * i + 2] = fz[i];
  }
  out[0] = pot;
  out[1] = vself;
  out[2] = vbgr;
}

}  // extern "C"
