// C entry points around reference routines of the electronic step that the
// oracle restates, compiled by build_ref.sh from their own sources:
//   CPNONLOCAL::CP_eke_calc       abinito_physics/cp_nonlocal/cp_eke.C:30-140
//   CPLOCAL::CP_hart_eext_calc    abinito_physics/cp_local/cp_hart_ext.C:56-405
//   FFTcache::expandGSpace / packGSpace   fft_slab_ctrl/fftCache.C:460-553 (the
//                                 two member functions, cut from the file by
//                                 build_ref.sh: the rest of it needs Charm++)
// with the PINY singletons of ref_ees.cpp / ref_ion.cpp filled for one
// Gamma-point, spin-unpolarised, fully periodic system.  Test infrastructure
// only: oracle/fftpath.py (eke, expand, pack) and oracle/density.py
// (hart_eext) are pinned to these.
#include <vector>
#include "standard_include.h"
#include "ckcomplex.h"
#include "../../include/Atoms.h"
#include "../../include/eesDataClass.h"
#include "allclass_cp.h"
#include "allclass_gen.h"
#include "allclass_mdatoms.h"
#include "CP_OPERATIONS/class_cpnonlocal.h"
#include "CP_OPERATIONS/class_cplocal.h"
#include "fftcache_shim.h"

namespace {
std::vector<double> l_occ, l_wk, l_vps[4], l_gz;
std::vector<int> l_typ1, l_locopt;
double* ob(std::vector<double>& v) { return v.data() - 1; }
}  // namespace

extern "C" {

// CP_eke_calc on one state's coefficients in the chare order the routine
// assumes (the nkx0 Gx=0 points first): forces[ncoef] complex (in/out), psi,
// g2 [ncoef]; ecut_ry = cpcoeffs_info->ecut_psi; occ[nstate]; *eke = E_kin.
void ref_eke(int ncoef, int istate, double* forces, const double* psi, int* kx, int* ky,
             int* kz, double* g2, int nkx0, double ecut_ry, int nstate, const double* occ,
             double* eke) {
  CP* cp = CP::get();
  l_occ.assign(occ, occ + nstate);
  l_wk.assign(1, 1.0);
  cp->cpcoeffs_info.ecut_psi = ecut_ry;
  cp->cpcoeffs_info.occ_up = ob(l_occ);
  cp->cpcoeffs_info.wght_kpt = ob(l_wk);
  double* g2k[1] = {g2};
  CPNONLOCAL::CP_eke_calc(ncoef, istate, reinterpret_cast<complex*>(forces),
                          reinterpret_cast<complex*>(const_cast<double*>(psi)), kx, ky, kz, g2k,
                          eke, 1, nkx0, 0, 1);
}

// CP_hart_eext_calc on the packed density sphere (point i at offset i):
// rho[npts] complex, kx/ky/kz of the points, ecut_ha = cpcoeffs_info->ecut
// (the sphere is g^2 <= 8 ecut_ha), cell hmat/hmati (row-major 3x3), alp_ewd,
// atoms: typ (0-based) and xyz [natm][3], q [natm]; local pseudopotential
// splines vloc [ntyp][4][nspl] (vps0..vps3 on gmin + k dg) and gzvps [ntyp].
// Out: vks[npts] complex (zero outside the sphere), e = {ehart, eext, ewd},
// f [natm][3] += the local and reciprocal Ewald atom forces.
void ref_hart_eext(int npts, const int* kx, const int* ky, const int* kz, const double* rho,
                   double ecut_ha, const double* hmat, const double* hmati, double vol,
                   double alp_ewd, int natm, int ntyp, const int* typ, const double* xyz,
                   const double* q, int nspl, double gmin, double dg, const double* vloc,
                   const double* gzvps, double* vks, double* e, double* f) {
  CP* cp = CP::get();
  GENERAL_DATA* gd = GENERAL_DATA::get();
  MDATOMS* md = MDATOMS::get();
  for (int k = 0; k < 9; ++k) {
    gd->gencell.hmat[k + 1] = hmat[k];
    gd->gencell.hmati[k + 1] = hmati[k];
  }
  gd->gencell.vol = vol;
  gd->genewald.alp_ewd = alp_ewd;
  cp->cpcoeffs_info.ecut = ecut_ha;
  CPPSEUDO* ps = &cp->cppseudo;
  ps->nsplin_g = nspl;
  ps->gmin_spl = gmin;
  ps->dg_spl = dg;
  ps->n_ang_max = 0;  // the local channel only: index_atm = (type-1) nsplin_g
  ps->n_rad_max = 1;
  l_locopt.assign(ntyp, 0);
  ps->loc_opt = l_locopt.data() - 1;
  for (int k = 0; k < 4; ++k) {
    l_vps[k].assign((size_t)ntyp * nspl, 0.0);
    for (int t = 0; t < ntyp; ++t)
      for (int i = 0; i < nspl; ++i)
        l_vps[k][(size_t)t * nspl + i] = vloc[((size_t)t * 4 + k) * nspl + i];
  }
  ps->vps0 = ob(l_vps[0]);
  ps->vps1 = ob(l_vps[1]);
  ps->vps2 = ob(l_vps[2]);
  ps->vps3 = ob(l_vps[3]);
  l_gz.assign(gzvps, gzvps + ntyp);
  ps->gzvps = ob(l_gz);
  md->mdclatoms_info.natm_tot = natm;
  md->mdatom_maps.natm_typ = ntyp;
  l_typ1.resize(natm);
  for (int i = 0; i < natm; ++i) l_typ1[i] = typ[i] + 1;
  md->mdatom_maps.iatm_atm_typ = l_typ1.data() - 1;
  std::vector<double> x(natm), y(natm), z(natm), qq(q, q + natm), fx(natm, 0.0), fy(natm, 0.0),
      fz(natm, 0.0);
  for (int i = 0; i < natm; ++i) {
    x[i] = xyz[3 * i];
    y[i] = xyz[3 * i + 1];
    z[i] = xyz[3 * i + 2];
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
  std::vector<gridPoint> pts(npts);
  for (int i = 0; i < npts; ++i) {
    pts[i].d1 = kz[i];
    pts[i].d2 = ky[i];
    pts[i].d3 = kx[i];
    pts[i].offset = i;
  }
  std::vector<int> index_atm(ntyp + 1, 0);
  std::vector<double> vtemp(natm + 1, 0.0);
  std::vector<complex> ei(natm + 1), ti(natm + 1);
  PSSCRATCH scr;
  scr.index_atm = index_atm.data();
  scr.vtemp = vtemp.data();
  scr.ei_inc = ei.data();
  scr.ti_inc = ti.data();
  for (int i = 0; i < 2 * npts; ++i) vks[i] = 0.0;
  CPLOCAL::CP_hart_eext_calc(npts, pts, reinterpret_cast<complex*>(const_cast<double*>(rho)),
                             natm, 3, &fa, reinterpret_cast<complex*>(vks), &e[0], &e[1], &e[2],
                             0, &scr, 1);
  for (int i = 0; i < natm; ++i) {
    f[3 * i] += fx[i];
    f[3 * i + 1] += fy[i];
    f[3 * i + 2] += fz[i];
  }
}

// FFTcache::expandGSpace / packGSpace on one state: runs [numRuns][7] ints
// (x, y, z, position, length, inc, nz), data [numRuns/2][nfftz] complex.
void ref_expand(double* data, const double* packed, const int* runs, int numRuns, int numPoints,
                int nfftz) {
  std::vector<RunDescriptor> r(numRuns);
  for (int i = 0; i < numRuns; ++i)
    r[i] = RunDescriptor(runs[7 * i], runs[7 * i + 1], runs[7 * i + 2], runs[7 * i + 3],
                         runs[7 * i + 4], runs[7 * i + 5], runs[7 * i + 6]);
  FFTcache fc;
  fc.expandGSpace(reinterpret_cast<complex*>(data),
                  reinterpret_cast<complex*>(const_cast<double*>(packed)), r.data(), numRuns,
                  numRuns / 2 * nfftz, numPoints, nfftz);
}

void ref_pack(const double* data, double* packed, const int* runs, int numRuns, int numPoints,
              int nfftz) {
  std::vector<RunDescriptor> r(numRuns);
  for (int i = 0; i < numRuns; ++i)
    r[i] = RunDescriptor(runs[7 * i], runs[7 * i + 1], runs[7 * i + 2], runs[7 * i + 3],
                         runs[7 * i + 4], runs[7 * i + 5], runs[7 * i + 6]);
  FFTcache fc;
  fc.packGSpace(reinterpret_cast<complex*>(const_cast<double*>(data)),
                reinterpret_cast<complex*>(packed), r.data(), numRuns, numRuns / 2 * nfftz,
                numPoints, nfftz);
}

}  // extern "C"
