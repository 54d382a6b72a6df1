// C entry points around the reference's CP thermostat and integrator,
// CPINTEGRATE::initCPNHC / cp_isoNHC_update (cp_integrate/cp_isokin.C:45-311)
// and CPINTEGRATE::CP_integrate_dyn / cp_evolve_vel / get_fictKE
// (cp_integrate/cp_dynamics.C:22-256), compiled by build_ref.sh from their
// own sources; fills the PINY singletons they read.  Test infrastructure
// only: oracle/isokin.py is pinned to this.
#include <vector>
#include "standard_include.h"
#include "ckcomplex.h"
#include "allclass_gen.h"
#include "allclass_cp.h"
#include "CP_OPERATIONS/class_cpintegrate.h"

namespace {
void set_params(double dt, int num, int nck, int nres, int nyosh, double te_ext, double tau_fs) {
  GENERAL_DATA* gd = GENERAL_DATA::get();
  CP* cp = CP::get();
  gd->gentimeinfo.dt = dt;
  gd->gentimeinfo.bomd_scale = 1.0;
  cp->cptherm_info.len_c_nhc = 2;
  cp->cptherm_info.num_c_nhc_iso = num;
  cp->cptherm_info.nck_c_nhc = nck;
  cp->cptherm_info.nres_c_nhc = nres;
  cp->cptherm_info.nyosh_c_nhc = nyosh;
  cp->cpopts.te_ext = te_ext;
  cp->cpopts.cp_tau_nhc = tau_fs;
}

// [nck][num][2] views of a flat array
struct Chain {
  std::vector<double**> lvl1;
  std::vector<double*> lvl2;
  double*** p;
  Chain(double* flat, int nck, int num) : lvl1(nck), lvl2((size_t)nck * num) {
    for (int k = 0; k < nck; ++k) {
      for (int i = 0; i < num; ++i) lvl2[(size_t)k * num + i] = flat + ((size_t)k * num + i) * 2;
      lvl1[k] = &lvl2[(size_t)k * num];
    }
    p = lvl1.data();
  }
};
}  // namespace

extern "C" {

// out9 = {kT, tau, degfree, degfreeNHC, mNHC[0], mNHC[1]}, v0/a2/a4[num],
// degFreeSplt[nck], istr/iend[nck]
void ref_init_cpnhc(int ncoef_use, int nzero, int num, int nck, double te_ext, double tau_fs,
                    double* out6, double* v0, double* a2, double* a4, double* dfs, int* istr,
                    int* iend) {
  set_params(1.0, num, nck, 4, 9, te_ext, tau_fs);
  double m[2];
  CPINTEGRATE::initCPNHC(ncoef_use, nzero, 2, num, nck, &out6[0], &out6[1], &out6[2], &out6[3],
                         m, v0, a2, a4, dfs, istr, iend);
  out6[4] = m[0];
  out6[5] = m[1];
}

// One CP_integrate_dyn on one chare's packed coefficients (redundant half
// first, then G = 0, the unique Gx = 0 points, the rest); psi, v, f are
// interleaved complex [ncoef]; x, xp, vn are [nck][num][2] and updated;
// out3 = {fictEke, ekeNhc, potNHC}.
void ref_cp_integrate_dyn(int ncoef, int iteration, double* f, double* v, double* psi,
                          double* cmass, int nred, int nuni, int nzero, int num, int nck,
                          double* x, double* xp, double* vn, double dt, int nres, int nyosh,
                          double te_ext, double tau_fs, double* out3) {
  set_params(dt, num, nck, nres, nyosh, te_ext, tau_fs);
  const int ncoef_use = ncoef - nred;
  double hdr[6], mNHC[2];
  std::vector<double> v0(num), a2(num), a4(num), dfs(nck);
  std::vector<int> istr(nck), iend(nck);
  CPINTEGRATE::initCPNHC(ncoef_use, nzero, 2, num, nck, &hdr[0], &hdr[1], &hdr[2], &hdr[3],
                         mNHC, v0.data(), a2.data(), a4.data(), dfs.data(), istr.data(),
                         iend.data());
  std::vector<double> fn((size_t)nck * num * 2, 0.0);
  Chain cx(x, nck, num), cxp(xp, nck, num), cvn(vn, nck, num), cfn(fn.data(), nck, num);
  std::vector<int> kx(ncoef, 0), ky(ncoef, 0), kz(ncoef, 0);
  CPINTEGRATE::CP_integrate_dyn(ncoef, 0, iteration, reinterpret_cast<complex*>(f),
                                reinterpret_cast<complex*>(v), reinterpret_cast<complex*>(psi),
                                cmass, kx.data(), ky.data(), kz.data(), 2, num, nck, cfn.p,
                                cvn.p, cx.p, cxp.p, mNHC, v0.data(), a2.data(), a4.data(),
                                hdr[0], &out3[0], nred, nuni, nzero, &out3[1], &out3[2], hdr[2],
                                hdr[3], dfs.data(), istr.data(), iend.data(), 1, false, 1.0,
                                1.0);
}

}  // extern "C"
