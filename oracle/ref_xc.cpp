// C entry points around the reference's exchange-correlation routines,
// compiled by build_ref.sh from their own sources (cp_becke.C,
// cp_grad_rho_ctrl.C, cp_pz_lda.C) with the PINY singletons of ref_ees.cpp
// filled for one Gamma-point, spin-unpolarised system.  Test infrastructure
// only: oracle/xc.py is pinned to these.
//
// The reference's grid loops (cp_pz_lda.C:108-160, cp_grad_rho_ctrl.C:81-176)
// walk rows padded to 2 (nf1/2 + 1) doubles; the entries below take unpadded
// [nf3][nf2][nf1] arrays and pad them on the way in and out.
#include <cstring>
#include <vector>
#include "standard_include.h"
#include "ckcomplex.h"
#include "allclass_cp.h"
#include "allclass_gen.h"
#include "CP_OPERATIONS/class_cpxcfnctls.h"

namespace {
int row_len(int nf1) { return 2 * (nf1 / 2 + 1); }

std::vector<double> pad(const double* a, int nf1, int nf2, int nf3) {
  const int xl = row_len(nf1);
  std::vector<double> p((size_t)xl * nf2 * nf3, 0.0);
  for (size_t r = 0; r < (size_t)nf2 * nf3; ++r)
    std::memcpy(&p[r * xl], a + r * nf1, sizeof(double) * nf1);
  return p;
}

void unpad(const std::vector<double>& p, double* a, int nf1, int nf2, int nf3) {
  const int xl = row_len(nf1);
  for (size_t r = 0; r < (size_t)nf2 * nf3; ++r)
    std::memcpy(a + r * nf1, &p[r * xl], sizeof(double) * nf1);
}
}  // namespace

extern "C" {

// becke_gcx_lda (cp_becke.C:20-77): out = {f, df/drho, df/d|grad rho|}
void ref_becke(double rho, double g_rho2, double beta, double* out) {
  CPXCFNCTS::becke_gcx_lda(rho, g_rho2, &out[0], &out[1], &out[2], beta);
}

// lyp_gcc (cp_becke.C:91-173)
void ref_lyp(double rho, double g_rho2, double* out) {
  CPXCFNCTS::lyp_gcc(rho, g_rho2, &out[0], &out[1], &out[2]);
}

// CP_getGGAFunctional (cp_grad_rho_ctrl.C:32-193) on unpadded arrays: vks +=
// df/drho, gx/gy/gz <- unit(grad rho) df/d|grad rho|, *exc = E_GGA.  The
// reference keeps its healing length in a function-level static set on the
// first call, so every call in one process must pass the same gga_cut.
void ref_gga_functional(int nf1, int nf2, int nf3, double vol, double gga_cut, int becke,
                        int lyp, const double* rho, double* gx, double* gy, double* gz,
                        double* vks, double* exc) {
  CP* cp = CP::get();
  GENERAL_DATA* gd = GENERAL_DATA::get();
  cp->cpopts.cp_becke = becke;
  cp->cpopts.cp_lyp = lyp;
  cp->cppseudo.gga_cut = gga_cut;
  gd->gencell.vol = vol;
  std::vector<double> d = pad(rho, nf1, nf2, nf3), x = pad(gx, nf1, nf2, nf3),
                      y = pad(gy, nf1, nf2, nf3), z = pad(gz, nf1, nf2, nf3),
                      v = pad(vks, nf1, nf2, nf3);
  CPXCFNCTS::CP_getGGAFunctional(nf1 * nf2 * nf3, nf1, nf2, nf3, d.data(), x.data(), y.data(),
                                 z.data(), v.data(), 0, exc, 1);
  unpad(x, gx, nf1, nf2, nf3);
  unpad(y, gy, nf1, nf2, nf3);
  unpad(z, gz, nf1, nf2, nf3);
  unpad(v, vks, nf1, nf2, nf3);
}

// CP_exc_calc (cp_pz_lda.C:23-170): vxc, exc, muxc; lyp = 1 switches the PZ
// correlation off (BLYP: Slater exchange here, LYP in the GGA routine)
void ref_exc_calc(int nf1, int nf2, int nf3, double vol, int lyp, const double* rho,
                  double* vxc, double* exc, double* muxc) {
  CP* cp = CP::get();
  GENERAL_DATA* gd = GENERAL_DATA::get();
  cp->cpopts.cp_lyp = lyp;
  gd->gencell.vol = vol;
  std::vector<double> d = pad(rho, nf1, nf2, nf3), v((size_t)row_len(nf1) * nf2 * nf3, 0.0);
  CPXCFNCTS::CP_exc_calc(nf1 * nf2 * nf3, nf1, nf2, nf3, d.data(), v.data(), exc, muxc, 1);
  unpad(v, vxc, nf1, nf2, nf3);
}

}  // extern "C"
