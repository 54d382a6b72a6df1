// C entry points around the reference's structure-factor (non-EES) nonlocal
// routines, compiled by build_ref.sh from their own sources (cp_struct_fact.C,
// cp_nlmat.C, cp_nl_energy_forc.C) on top of the PINY singletons that
// ref_ees_setup (ref_ees.cpp) fills.  One structure-factor group
// (numSfGrps = 1), double pack.  Test infrastructure only: oracle/sf.py is
// pinned to these.
#include <vector>
#include "standard_include.h"
#include "ckcomplex.h"
#include "../../include/Atoms.h"
#include "allclass_cp.h"
#include "allclass_gen.h"
#include "CP_OPERATIONS/class_cpnonlocal.h"

namespace {
std::vector<double> s_vn0, s_x, s_y, s_z, s_ax, s_ay, s_az, s_fx, s_fy, s_fz;
std::vector<complex> s_ei, s_ti;
std::vector<int> s_typ_lang;
FastAtoms s_atoms;
PSSCRATCH s_ps;
}  // namespace

extern "C" {

// After ref_ees_setup: every atom non-local with its type's l = 0 channel;
// vnorm0[natm] per non-local atom in the setup's type order (map_nl), xyz
// [natm][3] Cartesian positions.
void ref_sf_setup(int ntyp, const double* vnorm0, const double* xyz) {
  PSNONLOCAL* nl = &readonly_cp.cppseudo.nonlocal;
  const int natm = nl->natm;
  s_vn0.assign(vnorm0, vnorm0 + natm);
  nl->vnorm_0 = s_vn0.data() - 1;
  nl->natm_typ = ntyp;
  s_typ_lang.assign(2, 0);
  s_typ_lang[1] = ntyp;  // l = 0 types (natm_typ_lang[lang + 1])
  nl->natm_typ_lang = s_typ_lang.data();
  s_x.assign(natm + 1, 0.0);
  s_y.assign(natm + 1, 0.0);
  s_z.assign(natm + 1, 0.0);
  s_ei.assign(natm + 1, complex(0.0, 0.0));
  s_ti.assign(natm + 1, complex(0.0, 0.0));
  s_ps.x = s_x.data();
  s_ps.y = s_y.data();
  s_ps.z = s_z.data();
  s_ps.ei_inc = s_ei.data();
  s_ps.ti_inc = s_ti.data();
  s_ax.resize(natm);
  s_ay.resize(natm);
  s_az.resize(natm);
  for (int i = 0; i < natm; ++i) {
    s_ax[i] = xyz[3 * i];
    s_ay[i] = xyz[3 * i + 1];
    s_az[i] = xyz[3 * i + 2];
  }
  s_fx.assign(natm, 0.0);
  s_fy.assign(natm, 0.0);
  s_fz.assign(natm, 0.0);
  s_atoms.natm = natm;
  s_atoms.x = s_ax.data();
  s_atoms.y = s_ay.data();
  s_atoms.z = s_az.data();
  s_atoms.fx = s_fx.data();
  s_atoms.fy = s_fy.data();
  s_atoms.fz = s_fz.data();
}

// CP_calc_Struct_Fact (cp_struct_fact.C:33-221) over n packed points in the
// reference's line order; S* [natm][n] complex
void ref_sf_struct_fact(int n, int* kx, int* ky, int* kz, double* s, double* sx, double* sy,
                        double* sz) {
  CPNONLOCAL::CP_calc_Struct_Fact(n, kx, ky, kz, reinterpret_cast<complex*>(s),
                                  reinterpret_cast<complex*>(sx), reinterpret_cast<complex*>(sy),
                                  reinterpret_cast<complex*>(sz), &s_atoms, 1, 1, 0, &s_ps);
}

// CP_enl_matrix_calc (cp_nlmat.C:20-92): z* [natm] complex (real parts written)
void ref_sf_zmat(int n, double* psi, int* kx, int* ky, int* kz, double* s, double* sx,
                 double* sy, double* sz, double* z, double* zx, double* zy, double* zz,
                 int state) {
  CPNONLOCAL::CP_enl_matrix_calc(
      n, reinterpret_cast<complex*>(psi), kx, ky, kz, reinterpret_cast<complex*>(s),
      reinterpret_cast<complex*>(sx), reinterpret_cast<complex*>(sy),
      reinterpret_cast<complex*>(sz), reinterpret_cast<complex*>(z),
      reinterpret_cast<complex*>(zx), reinterpret_cast<complex*>(zy),
      reinterpret_cast<complex*>(zz), state, 1, 1, 0);
}

// CP_enl_atm_forc_calc (cp_nl_energy_forc.C:121-182): returns occ E_NL of the
// state, scales z in place, accumulates the atom forces (read by ref_sf_forces)
double ref_sf_atm_forc(double* z, double* zx, double* zy, double* zz, int state) {
  double enl = 0.0;
  CPNONLOCAL::CP_enl_atm_forc_calc(1, 0, &s_atoms, reinterpret_cast<complex*>(z),
                                   reinterpret_cast<complex*>(zx),
                                   reinterpret_cast<complex*>(zy),
                                   reinterpret_cast<complex*>(zz), &enl, 1, state);
  return enl;
}

void ref_sf_forces(double* f) {
  for (size_t i = 0; i < s_fx.size(); ++i) {
    f[3 * i] = s_fx[i];
    f[3 * i + 1] = s_fy[i];
    f[3 * i + 2] = s_fz[i];
  }
}

// CP_enl_force_calc (cp_nl_energy_forc.C:29-114): forces (complex n) -= z' S
void ref_sf_psi_force(double* z, int n, int* kx, int* ky, int* kz, double* s, double* forces,
                      int state) {
  CPNONLOCAL::CP_enl_force_calc(reinterpret_cast<complex*>(z), n, kx, ky, kz,
                                reinterpret_cast<complex*>(s), reinterpret_cast<complex*>(forces),
                                state, 1, 1, 0);
}

}  // extern "C"
