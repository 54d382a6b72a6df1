// C entry point around the reference's NVT atom integrator with massive
// Nose-Hoover chains, ATOMINTEGRATE::integrate_nvt_2nd_half / _1st_half /
// applyNHC / computeEkin / computeENHC (classical_physics/integrate/
// integration_drivers.C:89-190, :337-565), compiled by build_ref.sh from its
// own source.  Test infrastructure only: oracle/atomnhc.py is pinned to this.
#include <vector>
#include "standard_include.h"
#include "ckcomplex.h"
#include "../../include/Atoms.h"
#include "allclass_gen.h"
#include "allclass_mdintegrate.h"
#include "ATOM_OPERATIONS/class_atomintegrate.h"

MDINTEGRATE readonly_mdintegrate;

extern "C" {

// One MD step of the NVT branch of ctrl_atom_integrate: the second half of the
// previous step (itime > 0), E_kin and the NHC energies, the first half.
// xyz, vel, f: [natm][3]; mass, kT, posKT: [natm]; mnhc: [natm][len];
// vnhc: [natm][3][len] (x, y, z chains); out3 = {E_kin, E_kin NHC, pot NHC}.
void ref_atom_nvt_step(int natm, int len, int itime, double* xyz, double* vel, const double* f,
                       const double* mass, const double* kT, const double* mnhc, double* vnhc,
                       double* posKT, double dt, int nres, int nyosh, double* out3) {
  GENERAL_DATA::get()->gentimeinfo.dt = dt;
  MDINTEGRATE::get()->mdtherm_info.nres_nhc = nres;
  MDINTEGRATE::get()->mdtherm_info.nyosh_nhc = nyosh;
  std::vector<Atom> at(natm);
  std::vector<AtomNHC> an(natm);
  for (int i = 0; i < natm; ++i) {
    at[i].x = xyz[3 * i]; at[i].y = xyz[3 * i + 1]; at[i].z = xyz[3 * i + 2];
    at[i].vx = vel[3 * i]; at[i].vy = vel[3 * i + 1]; at[i].vz = vel[3 * i + 2];
    at[i].fx = f[3 * i]; at[i].fy = f[3 * i + 1]; at[i].fz = f[3 * i + 2];
    at[i].m = mass[i];
    an[i].len_nhc = len;
    an[i].kT = kT[i];
    an[i].posKT = posKT[i];
    for (int j = 0; j < len; ++j) {
      an[i].m[j] = mnhc[i * len + j];
      an[i].vx[j] = vnhc[(i * 3 + 0) * len + j];
      an[i].vy[j] = vnhc[(i * 3 + 1) * len + j];
      an[i].vz[j] = vnhc[(i * 3 + 2) * len + j];
    }
  }
  ATOMINTEGRATE::integrate_nvt_2nd_half(itime, natm, len, at.data(), an.data(), &out3[0],
                                        &out3[1], &out3[2], natm, 0, natm);
  ATOMINTEGRATE::integrate_nvt_1st_half(natm, len, at.data(), an.data(), natm, 0, natm, false,
                                        1.0);
  for (int i = 0; i < natm; ++i) {
    xyz[3 * i] = at[i].x; xyz[3 * i + 1] = at[i].y; xyz[3 * i + 2] = at[i].z;
    vel[3 * i] = at[i].vx; vel[3 * i + 1] = at[i].vy; vel[3 * i + 2] = at[i].vz;
    posKT[i] = an[i].posKT;
    for (int j = 0; j < len; ++j) {
      vnhc[(i * 3 + 0) * len + j] = an[i].vx[j];
      vnhc[(i * 3 + 1) * len + j] = an[i].vy[j];
      vnhc[(i * 3 + 2) * len + j] = an[i].vz[j];
    }
  }
}

}  // extern "C"
