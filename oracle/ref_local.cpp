// C entry points around reference routines of the electronic step that the
// oracle restates, compiled by build_ref.sh from their own sources:
//   CPNONLOCAL::CP_eke_calc       abinito_physics/cp_nonlocal/cp_eke.C:30-140
//   CPLOCAL::CP_hart_eext_calc    abinito_physics/cp_local/cp_hart_ext.C:56-405
//   FFTcache::expandGSpace / packGSpace   fft_slab_ctrl/fftCache.C:460-553 (the
//                                 two member functions, cut from the file by
//                                 build_ref.sh: the rest of it needs Charm++)
//   CPLOCAL::eesAtmBsplineRgrp, eesPackGridRchare, eesSetEesWghtGgrp,
//   eesHartEextGchare, eesEwaldGchare, eesAtmForceRchare
//                                 cp_local/cp_hart_ext.C:521-1470 (the EES form)
// with the PINY singletons of ref_ees.cpp / ref_ion.cpp filled for one
// Gamma-point, spin-unpolarised, fully periodic system.  Test infrastructure
// only: oracle/fftpath.py (eke, expand, pack), oracle/density.py
// (hart_eext) and oracle/eext_ees.py are pinned to these.
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

// ---------------------------------------------------------------------------
// The EES form of the local pass (cp_eext_ees_opt): CPLOCAL::eesAtmBsplineRgrp,
// eesPackGridRchare, eesSetEesWghtGgrp, eesHartEextGchare, eesEwaldGchare and
// eesAtmForceRchare (cp_hart_ext.C:521-1470) on one chare that owns the whole
// EES grid (planes 0..N-1, rows 0..N-1; rows of 2 (N/2 + 1) reals).
namespace {

struct EesLocal {
  int n = 0, ni = 0, natm = 0;
  PSSCRATCH ps;
  std::vector<double> sd[12];
  std::vector<int> si[6];
  std::vector<double*> sdp[9];
  std::vector<int*> sip[3];
  RHORHARTDATA rd;
  std::vector<int> pidx, nsub, itmp, ig;
  std::vector<double> m, dx, dy, dz;
  std::vector<int*> pidx_r, nsub_r, itmp_r;
  std::vector<int**> ig_c;
  std::vector<int*> ig_r;
  std::vector<double**> m_c, dx_c, dy_c, dz_c;
  std::vector<double*> m_r, dx_r, dy_r, dz_r;
  std::vector<double> store[9];
  std::vector<int> istore[3];
  std::vector<double> x, y, z, q, fx, fy, fz;
  std::vector<int> natm_eext;
  std::vector<std::vector<int>> map_rows;
  std::vector<int*> map_ptr;
  std::vector<double> q_typ;
  FastAtoms fa;
};

// singletons and B-splines of the atoms on the EES grid (eesAtmBsplineRgrp)
void ees_local_setup(EesLocal& e, int natm, int ntyp, const int* typ, const double* xyz,
                     const double* q, const double* qtyp, const double* hmati, double vol,
                     int ngrid, int n_interp) {
  CP* cp = CP::get();
  GENERAL_DATA* gd = GENERAL_DATA::get();
  MDATOMS* md = MDATOMS::get();
  for (int k = 0; k < 9; ++k) gd->gencell.hmati[k + 1] = hmati[k];
  gd->gencell.vol = vol;
  CPPSEUDO* ps = &cp->cppseudo;
  ps->n_interp_ps = n_interp;
  ps->ngrid_eext_a = ps->ngrid_eext_b = ps->ngrid_eext_c = ngrid;
  ps->natm_typ = ntyp;
  md->mdclatoms_info.natm_tot = natm;
  e.n = ngrid;
  e.ni = n_interp;
  e.natm = natm;
  // atoms of each type in index order (natm_eext / map_eext, 1-based), and
  // the whole set as type ntyp + 1 (the Ewald pass)
  e.natm_eext.assign(ntyp + 2, 0);
  e.map_rows.assign(ntyp + 2, std::vector<int>(1, 0));
  for (int i = 0; i < natm; ++i) {
    e.natm_eext[typ[i] + 1]++;
    e.map_rows[typ[i] + 1].push_back(i + 1);
  }
  e.natm_eext[ntyp + 1] = natm;
  e.map_ptr.assign(ntyp + 2, nullptr);
  for (int t = 1; t <= ntyp + 1; ++t) e.map_ptr[t] = e.map_rows[t].data();
  ps->natm_eext = e.natm_eext.data();
  ps->map_eext = e.map_ptr.data();
  e.q_typ.assign(ntyp + 1, 0.0);
  for (int t = 0; t < ntyp && qtyp; ++t) e.q_typ[t + 1] = qtyp[t];
  ps->q_typ = e.q_typ.data();
  // scratch: [1..n] vectors, [0..natm) vectors, [1..n][0..natm) matrices
  PSSCRATCH& p = e.ps;
  const int n = n_interp;
  auto vd = [&](int k, int len) { e.sd[k].assign(len + 1, 0.0); return e.sd[k].data(); };
  auto vi = [&](int k, int len) { e.si[k].assign(len + 1, 0); return e.si[k].data(); };
  p.aj = vd(0, n); p.rn = vd(1, n); p.rn1 = vd(2, n);
  p.frac_a = vd(3, natm); p.frac_b = vd(4, natm); p.frac_c = vd(5, natm);
  p.iatemp = vi(0, natm); p.ibtemp = vi(1, natm); p.ictemp = vi(2, natm);
  double*** dm[9] = {&p.mn_a, &p.mn_b, &p.mn_c, &p.ua, &p.ub, &p.uc,
                     &p.dmn_a, &p.dmn_b, &p.dmn_c};
  for (int k = 0; k < 9; ++k) {
    e.store[k].assign((size_t)(n + 1) * natm, 0.0);
    e.sdp[k].assign(n + 1, nullptr);
    for (int j = 1; j <= n; ++j) e.sdp[k][j] = e.store[k].data() + (size_t)j * natm;
    *dm[k] = e.sdp[k].data();
  }
  int*** im[3] = {&p.igrid_a, &p.igrid_b, &p.igrid_c};
  for (int k = 0; k < 3; ++k) {
    e.istore[k].assign((size_t)(n + 1) * natm, 0);
    e.sip[k].assign(n + 1, nullptr);
    for (int j = 1; j <= n; ++j) e.sip[k][j] = e.istore[k].data() + (size_t)j * natm;
    *im[k] = e.sip[k].data();
  }
  // one RHORHARTDATA over the whole grid
  RHORHARTDATA& r = e.rd;
  r.gridc_start = 0; r.gridc_end = ngrid; r.gridb_start = 0; r.gridb_end = ngrid;
  r.mygridc = ngrid; r.mygridb = ngrid;
  r.ngrid_a = r.ngrid_b = r.ngrid_c = ngrid;
  r.n_interp = n;
  r.natm = natm;
  const int nj = n * n + 1;
  e.pidx.assign((size_t)ngrid * natm, 0);
  e.nsub.assign((size_t)ngrid * natm, 0);
  e.itmp.assign((size_t)ngrid * (n + 1), 0);
  e.ig.assign((size_t)ngrid * natm * nj, 0);
  e.m.assign((size_t)ngrid * natm * nj, 0.0);
  e.dx.assign(e.m.size(), 0.0);
  e.dy.assign(e.m.size(), 0.0);
  e.dz.assign(e.m.size(), 0.0);
  e.pidx_r.resize(ngrid); e.nsub_r.resize(ngrid); e.itmp_r.resize(ngrid);
  e.ig_c.resize(ngrid); e.m_c.resize(ngrid); e.dx_c.resize(ngrid); e.dy_c.resize(ngrid);
  e.dz_c.resize(ngrid);
  e.ig_r.resize((size_t)ngrid * natm); e.m_r.resize(e.ig_r.size()); e.dx_r.resize(e.ig_r.size());
  e.dy_r.resize(e.ig_r.size()); e.dz_r.resize(e.ig_r.size());
  for (int c = 0; c < ngrid; ++c) {
    e.pidx_r[c] = e.pidx.data() + (size_t)c * natm;
    e.nsub_r[c] = e.nsub.data() + (size_t)c * natm;
    e.itmp_r[c] = e.itmp.data() + (size_t)c * (n + 1);
    for (int i = 0; i < natm; ++i) {
      const size_t o = ((size_t)c * natm + i) * nj;
      e.ig_r[(size_t)c * natm + i] = e.ig.data() + o;
      e.m_r[(size_t)c * natm + i] = e.m.data() + o;
      e.dx_r[(size_t)c * natm + i] = e.dx.data() + o;
      e.dy_r[(size_t)c * natm + i] = e.dy.data() + o;
      e.dz_r[(size_t)c * natm + i] = e.dz.data() + o;
    }
    e.ig_c[c] = e.ig_r.data() + (size_t)c * natm;
    e.m_c[c] = e.m_r.data() + (size_t)c * natm;
    e.dx_c[c] = e.dx_r.data() + (size_t)c * natm;
    e.dy_c[c] = e.dy_r.data() + (size_t)c * natm;
    e.dz_c[c] = e.dz_r.data() + (size_t)c * natm;
  }
  r.plane_index = e.pidx_r.data(); r.nSub = e.nsub_r.data(); r.itemp = e.itmp_r.data();
  r.igrid = e.ig_c.data(); r.mn = e.m_c.data();
  r.dmn_x = e.dx_c.data(); r.dmn_y = e.dy_c.data(); r.dmn_z = e.dz_c.data();
  e.x.resize(natm); e.y.resize(natm); e.z.resize(natm);
  e.q.assign(natm, 0.0);  // charges: read by the Ewald force pass only
  for (int i = 0; i < natm && q; ++i) e.q[i] = q[i];
  e.fx.assign(natm, 0.0); e.fy.assign(natm, 0.0); e.fz.assign(natm, 0.0);
  for (int i = 0; i < natm; ++i) {
    e.x[i] = xyz[3 * i];
    e.y[i] = xyz[3 * i + 1];
    e.z[i] = xyz[3 * i + 2];
  }
  e.fa.natm = natm;
  e.fa.x = e.x.data(); e.fa.y = e.y.data(); e.fa.z = e.z.data();
  e.fa.q = e.q.data();
  e.fa.fx = e.fx.data(); e.fa.fy = e.fy.data(); e.fa.fz = e.fz.data();
  std::vector<RHORHARTDATA> v(1, r);
  CPLOCAL::eesAtmBsplineRgrp(&e.fa, v, &p);
}

}  // namespace

extern "C" {

// eesPackGridRchare for every type: grids [ntyp][N][N][2 (N/2 + 1)] (planes c,
// rows b, padded a), typ 0-based, xyz [natm][3], hmati column-major.
void ref_eext_ees_spread(int natm, int ntyp, const int* typ, const double* xyz,
                         const double* hmati, double vol, int ngrid, int n_interp,
                         double* grids) {
  EesLocal e;
  ees_local_setup(e, natm, ntyp, typ, xyz, nullptr, nullptr, hmati, vol, ngrid, n_interp);
  const int row = 2 * (ngrid / 2 + 1);
  const int size = ngrid * ngrid * row;
  for (int t = 1; t <= ntyp; ++t)
    CPLOCAL::eesPackGridRchare(natm, t, grids + (size_t)(t - 1) * size, 0, ngrid, 0, ngrid, size,
                               e.rd.igrid, e.rd.mn, e.rd.plane_index, e.rd.nSub);
}

// eesSetEesWghtGgrp, then eesHartEextGchare for types 1..ntyp and
// eesEwaldGchare on the packed density sphere (point i at offset i).
// sfg [ntyp][npts] complex: the transformed spread grids at the points, on
// return the per-type force terms; stot [npts] complex out; rho the
// reference's rho(G); vks [npts] complex out; e = {ehart, eext, ewd}.
void ref_eext_ees_gspace(int npts, const int* kx, const int* ky, const int* kz, const double* rho,
                         double ecut_ha, const double* hmati, double vol, double alp_ewd,
                         int ngrid, int n_interp, int ntyp, const double* qtyp, int nspl,
                         double gmin, double dg, const double* vloc, const double* gzvps,
                         double* sfg, double* stot, double* vks, double* e) {
  CP* cp = CP::get();
  GENERAL_DATA* gd = GENERAL_DATA::get();
  for (int k = 0; k < 9; ++k) gd->gencell.hmati[k + 1] = hmati[k];
  gd->gencell.vol = vol;
  gd->genewald.alp_ewd = alp_ewd;
  cp->cpcoeffs_info.ecut = ecut_ha;
  CPPSEUDO* ps = &cp->cppseudo;
  ps->n_interp_ps = n_interp;
  ps->ngrid_eext_a = ps->ngrid_eext_b = ps->ngrid_eext_c = ngrid;
  ps->natm_typ = ntyp;
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
  std::vector<double> qt(qtyp, qtyp + ntyp);
  ps->q_typ = qt.data() - 1;
  std::vector<gridPoint> pts(npts);
  for (int i = 0; i < npts; ++i) {
    pts[i].d1 = kz[i];
    pts[i].d2 = ky[i];
    pts[i].d3 = kx[i];
    pts[i].offset = i;
  }
  std::vector<double> bre(npts), bim(npts);
  CPLOCAL::eesSetEesWghtGgrp(npts, pts, bre.data(), bim.data(), ngrid, ngrid, ngrid, n_interp);
  for (int i = 0; i < 2 * npts; ++i) {
    vks[i] = 0.0;
    stot[i] = 0.0;
  }
  e[0] = e[1] = e[2] = 0.0;
  for (int t = 1; t <= ntyp; ++t)
    CPLOCAL::eesHartEextGchare(npts, t, reinterpret_cast<complex*>(const_cast<double*>(rho)),
                               reinterpret_cast<complex*>(vks),
                               reinterpret_cast<complex*>(sfg + (size_t)(t - 1) * 2 * npts),
                               reinterpret_cast<complex*>(stot), bre.data(), bim.data(), &e[0],
                               &e[1], pts, nullptr, 0, 1);
  CPLOCAL::eesEwaldGchare(npts, reinterpret_cast<complex*>(stot), bre.data(), bim.data(), &e[2],
                          pts, 1, nullptr, 0, 1);
}

// eesAtmForceRchare: grids [ntyp + 1][N][N][2 (N/2 + 1)] the back-transformed
// per-type terms and the Ewald term; f [natm][3] += the atom forces.
void ref_eext_ees_force(int natm, int ntyp, const int* typ, const double* xyz, const double* q,
                        const double* hmati, double vol, int ngrid, int n_interp,
                        const double* grids, double* f) {
  EesLocal e;
  ees_local_setup(e, natm, ntyp, typ, xyz, q, nullptr, hmati, vol, ngrid, n_interp);
  const size_t size = (size_t)ngrid * ngrid * 2 * (ngrid / 2 + 1);
  for (int t = 1; t <= ntyp + 1; ++t)
    CPLOCAL::eesAtmForceRchare(natm, &e.fa, t <= ntyp ? t : ntyp, e.rd.igrid, e.rd.dmn_x,
                               e.rd.dmn_y, e.rd.dmn_z, e.rd.plane_index, e.rd.nSub,
                               const_cast<double*>(grids + (t - 1) * size), 0, ngrid, 0, ngrid,
                               t <= ntyp ? 0 : 1);
  for (int i = 0; i < natm; ++i) {
    f[3 * i] += e.fx[i];
    f[3 * i + 1] += e.fy[i];
    f[3 * i + 2] += e.fz[i];
  }
}

}  // extern "C"
