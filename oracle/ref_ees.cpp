// C entry points around the reference's EES non-local routines, compiled by
// build_ref.sh from their own sources (cp_ees_nonlocal.C, set_cp_ewald.C) with
// the PINY singletons below filled for one Gamma-point system.  Test
// infrastructure only: oracle/ees.py is pinned to these.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "standard_include.h"
#include "ckcomplex.h"
#include "../../include/Atoms.h"
#include "../../include/eesDataClass.h"
#include "allclass_cp.h"
#include "allclass_gen.h"
#include "CP_OPERATIONS/class_cpnonlocal.h"

// GEN_WAVE's constructor lives in gen_wave.C, which the oracle does not build;
// the singleton's wave-generation member is never read here.
GEN_WAVE::GEN_WAVE() {}
GEN_WAVE::~GEN_WAVE() {}

CP readonly_cp;
GENERAL_DATA readonly_general_data;

// determinant of a 1-based 3x3 (only referenced by set_cp_ewald.C routines the
// oracle does not call)
double getdeth(double* h) {
  return h[1] * (h[5] * h[9] - h[8] * h[6]) - h[4] * (h[2] * h[9] - h[8] * h[3]) +
         h[7] * (h[2] * h[6] - h[5] * h[3]);
}

void init_nonlocal_ees(int* kmax, double ecut, PSNONLOCAL* psnonlocal, int fft_opt);

namespace {
std::vector<double> g_vps[4], g_gz, g_norm, g_occ, g_wk, g_kp;
std::vector<int> g_map, g_natm_lang, g_str, g_lang, g_mang, g_ityp;
std::vector<int*> g_typ_lang_rows;
std::vector<std::vector<int>> g_typ_lang;
int g_natm = 0, g_ntyp = 0, g_nchan = 0;

double* one_based(std::vector<double>& v) { return v.data() - 1; }
int* one_based_i(std::vector<int>& v) { return v.data() - 1; }

struct Scratch {
  PSSCRATCH ps;
  std::vector<double> d[20];
  std::vector<int> i[12];
  std::vector<double*> dp[12];
  std::vector<int*> ip[3];
};
Scratch* g_scr = nullptr;

void alloc_scratch(int natm, int n) {
  delete g_scr;
  g_scr = new Scratch();
  Scratch& s = *g_scr;
  PSSCRATCH& p = s.ps;
  auto vd = [&](int k, int len) { s.d[k].assign(len + 1, 0.0); return s.d[k].data(); };
  auto vi = [&](int k, int len) { s.i[k].assign(len + 1, 0); return s.i[k].data(); };
  p.aj = vd(0, n); p.rn = vd(1, n); p.rn1 = vd(2, n);
  p.index_a = vi(0, n); p.index_b = vi(1, n); p.igrid_at = vi(2, n); p.igrid_bt = vi(3, n);
  p.frac_a = vd(3, natm); p.frac_b = vd(4, natm); p.frac_c = vd(5, natm);
  p.iatemp = vi(4, natm); p.ibtemp = vi(5, natm); p.ictemp = vi(6, natm);
  // [1..n][0..natm-1] matrices
  double*** dm[12] = {&p.mn_a, &p.mn_b, &p.mn_c, &p.ua, &p.ub, &p.uc,
                      &p.dmn_a, &p.dmn_b, &p.dmn_c, nullptr, nullptr, nullptr};
  for (int k = 0; k < 9; ++k) {
    s.d[8 + k].assign((size_t)(n + 1) * natm, 0.0);
    s.dp[k].assign(n + 1, nullptr);
    for (int j = 1; j <= n; ++j) s.dp[k][j] = s.d[8 + k].data() + (size_t)j * natm;
    *dm[k] = s.dp[k].data();
  }
  int*** im[3] = {&p.igrid_a, &p.igrid_b, &p.igrid_c};
  for (int k = 0; k < 3; ++k) {
    s.i[7 + k].assign((size_t)(n + 1) * natm, 0);
    s.ip[k].assign(n + 1, nullptr);
    for (int j = 1; j <= n; ++j) s.ip[k][j] = s.i[7 + k].data() + (size_t)j * natm;
    *im[k] = s.ip[k].data();
  }
}

// per-plane RPPDATA storage
struct Planes {
  std::vector<RPPDATA> rpp;
  std::vector<RPPDATA*> ptr;
  std::vector<std::vector<int>> pidx;
  std::vector<std::vector<int>> ig;
  std::vector<std::vector<double>> m, dx, dy, dz;
  std::vector<std::vector<int*>> igr;
  std::vector<std::vector<double*>> mr, dxr, dyr, dzr;
};
Planes* g_pl = nullptr;
}  // namespace

extern "C" {

// init_nonlocal_ees (set_cp_ewald.C:1329-1400) for a cubic box: NL grid size.
int ref_nl_grid_size(int kmax, double scale, int n_interp) {
  PSNONLOCAL nl;
  nl.n_interp = n_interp;
  nl.fft_size_scale = scale;
  int km[4] = {0, kmax, kmax, kmax};
  init_nonlocal_ees(km, 0.0, &nl, 0);
  return nl.ngrid_a;
}

// Fill the PINY singletons for one Gamma-point system with EES non-local.
//   typ[natm] 0-based types; channels c = 0..nchan-1 with type, l, m;
//   vnl[ntyp][lmax+1][4][nspl] spline tables (v0..v3), gz[ntyp] the G=0 s value,
//   vnorm[ntyp][lmax+1]; occ[nstate]; hmati[9] column-major 0-based.
void ref_ees_setup(int nkf, int n_interp, const double* hmati, double vol, int nspl,
                   double gmin, double dg, int ntyp, int lmax, const double* vnl,
                   const double* gz, const double* vnorm, int natm, const int* typ, int nchan,
                   const int* ch_type, const int* ch_l, const int* ch_m, int nstate,
                   const double* occ) {
  CP* cp = &readonly_cp;
  GENERAL_DATA* gd = &readonly_general_data;
  CPPSEUDO* ps = &cp->cppseudo;
  PSNONLOCAL* nl = &ps->nonlocal;
  g_natm = natm;
  g_ntyp = ntyp;
  g_nchan = nchan;
  // GENCELL owns its hmati array (constructor/destructor): fill it in place
  for (int k = 0; k < 9; ++k) gd->gencell.hmati[k + 1] = hmati[k];
  gd->gencell.vol = vol;
  ps->nsplin_g = nspl;
  ps->gmin_spl = gmin;
  ps->dg_spl = dg;
  ps->n_ang_max = lmax;
  ps->n_interp_ps = n_interp;
  const size_t tab = (size_t)ntyp * (lmax + 1) * nspl;
  for (int k = 0; k < 4; ++k) {
    g_vps[k].assign(tab, 0.0);
    for (int t = 0; t < ntyp; ++t)
      for (int l = 0; l <= lmax; ++l)
        for (int i = 0; i < nspl; ++i)
          g_vps[k][((size_t)t * (lmax + 1) + l) * nspl + i] =
              vnl[(((size_t)t * (lmax + 1) + l) * 4 + k) * nspl + i];
  }
  ps->vps0 = one_based(g_vps[0]);
  ps->vps1 = one_based(g_vps[1]);
  ps->vps2 = one_based(g_vps[2]);
  ps->vps3 = one_based(g_vps[3]);
  g_gz.assign(gz, gz + ntyp);
  ps->gzvps0 = one_based(g_gz);
  g_norm.assign(vnorm, vnorm + (size_t)ntyp * (lmax + 1));
  ps->vpsnorm = one_based(g_norm);
  // non-local atom list in type order; map_nl[1-based nl index] = 1-based atom
  g_map.clear();
  g_natm_lang.assign(ntyp, 0);
  g_str.assign(ntyp, 0);
  int at = 1;
  for (int t = 0; t < ntyp; ++t) {
    g_str[t] = at;
    for (int i = 0; i < natm; ++i)
      if (typ[i] == t) {
        g_map.push_back(i + 1);
        ++g_natm_lang[t];
        ++at;
      }
  }
  nl->natm = natm;
  nl->natm_tot = natm;
  nl->n_interp = n_interp;
  nl->n_interp2 = n_interp * n_interp;
  nl->ngrid_a = nl->ngrid_b = nl->ngrid_c = nkf;
  nl->map_nl = one_based_i(g_map);
  nl->natm_lang = one_based_i(g_natm_lang);
  nl->iatm_str_lang = one_based_i(g_str);
  // iatm_typ_lang[ityp][lang+1] = true type: identity (ityp is the true type)
  g_typ_lang.assign(ntyp, std::vector<int>(lmax + 2, 0));
  g_typ_lang_rows.assign(ntyp, nullptr);
  for (int t = 0; t < ntyp; ++t) {
    for (int l = 0; l <= lmax; ++l) g_typ_lang[t][l + 1] = t + 1;
    g_typ_lang_rows[t] = g_typ_lang[t].data();
  }
  nl->iatm_typ_lang = g_typ_lang_rows.data() - 1;
  g_lang.assign(ch_l, ch_l + nchan);
  g_mang.assign(ch_m, ch_m + nchan);
  g_ityp.resize(nchan);
  for (int c = 0; c < nchan; ++c) g_ityp[c] = ch_type[c] + 1;
  nl->lang_v = one_based_i(g_lang);
  nl->mang_v = one_based_i(g_mang);
  nl->ityp_v = one_based_i(g_ityp);
  nl->nl_iter = nchan;
  // Gamma point, double pack
  g_occ.assign(occ, occ + nstate);
  cp->cpcoeffs_info.occ_up = one_based(g_occ);
  g_wk.assign(1, 1.0);
  cp->cpcoeffs_info.wght_kpt = one_based(g_wk);
  cp->cpcoeffs_info.nkpoint = 1;
  cp->cpcoeffs_info.igamma_kpt_ind = 1;
  g_kp.assign(1, 0.0);
  cp->cpewald.akpoint = one_based(g_kp);
  cp->cpewald.bkpoint = one_based(g_kp);
  cp->cpewald.ckpoint = one_based(g_kp);
  cp->cpewald.doublepack = 1;
  const double fpi = 4.0 * M_PI;
  CPYLM_CONS* y = &cp->cpylm_cons;
  y->rt_fpi = 1.0 / sqrt(fpi);
  y->rt_thrfpi = sqrt(3.0 / fpi);
  y->rt_threpi = sqrt(1.50 / fpi);
  y->hrt_fivfpi = 0.50 * sqrt(5.0 / fpi);
  y->rt_fiftepi = sqrt(7.50 / fpi);
  y->hrt_sevfpi = 0.50 * sqrt(7.0 / fpi);
  y->hrt_toepi = 0.50 * sqrt(10.50 / fpi) / sqrt(2.0);
  y->hrt_ohffpi = 0.50 * sqrt(105.0 / fpi) / sqrt(2.0);
  y->hrt_tfepi = 0.50 * sqrt(17.50 / fpi) / sqrt(2.0);
  alloc_scratch(natm, n_interp);
}

// eesSetEesWghtGgrp (cp_ees_nonlocal.C:60-169): b(G).
void ref_ees_weights(int ncoef, int* ka, int* kb, int* kc, double* bre, double* bim) {
  PSNONLOCAL* nl = &readonly_cp.cppseudo.nonlocal;
  CPNONLOCAL::eesSetEesWghtGgrp(ncoef, ka, kb, kc, bre, bim, nl->ngrid_a, nl->ngrid_b,
                                nl->ngrid_c, nl->n_interp);
}

// eesSplProjectorGgrp (:182-240): spline index (1-based) and offset per point.
void ref_ees_spline(int ncoef, int* ka, int* kb, int* kc, double* h, int* ind) {
  double* hp[1] = {h};
  int* ip[1] = {ind};
  CPNONLOCAL::eesSplProjectorGgrp(ncoef, ka, kb, kc, hp, ip);
}

// eesProjGchare + eesYlmOnD (:594-1236) for channel iter (0-based):
// dyp and projPsiG = conj(dyp psi).  ind_g0 = -1 when G = 0 is absent.
void ref_ees_proj(int ncoef, const double* psi, int* ka, int* kb, int* kc, int ind_g0, int iter,
                  double* dre, double* dim, int* ind, double* h, double* dyp_re,
                  double* dyp_im, double* proj) {
  int* ip[1] = {ind};
  double* hp[1] = {h};
  CPNONLOCAL::eesProjGchare(ncoef, (complex*)psi, ka, kb, kc, ind_g0 >= 0 ? 1 : 0,
                            ind_g0 >= 0 ? ind_g0 : 0, iter + 1, dre, dim, dyp_re, dyp_im,
                            (complex*)proj, ip, hp, 0, 0, 0, 1, 0);
}

// eesAtmBsplineRgrp (:256-580) with every plane allowed.  Outputs per plane p
// and atom i: plane_index[p][i] (0 = off the plane) and, for the n^2 points,
// igrid / mn / dmn_x,y,z [p][i][n^2].
void ref_ees_bspline(const double* xyz, int* plane_index, int* igrid, double* mn, double* dmx,
                     double* dmy, double* dmz) {
  PSNONLOCAL* nl = &readonly_cp.cppseudo.nonlocal;
  const int natm = g_natm, n2 = nl->n_interp * nl->n_interp, np = nl->ngrid_c;
  std::vector<double> x(natm), y(natm), z(natm), f(natm, 0.0);
  for (int i = 0; i < natm; ++i) {
    x[i] = xyz[3 * i];
    y[i] = xyz[3 * i + 1];
    z[i] = xyz[3 * i + 2];
  }
  FastAtoms fa;
  fa.natm = natm;
  fa.x = x.data(); fa.y = y.data(); fa.z = z.data();
  fa.fx = f.data(); fa.fy = f.data(); fa.fz = f.data();
  delete g_pl;
  g_pl = new Planes();
  Planes& P = *g_pl;
  P.rpp.resize(np);
  P.ptr.resize(np);
  P.pidx.assign(np, std::vector<int>(natm, 0));
  P.ig.assign(np, std::vector<int>((size_t)natm * (n2 + 1), 0));
  P.m.assign(np, std::vector<double>((size_t)natm * (n2 + 1), 0.0));
  P.dx = P.m; P.dy = P.m; P.dz = P.m;
  P.igr.assign(np, std::vector<int*>(natm));
  P.mr.assign(np, std::vector<double*>(natm));
  P.dxr = P.mr; P.dyr = P.mr; P.dzr = P.mr;
  std::vector<int> allowed(np, 1);
  for (int p = 0; p < np; ++p) {
    for (int i = 0; i < natm; ++i) {
      P.igr[p][i] = P.ig[p].data() + (size_t)i * (n2 + 1);
      P.mr[p][i] = P.m[p].data() + (size_t)i * (n2 + 1);
      P.dxr[p][i] = P.dx[p].data() + (size_t)i * (n2 + 1);
      P.dyr[p][i] = P.dy[p].data() + (size_t)i * (n2 + 1);
      P.dzr[p][i] = P.dz[p].data() + (size_t)i * (n2 + 1);
    }
    RPPDATA& r = P.rpp[p];
    r.plane_index = P.pidx[p].data();
    r.igrid = P.igr[p].data();
    r.mn = P.mr[p].data();
    r.dmn_x = P.dxr[p].data();
    r.dmn_y = P.dyr[p].data();
    r.dmn_z = P.dzr[p].data();
    P.ptr[p] = &r;
  }
  CPNONLOCAL::eesAtmBsplineRgrp(&fa, allowed.data(), P.ptr.data(), &g_scr->ps);
  for (int p = 0; p < np; ++p)
    for (int i = 0; i < natm; ++i) {
      plane_index[(size_t)p * natm + i] = P.pidx[p][i];
      for (int j = 1; j <= n2; ++j) {
        size_t o = ((size_t)p * natm + i) * n2 + (j - 1);
        igrid[o] = P.ig[p][(size_t)i * (n2 + 1) + j];
        mn[o] = P.m[p][(size_t)i * (n2 + 1) + j];
        dmx[o] = P.dx[p][(size_t)i * (n2 + 1) + j];
        dmy[o] = P.dy[p][(size_t)i * (n2 + 1) + j];
        dmz[o] = P.dz[p][(size_t)i * (n2 + 1) + j];
      }
    }
}

// eesZmatRchare (:1238-1346) over every plane of one state and channel, summed
// over planes in plane order (the reference's plane reduction).  projPsiR is
// [ngrid_c][ngrid_b][ngrid_a + 2].  zmat: [atoms of the channel's type].
void ref_ees_zmat(const double* projPsiR, int iter, int state, double* zmat) {
  PSNONLOCAL* nl = &readonly_cp.cppseudo.nonlocal;
  const int np = nl->ngrid_c, plane = (nl->ngrid_a + 2) * nl->ngrid_b;
  const int t = g_ityp[iter] - 1;
  const int na = g_natm_lang[t];
  std::vector<double> zp(na);
  for (int i = 0; i < na; ++i) zmat[i] = 0.0;
  for (int p = 0; p < np; ++p) {
    CPNONLOCAL::eesZmatRchare(const_cast<double*>(projPsiR) + (size_t)p * plane, iter + 1,
                              zp.data(), g_pl->rpp[p].igrid, g_pl->rpp[p].mn,
                              g_pl->rpp[p].plane_index, state, p);
    for (int i = 0; i < na; ++i) zmat[i] += zp[i];
  }
}

// eesEnergyAtmForcRchare (:1480-1700) on every plane of one state and channel
// with the plane-reduced zmat: the energy (counted once, as the reference's
// reduction plane does), atom forces added to f[natm][3] (full atom order) and
// the scattered projPsiRScr [ngrid_c][ngrid_b][ngrid_a + 2].
double ref_ees_energy_force(const double* zmat, const double* projPsiR, int iter, int state,
                            double* f, double* scr) {
  PSNONLOCAL* nl = &readonly_cp.cppseudo.nonlocal;
  const int np = nl->ngrid_c, plane = (nl->ngrid_a + 2) * nl->ngrid_b;
  const int t = g_ityp[iter] - 1;
  const int na = g_natm_lang[t];
  std::vector<double> fx(g_natm, 0.0), fy(g_natm, 0.0), fz(g_natm, 0.0), z(na);
  FastAtoms fa;
  fa.natm = g_natm;
  fa.fx = fx.data(); fa.fy = fy.data(); fa.fz = fz.data();
  double e_first = 0.0;
  for (int p = 0; p < np; ++p) {
    for (int i = 0; i < na; ++i) z[i] = zmat[i];
    double e = 0.0;
    CPNONLOCAL::eesEnergyAtmForcRchare(iter + 1, &e, z.data(), g_pl->rpp[p].igrid,
                                       g_pl->rpp[p].mn, g_pl->rpp[p].dmn_x, g_pl->rpp[p].dmn_y,
                                       g_pl->rpp[p].dmn_z, const_cast<double*>(projPsiR) +
                                       (size_t)p * plane, scr + (size_t)p * plane,
                                       g_pl->rpp[p].plane_index, nullptr, nullptr, p, state,
                                       0, &fa);
    if (p == 0) e_first = e;
  }
  for (int i = 0; i < g_natm; ++i) {
    f[3 * i] += fx[i];
    f[3 * i + 1] += fy[i];
    f[3 * i + 2] += fz[i];
  }
  return e_first;
}

// eesPsiForcGspace (:2000-2064): fpsi += -w conj(dyp projPsiG); the first nkx0
// points carry weight 1.  projPsiG and dyp_im are modified at G = 0 as in the
// reference.
void ref_ees_psi_force(int ncoef, int ind_g0, int nkx0, double* projPsiG, double* fpsi,
                       double* dyp_re, double* dyp_im, int* ka, int* kb, int* kc) {
  CPNONLOCAL::eesPsiForcGspace(ncoef, ind_g0 >= 0 ? 1 : 0, ind_g0 >= 0 ? ind_g0 : 0, nkx0,
                               (complex*)projPsiG, (complex*)fpsi, dyp_re, dyp_im, ka, kb, kc,
                               0, 0, 1, 1, 0);
}
}
