// The CP electronic step: forces -> orthonormality constraint -> Verlet
// update of the coefficients -> Loewdin re-orthonormalisation.
//
//   CPINTEGRATE::CP_integrate_dyn / cp_evolve_vel / get_fictKE
//                  src_piny_physics_v1.0/abinito_physics/cp_integrate/cp_dynamics.C:29-258
//   set_cpmass     src_piny_physics_v1.0/interface/cp_ewald/set_cp_ewald.C:32-74
//   Gx=0 redundant half sync  CP_State_GSpacePlane::sendRedPsi/unpackRedPsi
//                  cp_state_ctrl/CP_State_GSpacePlane.C:2862-3061
//   lambda, constrained force, S, T, psi.T  (PairCalculator / Ortho, see paircalc.cu, ortho.cu)
//
// Point classes of the packed layout (the reference's nkx0_red / nkx0_zero /
// nkx0_uni ranges of every chunk): 0 = redundant lower Gx=0 half (overwritten
// by the conjugate of its partner, not integrated), 1 = G=0 (imaginary parts
// zeroed), 2 = unique Gx=0 (force and mass doubled), 3 = Gx>0.
#include <algorithm>
#include <cmath>
#include <vector>
#include "ctx.cuh"

namespace stp {

// The whole Verlet update in one pass over psi, v and F (the two kicks, the
// fictitious KE between them, the drift), in the per-element order of the
// reference's half steps: second half kick of the previous step when
// `first`, KE, first half kick, psi += v dt.
__global__ void k_integrate(double2* __restrict__ psi, double2* __restrict__ v,
                            const double2* __restrict__ f, const double* __restrict__ cmass,
                            const int* __restrict__ cls, int npts, int nstates, double dt,
                            int first, double* __restrict__ ke_part) {
  __shared__ double red[32];
  double ke = 0.0;
  const double dt2 = 0.5 * dt;
  const size_t n = (size_t)npts * nstates;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    int p = (int)(i % npts);
    int c = cls[p];
    if (c == 0) continue;
    double m = cmass[p];
    double2 vv = v[i];
    double2 ff = f[i];
    if (c == 1) { vv.y = 0.0; ff.y = 0.0; }
    const double fm = (c == 2) ? (2.0 * dt2) / (2.0 * m) : dt2 / m;
    if (first) {
      vv.x += ff.x * fm;
      vv.y += ff.y * fm;
      if (c == 1) vv.y = 0.0;
    }
    ke += (vv.x * vv.x + vv.y * vv.y) * (c == 2 ? 2.0 * m : m);
    vv.x += ff.x * fm;
    vv.y += ff.y * fm;
    if (c == 1) vv.y = 0.0;
    v[i] = vv;
    double2 a = psi[i];
    a.x += vv.x * dt;
    a.y += vv.y * dt;
    psi[i] = a;
  }
  double t = block_sum(ke, red);
  if (threadIdx.x == 0) ke_part[blockIdx.x] = 0.5 * t;
}

// After the drift, the redundant half mirrors its partner:
// psi(0,-ky,-kz) = conj psi(0,ky,kz) (and the same for v).
__global__ void k_sync_red(double2* __restrict__ psi, double2* __restrict__ v,
                           const int* __restrict__ red_idx, const int* __restrict__ red_src,
                           int nred, int npts, int nstates) {
  const size_t n = (size_t)nred * nstates;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    int s = (int)(i / nred), r = (int)(i % nred);
    size_t d = (size_t)s * npts + red_idx[r], q = (size_t)s * npts + red_src[r];
    double2 a = psi[q];
    psi[d] = make_double2(a.x, -a.y);
    if (v) {
      double2 b = v[q];
      v[d] = make_double2(b.x, -b.y);
    }
  }
}

__global__ void k_sum(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  double t = block_sum(s, red);
  if (threadIdx.x == 0) *out = t;
}

// energies[KE] = sum eke[s]; energies[TOT] = KE + NL + HART + EXT + EXC
__global__ void k_energy_tot(const double* __restrict__ eke, int nstates,
                             double* __restrict__ e) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double k = 0.0;
    for (int s = 0; s < nstates; ++s) k += eke[s];
    e[CPSTEP_E_KE] = k;
    e[CPSTEP_E_TOT] = k + e[CPSTEP_E_NL] + e[CPSTEP_E_HART] + e[CPSTEP_E_EXT] + e[CPSTEP_E_EXC];
  }
}

}  // namespace stp

// ===========================================================================

int step_init_classes(cpstep_ctx* c) {
  const int np = c->npts;
  std::vector<int> cls(np);
  std::vector<int> ridx, rsrc;
  // partner lookup on the Gx=0 plane
  int kymax = 0, kzmax = 0;
  for (int i = 0; i < np; ++i) {
    if (c->h_kx[i] == 0) {
      kymax = std::max(kymax, std::abs(c->h_ky[i]));
      kzmax = std::max(kzmax, std::abs(c->h_kz[i]));
    }
  }
  const int wy = 2 * kymax + 1, wz = 2 * kzmax + 1;
  std::vector<int> where((size_t)wy * wz, -1);
  for (int i = 0; i < np; ++i)
    if (c->h_kx[i] == 0) where[(size_t)(c->h_ky[i] + kymax) * wz + (c->h_kz[i] + kzmax)] = i;
  for (int i = 0; i < np; ++i) {
    int kx = c->h_kx[i], ky = c->h_ky[i], kz = c->h_kz[i];
    if (kx != 0) {
      cls[i] = 3;
    } else if (ky == 0 && kz == 0) {
      cls[i] = 1;
    } else if (ky > 0 || (ky == 0 && kz > 0)) {
      cls[i] = 2;
    } else {
      cls[i] = 0;
      int src = where[(size_t)(-ky + kymax) * wz + (-kz + kzmax)];
      if (src < 0) {
        cpstep_set_error("layout: Gx=0 point (0,%d,%d) has no stored partner", ky, kz);
        return CPSTEP_ERR_LAYOUT;
      }
      ridx.push_back(i);
      rsrc.push_back(src);
    }
  }
  c->nred = (int)ridx.size();
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_cls, sizeof(int) * np));
  CPSTEP_CUDA_TRY(cudaMemcpy(c->d_cls, cls.data(), sizeof(int) * np, cudaMemcpyHostToDevice));
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_red_idx, sizeof(int) * std::max(1, c->nred)));
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_red_src, sizeof(int) * std::max(1, c->nred)));
  if (c->nred) {
    CPSTEP_CUDA_TRY(cudaMemcpy(c->d_red_idx, ridx.data(), sizeof(int) * c->nred, cudaMemcpyHostToDevice));
    CPSTEP_CUDA_TRY(cudaMemcpy(c->d_red_src, rsrc.data(), sizeof(int) * c->nred, cudaMemcpyHostToDevice));
  }
  c->nblk_ke = 2 * c->num_sms;
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_step_part, sizeof(double) * (c->nblk_ke + 16)));
  return CPSTEP_OK;
}

void step_free(cpstep_ctx* c) {
  cudaFree(c->d_cls); cudaFree(c->d_red_idx); cudaFree(c->d_red_src); cudaFree(c->d_cmass);
  cudaFree(c->d_step_part); cudaFree(c->d_lambda); cudaFree(c->d_smat); cudaFree(c->d_tmat);
  cudaFree(c->d_psi_tmp); cudaFree(c->d_rho); cudaFree(c->d_vks); cudaFree(c->d_eke);
  cudaFree(c->d_force);
}

// set_cpmass (set_cp_ewald.C:32-74): cmass0 = 4 tau^2 CP_EMAGIC (tau in a.u.),
// cmass = cmass0 * max(1, (g^2/2) / (cut/2)) above the mass cutoff, cmass(G=0) = cmass0/2.
int step_set_mass(cpstep_ctx* c, double tau_fs, double cut_ry) {
  const double time_conv = 0.0241888, emagic = 0.00050;
  double tau = tau_fs / time_conv;
  double m0 = 4.0 * tau * tau * emagic;
  std::vector<double> cm(c->npts);
  std::vector<double> g2(c->npts);
  CPSTEP_CUDA_TRY(cudaMemcpy(g2.data(), c->d_g2, sizeof(double) * c->npts, cudaMemcpyDeviceToHost));
  for (int i = 0; i < c->npts; ++i) {
    double en = 0.5 * g2[i];
    bool g0 = (c->h_kx[i] == 0 && c->h_ky[i] == 0 && c->h_kz[i] == 0);
    cm[i] = g0 ? 0.5 * m0 : (en > 0.5 * cut_ry ? m0 * en / (0.5 * cut_ry) : m0);
  }
  if (!c->d_cmass) CPSTEP_CUDA_TRY(cudaMalloc(&c->d_cmass, sizeof(double) * c->npts));
  CPSTEP_CUDA_TRY(cudaMemcpy(c->d_cmass, cm.data(), sizeof(double) * c->npts, cudaMemcpyHostToDevice));
  return CPSTEP_OK;
}

// Velocity Verlet of CP_integrate_dyn: second half kick of the previous step
// (iteration > 1), fictitious KE, first half kick, drift (with the isokinetic
// NHC of nhc.cu around the kicks when the thermostat is on), and the
// redundant-half sync.  d_enhc (2 doubles, may be NULL): the NHC kinetic
// energy and potential of get_fictKE, zero without the thermostat.
int step_integrate(cpstep_ctx* c, const double* force, double* psi, double* vpsi, double dt,
                   int iteration, double* d_fict_ke, double* d_enhc) {
  if (!c->d_cmass) {
    cpstep_set_error("integrate: CP masses not set (cpstep_set_cp_mass)");
    return CPSTEP_ERR_STATE;
  }
  double2* p = reinterpret_cast<double2*>(psi);
  double2* v = reinterpret_cast<double2*>(vpsi);
  const double2* f = reinterpret_cast<const double2*>(force);
  int nb = c->nblk_ke;
  if (c->nhc.on) {
    int rc = nhc_integrate(c, force, psi, vpsi, dt, iteration, d_fict_ke, d_enhc);
    if (rc) return rc;
    if (c->nred) {
      stp::k_sync_red<<<nb, 256, 0, c->stream>>>(p, v, c->d_red_idx, c->d_red_src, c->nred,
                                                 c->npts, c->nstates);
      CPSTEP_LAUNCH_CHECK();
    }
    return CPSTEP_OK;
  }
  if (d_enhc) CPSTEP_CUDA_TRY(cudaMemsetAsync(d_enhc, 0, 2 * sizeof(double), c->stream));
  stp::k_integrate<<<nb, 256, 0, c->stream>>>(p, v, f, c->d_cmass, c->d_cls, c->npts,
                                              c->nstates, dt, iteration > 1 ? 1 : 0,
                                              c->d_step_part);
  CPSTEP_LAUNCH_CHECK();
  if (d_fict_ke) {
    stp::k_sum<<<1, 256, 0, c->stream>>>(c->d_step_part, nb, d_fict_ke);
    CPSTEP_LAUNCH_CHECK();
  }
  if (c->nred) {
    stp::k_sync_red<<<nb, 256, 0, c->stream>>>(p, v, c->d_red_idx, c->d_red_src, c->nred, c->npts,
                                               c->nstates);
    CPSTEP_LAUNCH_CHECK();
  }
  return CPSTEP_OK;
}

static int ensure_buf(double** p, size_t bytes) {
  if (*p) return CPSTEP_OK;
  CPSTEP_CUDA_TRY(cudaMalloc(p, bytes));
  return CPSTEP_OK;
}

// One CP electronic step on psi (orthonormal on entry and exit).
int step_run(cpstep_ctx* c, double* psi, double* vpsi, const double* occ, double dt,
             int iteration, double* energies, double* atom_force, int ortho_check) {
  const int S = c->nstates;
  const size_t nr = (size_t)c->nx * c->ny * c->nz;
  const size_t ncoef = (size_t)S * c->npts;
  int rc;
  if ((rc = ensure_buf(&c->d_rho, sizeof(double) * nr)) ||
      (rc = ensure_buf(&c->d_vks, sizeof(double) * nr)) ||
      (rc = ensure_buf(&c->d_eke, sizeof(double) * S)) ||
      (rc = ensure_buf(&c->d_force, sizeof(double2) * ncoef)) ||
      (rc = ensure_buf(&c->d_psi_tmp, sizeof(double2) * ncoef)) ||
      (rc = ensure_buf(&c->d_lambda, sizeof(double) * S * S)) ||
      (rc = ensure_buf(&c->d_smat, sizeof(double) * S * S)) ||
      (rc = ensure_buf(&c->d_tmat, sizeof(double) * S * S)))
    return rc;
  if (c->profile && c->prof_pending == cpstep_ctx::PROF_RING) {
    if ((rc = prof_fold(c))) return rc;
  }
  auto mark = [&](int k) {
    if (c->profile)
      cudaEventRecord(c->prof_ev[(size_t)c->prof_pending * (CPSTEP_NPHASE + 1) + k], c->stream);
  };
  mark(0);
  // 1. density and V_KS (XC, Hartree, local pseudopotential, Ewald)
  if ((rc = statefft_density(c, psi, occ, c->d_rho))) return rc;
  mark(1);
  if ((rc = rho_xc(c, c->d_rho, c->d_vks, energies))) return rc;
  if ((rc = rho_r2g(c, c->d_rho))) return rc;
  if (c->xc == CPSTEP_XC_BLYP && (rc = rho_gga(c, c->d_rho, c->d_vks, energies))) return rc;
  if ((rc = rho_hart(c, energies, atom_force))) return rc;
  if ((rc = rho_vks_r(c, c->d_vks))) return rc;
  mark(2);
  // 2. V.psi force with the kinetic term (z-pencils of psi are still valid)
  if ((rc = statefft_vpsi(c, psi, c->d_vks, occ, c->d_force, c->d_eke, 1))) return rc;
  mark(3);
  // 2b. non-local energy, psi force and atom forces (EES or structure factors)
  if (c->nl.on) {
    if ((rc = nl_run(c, psi, occ, c->d_force, energies, atom_force))) return rc;
  } else if (c->sf.on) {
    if ((rc = sf_run(c, psi, occ, c->d_force, energies, atom_force))) return rc;
  } else {
    CPSTEP_CUDA_TRY(cudaMemsetAsync(energies + CPSTEP_E_NL, 0, sizeof(double), c->stream));
  }
  stp::k_energy_tot<<<1, 32, 0, c->stream>>>(c->d_eke, S, energies);
  CPSTEP_LAUNCH_CHECK();
  mark(4);
  // 3. lambda_ji = sum_p Re(conj psi_j F_i); F <- F - (wpt/2) psi.lambda
  const int K = 2 * c->npts;
  if ((rc = pc_overlap_launch(c, psi, c->d_force, S, S, K, nullptr, 1.0, 0.0, c->d_lambda, S))) return rc;
  if ((rc = pc_backmul_w_launch(c, c->d_lambda, S, psi, K, c->d_force, K, S, S, K, -0.5, 1.0,
                                c->d_wpt)))
    return rc;
  mark(5);
  // 4. Verlet update
  if ((rc = step_integrate(c, c->d_force, psi, vpsi, dt, iteration, energies + CPSTEP_E_FICT,
                           energies + CPSTEP_E_NHC_KE)))
    return rc;
  mark(6);
  // 5. S = overlap, T = (S/2)^(-1/2), psi <- psi.T
  if ((rc = pc_overlap_launch(c, psi, psi, S, S, K, c->d_wpt, 1.0, 0.0, c->d_smat, S))) return rc;
  const int mixed = c->precision == CPSTEP_PREC_MIXED;
  if ((rc = ortho_tmat(c, c->d_smat, c->d_tmat, S, mixed, 0, mixed ? 2e-6 : 1e-15,
                       mixed ? 20 : 10, nullptr, nullptr, ortho_check)))
    return rc;
  if ((rc = pc_backmul_launch(c, c->d_tmat, S, psi, K, c->d_psi_tmp, K, S, S, K, 1.0, 0.0))) return rc;
  CPSTEP_CUDA_TRY(cudaMemcpyAsync(psi, c->d_psi_tmp, sizeof(double2) * ncoef,
                                  cudaMemcpyDeviceToDevice, c->stream));
  mark(7);
  if (c->profile) c->prof_pending += 1;
  return CPSTEP_OK;
}
