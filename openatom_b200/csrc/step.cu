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
// The constraint of the reference's CP dynamics (CPSTEP_CONSTRAINT_ORTHO_T,
// the default), src_charm_driver/:
//   lambda = <psi_o|F>   asymmetric PairCalculator, alpha = 1 (main/cpaimd.C:2527)
//   gamma = orthoT lambda            orthog_ctrl/ortho.C:541-583 (orthoT: the previous
//                                    step's T, :358-365; the identity after a reset)
//   F_c = F orthoT - W psi_o gamma   paircalc/ckPairCalculator.C:1444-1510 (-F.T) and
//                                    :1372-1420 (gamma), negated by unpackLambda and
//                                    scaled 1/sqrt(2) on Gx=0 by doLambda
//                                    (cp_state_ctrl/CP_State_GSpacePlane.C:2197-2202,
//                                    :2253-2268): W = 1/2 on Gx=0, 1 elsewhere
//   Verlet on the non-orthogonal psi_no (doLambda restores it, integrateModForce)
//   S = overlap(psi_no); max |S - 2I| >= cp_norb_tol fails Ortho::maxCheck
//                                    (ortho.C:255-262, :461-483): fatal on the first
//                                    step, later the finite-difference PsiV reset
//                                    (CP_State_GSpacePlane.C:3707-3770, order 0)
//   psi_o = psi_no T                 (ckPairCalculator.C:1314)
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
// skip (device, may be NULL): nonzero after a PsiV reset, when the reference
// evolves the next step with halfStepEvolve = 0 (no second half kick).
__global__ void k_integrate(double2* __restrict__ psi, double2* __restrict__ v,
                            const double2* __restrict__ f, const double* __restrict__ cmass,
                            const int* __restrict__ cls, int npts, int nstates, double dt,
                            int first_in, const int* __restrict__ skip,
                            double* __restrict__ ke_part) {
  __shared__ double red[32];
  const int first = first_in && !(skip && *skip);
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

// max |S - 2I| over the n x n overlap (Ortho::array_diag_max with diag = 2,
// ortho.h:282-310) against cp_norb_tol (Ortho::maxCheck, ortho.C:461-483):
// after the first step a failure asks for the PsiV reset (flags[0]); on the
// first step it is fatal (flags[3]).  A NaN fails, as !(max < tol) does there.
__global__ void k_norb_check(const double* __restrict__ S, int n, double tol, int later,
                             int* __restrict__ flags, double* __restrict__ dev) {
  __shared__ double red[32];
  double m = 0.0;
  const int nn = n * n;
  for (int i = threadIdx.x; i < nn; i += blockDim.x) {
    const double a = fabs(S[i] - ((i % n) == (i / n) ? 2.0 : 0.0));
    m = (a > m || a != a) ? a : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double b = __shfl_xor_sync(0xffffffffu, m, o);
    m = (b > m || b != b) ? b : m;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = (red[w] > m || red[w] != red[w]) ? red[w] : m;
    *dev = m;
    const int fail = !(m < tol);
    flags[0] = later && fail;
    if (!later && fail) flags[3] = 1;
  }
}

// finiteDifferencePsiV (CP_State_GSpacePlane.C:3707-3770), first part: keep
// psi_o(t) before psi_o(t+dt) overwrites it (only when this step resets).
__global__ void k_psiv_save(const int* __restrict__ flags, const double2* __restrict__ psi,
                            double2* __restrict__ save, size_t n) {
  if (!flags[0]) return;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    save[i] = psi[i];
}

// second part: psi_no <- psi_o(t+dt), v = (psi_o(t+dt) - psi_o(t)) / dt
// (norb_fin_diff_order 0), orthoT <- I (ortho.C:545-562); the next
// integrate runs without the second half kick (flags[1]).
__global__ void k_psiv_apply(int* __restrict__ flags, const double2* __restrict__ psi,
                             const double2* __restrict__ save, double2* __restrict__ psi_no,
                             double2* __restrict__ v, double* __restrict__ T, int nst, size_t n,
                             double rdt) {
  const int f = flags[0];
  if (f) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const double2 a = psi[i], b = save[i];
      v[i] = make_double2((a.x - b.x) * rdt, (a.y - b.y) * rdt);
      psi_no[i] = a;
    }
    const size_t nt = (size_t)nst * nst;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += stride)
      T[i] = (i % nst) == (i / nst) ? 1.0 : 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    flags[1] = f;
    flags[2] += f;
  }
}

// identity into T (n x n) and the reset flags cleared: the state before the
// first step of the reference form
__global__ void k_dyn_start(double* __restrict__ T, int n, int* __restrict__ flags,
                            double* __restrict__ dev) {
  const size_t nt = (size_t)n * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nt;
       i += (size_t)gridDim.x * blockDim.x)
    T[i] = (i % n) == (i / n) ? 1.0 : 0.0;
  if (blockIdx.x == 0 && threadIdx.x < 4) flags[threadIdx.x] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *dev = 0.0;
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
  cudaFree(c->d_force); cudaFree(c->d_psi_no); cudaFree(c->d_gamma); cudaFree(c->d_dyn_flags);
  cudaFree(c->d_dyn_dev);
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
                   int iteration, double* d_fict_ke, double* d_enhc, const int* d_skip_half) {
  if (!c->d_cmass) {
    cpstep_set_error("integrate: CP masses not set (cpstep_set_cp_mass)");
    return CPSTEP_ERR_STATE;
  }
  double2* p = reinterpret_cast<double2*>(psi);
  double2* v = reinterpret_cast<double2*>(vpsi);
  const double2* f = reinterpret_cast<const double2*>(force);
  int nb = c->nblk_ke;
  if (c->nhc.on) {
    int rc = nhc_integrate(c, force, psi, vpsi, dt, iteration, d_fict_ke, d_enhc, d_skip_half);
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
                                              d_skip_half, c->d_step_part);
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
  const int K = 2 * c->npts;
  const int mixed = c->precision == CPSTEP_PREC_MIXED;
  if (c->dyn_form == CPSTEP_CONSTRAINT_LOWDIN) {
    // 3. lambda_ji = sum_p Re(conj psi_j F_i); F <- F - (wpt/2) psi.lambda
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
    if ((rc = ortho_tmat(c, c->d_smat, c->d_tmat, S, mixed, 0, mixed ? 2e-6 : 1e-15,
                         mixed ? 20 : 10, nullptr, nullptr, ortho_check)))
      return rc;
    if ((rc = pc_backmul_launch(c, c->d_tmat, S, psi, K, c->d_psi_tmp, K, S, S, K, 1.0, 0.0))) return rc;
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(psi, c->d_psi_tmp, sizeof(double2) * ncoef,
                                    cudaMemcpyDeviceToDevice, c->stream));
  } else {
    // the reference's dynamics: psi_no and orthoT (d_tmat) carry over
    if ((rc = ensure_buf(&c->d_psi_no, sizeof(double2) * ncoef)) ||
        (rc = ensure_buf(&c->d_gamma, sizeof(double) * S * S)) ||
        (rc = ensure_buf(&c->d_dyn_dev, sizeof(double))))
      return rc;
    if (!c->d_dyn_flags) CPSTEP_CUDA_TRY(cudaMalloc(&c->d_dyn_flags, 4 * sizeof(int)));
    if (iteration == 1 && !c->dyn_loaded) {
      // iteration 0 of the reference orthonormalised the input: psi_no = psi, orthoT = I
      CPSTEP_CUDA_TRY(cudaMemcpyAsync(c->d_psi_no, psi, sizeof(double2) * ncoef,
                                      cudaMemcpyDeviceToDevice, c->stream));
      stp::k_dyn_start<<<cdiv(S * S, 256), 256, 0, c->stream>>>(c->d_tmat, S, c->d_dyn_flags,
                                                                 c->d_dyn_dev);
      CPSTEP_LAUNCH_CHECK();
      c->dyn_init = 1;
    } else if (!c->dyn_init) {
      cpstep_set_error("cp_step: iteration %d of the orthoT form needs iteration 1 or a state "
                       "loaded by cpstep_dyn_state", iteration);
      return CPSTEP_ERR_STATE;
    }
    c->dyn_loaded = 0;
    // 3. lambda = <psi_o|F>, gamma = orthoT lambda, F_c = F.orthoT - W psi_o.gamma
    if ((rc = pc_overlap_launch(c, psi, c->d_force, S, S, K, nullptr, 1.0, 0.0, c->d_lambda, S))) return rc;
    if ((rc = dgemm_launch(c->stream, 0, 0, S, S, S, 1.0, c->d_tmat, S, c->d_lambda, S, 0.0,
                           c->d_gamma, S)))
      return rc;
    if ((rc = pc_backmul_launch(c, c->d_tmat, S, c->d_force, K, c->d_psi_tmp, K, S, S, K, 1.0,
                                0.0)))
      return rc;
    if ((rc = pc_backmul_w_launch(c, c->d_gamma, S, psi, K, c->d_psi_tmp, K, S, S, K, -0.5, 1.0,
                                  c->d_wpt)))
      return rc;
    mark(5);
    // 4. Verlet update of the non-orthogonal coefficients (no second half kick
    // after a reset: flags[1])
    if ((rc = step_integrate(c, c->d_psi_tmp, c->d_psi_no, vpsi, dt, iteration,
                             energies + CPSTEP_E_FICT, energies + CPSTEP_E_NHC_KE,
                             c->d_dyn_flags + 1)))
      return rc;
    mark(6);
    // 5. S = overlap(psi_no), the norb check, T = (S/2)^(-1/2), psi_o = psi_no.T
    // written straight into psi; the PsiV reset on a failed check
    if ((rc = pc_overlap_launch(c, c->d_psi_no, c->d_psi_no, S, S, K, c->d_wpt, 1.0, 0.0,
                                c->d_smat, S)))
      return rc;
    stp::k_norb_check<<<1, 1024, 0, c->stream>>>(c->d_smat, S, c->tol_norb, iteration > 1,
                                                 c->d_dyn_flags, c->d_dyn_dev);
    CPSTEP_LAUNCH_CHECK();
    if ((rc = ortho_tmat(c, c->d_smat, c->d_tmat, S, mixed, 0, mixed ? 2e-6 : 1e-15,
                         mixed ? 20 : 10, nullptr, nullptr, ortho_check)))
      return rc;
    const int nb = c->nblk_ke;
    bool fused = false;
    if ((rc = pc_backmul_psiv_tc_launch(c, c->d_tmat, S, c->d_psi_no, psi, K, S, c->d_dyn_flags,
                                        vpsi, 1.0 / dt, &fused)))
      return rc;
    if (!fused) {
      stp::k_psiv_save<<<nb, 256, 0, c->stream>>>(c->d_dyn_flags,
                                                   reinterpret_cast<const double2*>(psi),
                                                   reinterpret_cast<double2*>(c->d_force), ncoef);
      CPSTEP_LAUNCH_CHECK();
      if ((rc = pc_backmul_launch(c, c->d_tmat, S, c->d_psi_no, K, psi, K, S, S, K, 1.0, 0.0)))
        return rc;
    }
    // the reset's v and psi_no (unless the back-multiply wrote them), T = I, the flags
    stp::k_psiv_apply<<<fused ? cdiv(S * S, 256) : nb, 256, 0, c->stream>>>(
        c->d_dyn_flags, reinterpret_cast<const double2*>(psi),
        reinterpret_cast<const double2*>(c->d_force), reinterpret_cast<double2*>(c->d_psi_no),
        reinterpret_cast<double2*>(vpsi), c->d_tmat, S, fused ? 0 : ncoef, 1.0 / dt);
    CPSTEP_LAUNCH_CHECK();
  }
  mark(7);
  if (c->profile) c->prof_pending += 1;
  return CPSTEP_OK;
}
