// Atoms between electronic steps: the real-space ion-ion (Ewald) forces and
// the NVE velocity-Verlet step of the ions.
//
//   CPRSPACEION::CP_getionforce  src_piny_physics_v1.0/abinito_physics/cp_ions/
//                                cp_rspace_ion.C:25-250 (iperd = 3, no Grimme term)
//   ATOMINTEGRATE::integrate_nve_2nd_half / _1st_half / computeEkin
//                                classical_physics/integrate/integration_drivers.C:17-88,
//                                :337-355 (the NVE branch of ctrl_atom_integrate,
//                                control_integrate.C:22-200)
//
// The pair sum runs as one block per atom over all partners (each pair seen
// from both ends, so the forces need no atomics and the sums have a fixed
// order); the reference's erfc approximation (9-term polynomial in
// tt = 1/(1 + p alp r) times e^{-(alp r)^2}) is restated with its constants.
#include <cmath>
#include <vector>

#include "ctx.cuh"

namespace ions {

struct Cell {
  double h[9], hi[9];  // 0-based column-major hmat, hmati
  double hmin;         // half the shortest cell vector
};

__constant__ double kE[9] = {0.2041422096422003, 0.1997535956961481, 0.2213176596405576,
                             0.03360430734640255, 0.4732592578721755, -0.509078520069735,
                             0.6772631491947646, -0.369912979092217, 0.06965131976970335};
constexpr double kP = 0.3614;

__device__ __forceinline__ double round_half_away(double x) {
  return x >= 0.0 ? floor(x + 0.5) : ceil(x - 0.5);
}

// q per type (typ[atom])
__global__ void k_ion_rs(const double* __restrict__ pos, const int* __restrict__ typ,
                         const double* __restrict__ q, int natm, Cell cell, double alp,
                         double* __restrict__ f, double* __restrict__ epart) {
  __shared__ double red[32];
  const int i = blockIdx.x;
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2], qi = q[typ[i]];
  double fx = 0.0, fy = 0.0, fz = 0.0, e = 0.0;
  for (int j = threadIdx.x; j < natm; j += blockDim.x) {
    if (j == i) continue;
    double d[3] = {xi - pos[3 * j], yi - pos[3 * j + 1], zi - pos[3 * j + 2]};
    double s[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      s[r] = cell.hi[r] * d[0] + cell.hi[r + 3] * d[1] + cell.hi[r + 6] * d[2];
      s[r] -= round_half_away(s[r]);
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) d[r] = cell.h[r] * s[0] + cell.h[r + 3] * s[1] + cell.h[r + 6] * s[2];
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double r = sqrt(r2);
    if (r > cell.hmin) continue;
    const double qij = qi * q[typ[j]];
    const double x = r * alp;
    const double eee = exp(-x * x);
    const double tt = 1.0 / (1.0 + kP * x);
    double pg = 0.0, pd = 0.0;
#pragma unroll
    for (int k = 8; k >= 0; --k) {
      pg = pg * tt + kE[k];
      pd = pd * tt + (k + 1) * kE[k];
    }
    const double g = pg * tt * eee;
    const double dg = pd * tt * tt * eee * kP * alp + 2.0 * alp * alp * g * r;
    const double dv = (g / r2 + dg / r) * qij / r;
    e += 0.5 * qij * g / r;
    fx += d[0] * dv;
    fy += d[1] * dv;
    fz += d[2] * dv;
  }
  fx = block_sum(fx, red);
  fy = block_sum(fy, red);
  fz = block_sum(fz, red);
  e = block_sum(e, red);
  if (threadIdx.x == 0) {
    f[3 * i] += fx;
    f[3 * i + 1] += fy;
    f[3 * i + 2] += fz;
    epart[i] = e;
  }
}

// energies[EWD_RS] = sum of the pair energies + vself + vbgr (fixed order)
__global__ void k_ion_finish(const double* __restrict__ epart, int natm, double econst,
                             double* __restrict__ energies) {
  __shared__ double red[32];
  double e = 0.0;
  for (int i = threadIdx.x; i < natm; i += blockDim.x) e += epart[i];
  e = block_sum(e, red);
  if (threadIdx.x == 0) energies[CPSTEP_E_EWD_RS] = e + econst;
}

// NVE: v += dt/2 f/m (itime > 0), E_kin part, v += dt/2 f/m, x += dt v
__global__ void k_atoms_nve(double* __restrict__ pos, double* __restrict__ vel,
                            const double* __restrict__ f, const double* __restrict__ mass,
                            int natm, double dt, int itime, double* __restrict__ ekin) {
  __shared__ double red[32];
  double e = 0.0;
  for (int i = threadIdx.x; i < natm; i += blockDim.x) {
    const double m = mass[i], h = 0.5 * dt / m;
    double v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      v[d] = vel[3 * i + d];
      if (itime > 0) v[d] += h * f[3 * i + d];
      e += m * v[d] * v[d];
      v[d] += h * f[3 * i + d];
      vel[3 * i + d] = v[d];
      pos[3 * i + d] += dt * v[d];
    }
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0 && ekin) *ekin = 0.5 * e;
}

// NVT with massive Nose-Hoover chains (integrate_nvt_2nd_half / _1st_half,
// applyNHC, computeENHC: integration_drivers.C:89-190, :358-565): every
// Cartesian component of every atom has its own chain of length L; one thread
// per atom (the three components in lockstep, so the chain positions add up
// in the reference's order).
constexpr int kMaxLen = 5;

struct NvtPar {
  int len, nres, nyosh;
  double w[9];  // Yoshida weights times dt / nres
};

__device__ void apply_nhc(double* v, double m, double kT, const double* mn, double (*vn)[kMaxLen],
                          double& pkt, const NvtPar& P) {
  const int L = P.len;
  double f[3][kMaxLen], mv2[3];
  for (int d = 0; d < 3; ++d) {
    mv2[d] = m * v[d] * v[d];
    f[d][0] = (mv2[d] - kT) / mn[0];
    for (int ic = 1; ic < L; ++ic) f[d][ic] = (mn[ic - 1] * vn[d][ic - 1] * vn[d][ic - 1] - kT) / mn[ic];
  }
  for (int ir = 0; ir < P.nres; ++ir) {
    for (int iy = 0; iy < P.nyosh; ++iy) {
      const double w2 = P.w[iy] * 0.5, w4 = P.w[iy] * 0.25, w8 = P.w[iy] * 0.125;
      for (int d = 0; d < 3; ++d) {
        vn[d][L - 1] += f[d][L - 1] * w4;
        for (int ic = L - 2; ic >= 0; --ic) {
          const double aa = exp(-w8 * vn[d][ic + 1]);
          vn[d][ic] = vn[d][ic] * aa * aa + w4 * f[d][ic] * aa;
        }
        const double aa = exp(-w2 * vn[d][0]);
        v[d] *= aa;
        mv2[d] *= aa * aa;
      }
      const double pre = kT * w2;
      for (int ic = 0; ic < L; ++ic) pkt += pre * (vn[0][ic] + vn[1][ic] + vn[2][ic]);
      for (int d = 0; d < 3; ++d) {
        f[d][0] = (mv2[d] - kT) / mn[0];
        for (int ic = 0; ic < L - 1; ++ic) {
          const double aa = exp(-w8 * vn[d][ic + 1]);
          vn[d][ic] = vn[d][ic] * aa * aa + w4 * f[d][ic] * aa;
          f[d][ic + 1] = (mn[ic] * vn[d][ic] * vn[d][ic] - kT) / mn[ic + 1];
        }
        vn[d][L - 1] += f[d][L - 1] * w4;
      }
    }
  }
}

// ekin[0] = E_kin; enhc = {E_kin NHC, pot NHC} at the time of computeENHC
__global__ void k_atoms_nvt(double* __restrict__ pos, double* __restrict__ vel,
                            const double* __restrict__ f, const double* __restrict__ mass,
                            const double* __restrict__ kTa, const double* __restrict__ mnhc,
                            double* __restrict__ vnhc, double* __restrict__ pkta, int natm,
                            double dt, int itime, NvtPar P, double* __restrict__ ekin,
                            double* __restrict__ enhc) {
  __shared__ double red[32];
  double e = 0.0, en = 0.0, ep = 0.0;
  const int L = P.len;
  for (int i = threadIdx.x; i < natm; i += blockDim.x) {
    const double m = mass[i], h = 0.5 * dt / m, kT = kTa[i];
    const double* mn = mnhc + (size_t)i * L;
    double v[3], vn[3][kMaxLen], pkt = pkta[i];
    for (int d = 0; d < 3; ++d) {
      v[d] = vel[3 * i + d];
      for (int ic = 0; ic < L; ++ic) vn[d][ic] = vnhc[((size_t)i * 3 + d) * L + ic];
    }
    if (itime > 0) {
      for (int d = 0; d < 3; ++d) v[d] += h * f[3 * i + d];
      apply_nhc(v, m, kT, mn, vn, pkt, P);
    }
    e += m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int ic = 0; ic < L; ++ic)
      en += mn[ic] * (vn[0][ic] * vn[0][ic] + vn[1][ic] * vn[1][ic] + vn[2][ic] * vn[2][ic]);
    ep += pkt;
    apply_nhc(v, m, kT, mn, vn, pkt, P);
    for (int d = 0; d < 3; ++d) {
      v[d] += h * f[3 * i + d];
      vel[3 * i + d] = v[d];
      pos[3 * i + d] += dt * v[d];
      for (int ic = 0; ic < L; ++ic) vnhc[((size_t)i * 3 + d) * L + ic] = vn[d][ic];
    }
    pkta[i] = pkt;
  }
  e = block_sum(e, red);
  en = block_sum(en, red);
  ep = block_sum(ep, red);
  if (threadIdx.x == 0) {
    if (ekin) *ekin = 0.5 * e;
    enhc[0] = 0.5 * en;
    enhc[1] = ep;
  }
}

}  // namespace ions

namespace {
// hmat from hmati (3 x 3 inverse, column-major)
void invert3(const double* a, double* b) {
  auto A = [&](int r, int c) { return a[r + 3 * c]; };
  const double det = A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) -
                     A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
                     A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const int r1 = (c + 1) % 3, r2 = (c + 2) % 3, c1 = (r + 1) % 3, c2 = (r + 2) % 3;
      b[r + 3 * c] = (A(r1, c1) * A(r2, c2) - A(r1, c2) * A(r2, c1)) / det;
    }
}
}  // namespace

int ion_forces(cpstep_ctx* c, double* fatm, double* energies) {
  AtomData& a = c->atoms;
  if (a.natm <= 0 || !a.pos) {
    cpstep_set_error("ion_forces: no atoms set");
    return CPSTEP_ERR_STATE;
  }
  if (!c->d_ion_e) CPSTEP_CUDA_TRY(cudaMalloc(&c->d_ion_e, sizeof(double) * a.natm));
  ions::Cell cell;
  for (int k = 0; k < 9; ++k) cell.hi[k] = c->hmati[k];
  invert3(cell.hi, cell.h);
  double lmin = 1e300;
  for (int col = 0; col < 3; ++col)
    lmin = std::min(lmin, std::sqrt(cell.h[3 * col] * cell.h[3 * col] +
                                    cell.h[3 * col + 1] * cell.h[3 * col + 1] +
                                    cell.h[3 * col + 2] * cell.h[3 * col + 2]));
  cell.hmin = 0.5 * lmin;
  ions::k_ion_rs<<<a.natm, 128, 0, c->stream>>>(a.pos, a.typ, a.q, a.natm, cell, a.alp_ewd,
                                                fatm, c->d_ion_e);
  CPSTEP_LAUNCH_CHECK();
  // vself and vbgr from the host copies of the charges (cp_rspace_ion.C:198-213);
  // the Ewald cut-off is the density sphere's, |G|^2 / 2 <= 4 Ecut
  double qsum = 0.0, q2sum = 0.0;
  for (double qq : a.h_q) {
    qsum += qq;
    q2sum += qq * qq;
  }
  const double alp = a.alp_ewd, ecut = 4.0 * 0.5 * c->ecut_ry;
  const double x = std::sqrt(2.0 * ecut) / (2.0 * alp);
  const double tt = 1.0 / (1.0 + 0.3614 * x);
  const double E[9] = {0.2041422096422003, 0.1997535956961481, 0.2213176596405576,
                       0.03360430734640255, 0.4732592578721755, -0.509078520069735,
                       0.6772631491947646, -0.369912979092217, 0.06965131976970335};
  double pg = 0.0;
  for (int k = 8; k >= 0; --k) pg = pg * tt + E[k];
  const double self_erf = 1.0 - pg * tt * std::exp(-x * x);
  const double vself = -(q2sum * alp) / std::sqrt(M_PI) * self_erf;
  const double vbgr = -(0.5 * qsum * qsum * M_PI) / (alp * alp * c->vol);
  ions::k_ion_finish<<<1, 256, 0, c->stream>>>(c->d_ion_e, a.natm, vself + vbgr, energies);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

int atoms_integrate(cpstep_ctx* c, int itime, double* pos, double* vel, const double* fatm,
                    const double* mass, double dt, double* ekin) {
  AtomData& a = c->atoms;
  if (a.natm <= 0) {
    cpstep_set_error("atoms_integrate: no atoms set");
    return CPSTEP_ERR_STATE;
  }
  AtomNvt& t = c->atom_nvt;
  if (t.len > 0 && t.natm != a.natm) {
    cpstep_set_error("atoms_integrate: atom thermostat set for %d atoms, %d now", t.natm, a.natm);
    return CPSTEP_ERR_STATE;
  }
  if (t.len > 0) {
    ions::NvtPar P;
    P.len = t.len; P.nres = t.nres; P.nyosh = t.nyosh;
    double w[9] = {0};
    nhc_yosh(t.nyosh, w);
    for (int k = 0; k < 9; ++k) P.w[k] = w[k] * (dt / t.nres);
    ions::k_atoms_nvt<<<1, 256, 0, c->stream>>>(pos, vel, fatm, mass, t.d_kT, t.d_mnhc, t.d_vn,
                                                t.d_pkt, a.natm, dt, itime, P, ekin, t.d_e);
  } else {
    ions::k_atoms_nve<<<1, 256, 0, c->stream>>>(pos, vel, fatm, mass, a.natm, dt, itime, ekin);
  }
  CPSTEP_LAUNCH_CHECK();
  return atoms_set_positions_dev(c, pos);
}

void atom_nvt_free(cpstep_ctx* c) {
  AtomNvt& t = c->atom_nvt;
  cudaFree(t.d_kT); cudaFree(t.d_mnhc); cudaFree(t.d_vn); cudaFree(t.d_pkt); cudaFree(t.d_e);
  t = AtomNvt();
}

int atom_nvt_set(cpstep_ctx* c, int len, int nres, int nyosh, const double* h_kT,
                 const double* h_mnhc) {
  atom_nvt_free(c);
  if (len <= 0) return CPSTEP_OK;  // NVE
  const int n = c->atoms.natm;
  if (n <= 0) {
    cpstep_set_error("set_atom_thermostat: no atoms set");
    return CPSTEP_ERR_STATE;
  }
  if (len > ions::kMaxLen || nres < 1 || !h_kT || !h_mnhc ||
      !(nyosh == 1 || nyosh == 3 || nyosh == 5 || nyosh == 7 || nyosh == 9)) {
    cpstep_set_error("set_atom_thermostat: len_nhc in 1..%d, nres >= 1, nyosh in {1,3,5,7,9}",
                     ions::kMaxLen);
    return CPSTEP_ERR_ARG;
  }
  AtomNvt& t = c->atom_nvt;
  // t.len is published last: a failed allocation or copy leaves the NVE branch
  // selected (the buffers made so far are released by the next atom_nvt_free)
  t.nres = nres; t.nyosh = nyosh; t.natm = n;
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_kT, sizeof(double) * n));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_mnhc, sizeof(double) * n * len));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_vn, sizeof(double) * n * 3 * len));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_pkt, sizeof(double) * n));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_e, sizeof(double) * 2));
  CPSTEP_CUDA_TRY(cudaMemcpy(t.d_kT, h_kT, sizeof(double) * n, cudaMemcpyHostToDevice));
  CPSTEP_CUDA_TRY(cudaMemcpy(t.d_mnhc, h_mnhc, sizeof(double) * n * len, cudaMemcpyHostToDevice));
  CPSTEP_CUDA_TRY(cudaMemset(t.d_vn, 0, sizeof(double) * n * 3 * len));
  CPSTEP_CUDA_TRY(cudaMemset(t.d_pkt, 0, sizeof(double) * n));
  CPSTEP_CUDA_TRY(cudaMemset(t.d_e, 0, sizeof(double) * 2));
  t.len = len;
  return CPSTEP_OK;
}

int atom_nvt_state(cpstep_ctx* c, int set, double* h_vn, double* h_pkt, double* h_e2) {
  AtomNvt& t = c->atom_nvt;
  if (t.len <= 0) {
    cpstep_set_error("atom_thermostat_state: the atom thermostat is off");
    return CPSTEP_ERR_STATE;
  }
  const int n = t.natm;
  const size_t bv = sizeof(double) * n * 3 * t.len, bp = sizeof(double) * n;
  auto dir = set ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  if (h_vn) CPSTEP_CUDA_TRY(cudaMemcpyAsync(set ? (void*)t.d_vn : (void*)h_vn,
                                            set ? (const void*)h_vn : (const void*)t.d_vn, bv,
                                            dir, c->stream));
  if (h_pkt) CPSTEP_CUDA_TRY(cudaMemcpyAsync(set ? (void*)t.d_pkt : (void*)h_pkt,
                                             set ? (const void*)h_pkt : (const void*)t.d_pkt, bp,
                                             dir, c->stream));
  if (h_e2 && !set)
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(h_e2, t.d_e, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
  CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CPSTEP_OK;
}
