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
  ions::k_atoms_nve<<<1, 256, 0, c->stream>>>(pos, vel, fatm, mass, a.natm, dt, itime, ekin);
  CPSTEP_LAUNCH_CHECK();
  return atoms_set_positions_dev(c, pos);
}
