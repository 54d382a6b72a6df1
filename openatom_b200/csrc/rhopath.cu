// Density side of the step: PZ-LDA or BLYP exchange-correlation, the density
// FFT on the density sphere, Hartree + local pseudopotential + reciprocal
// Ewald in G space with the atom forces, and V_KS(r).
//
//   CPXCFNCTS::CP_exc_calc       src_piny_physics_v1.0/abinito_physics/cp_xc_fnctl/cp_pz_lda.C:23-170
//   BLYP gradient correction     CP_getGGAFunctional (cp_xc_fnctl/cp_grad_rho_ctrl.C:32-193),
//                                becke_gcx_lda / lyp_gcc (cp_becke.C:20-173); gradients and
//                                White-Bird term CP_Rho_GSpacePlane::divRhoVksGspace /
//                                acceptWhiteByrd (CP_Rho_GSpacePlane.C:278-400),
//                                CP_Rho_RealSpacePlane::whiteByrdFFT / acceptWhiteByrd
//                                (CP_Rho_RealSpacePlane.C:1237-1340)
//   CPLOCAL::CP_hart_eext_calc   src_piny_physics_v1.0/abinito_physics/cp_local/cp_hart_ext.C:56-405
//   CP_get_vpsnow (spline)       cp_hart_ext.C:433-475
//   density FFTs                 CP_Rho_RealSpacePlane::fftRhoRtoRhoG (cp_density_ctrl/
//                                CP_Rho_RealSpacePlane.C:831-864), CP_Rho_GHartExt::FFTVks
//                                (CP_Rho_GHartExt.C:532-540), acceptHartVks (:1365-1415)
//
// The density sphere (|G|^2/2 <= 4 Ecut) is held in the same packed line
// layout as the states, so the state FFT kernels (FP64) transform it.  Those
// compute sum_r f e^{+iG.r} and sum_G c e^{-iG.r}; the reference's rho(G) uses
// e^{-iG.r} and V(r) = sum vks(G) e^{+iG.r}, so the kernels below read conj of
// the transformed density and store conj of vks: the arithmetic on rho(G),
// vks(G), the energies and forces is the reference's.
#include <algorithm>
#include <cmath>
#include <vector>
#include "ctx.cuh"

int cpstep_density_layout(double box_len, double ecut_ry, int nfft, std::vector<int>& kx,
                          std::vector<int>& ky, std::vector<int>& kz, std::vector<int>& runs);

namespace rho {

// PZ-LDA constants (cp_pz_lda.C:47-53)
__constant__ double kPZ[7] = {-0.14230, 1.05290, 0.33340, 0.03110, -0.0480, 0.00200, -0.01160};

// corr = 0 drops the PZ correlation (cp_lyp = 1: BLYP's LDA part is Slater
// exchange only, cp_pz_lda.C:62-63)
__global__ void k_xc(const double* __restrict__ rho, double* __restrict__ vxc, size_t n,
                     double corr, double* __restrict__ part) {
  __shared__ double red[32];
  const double gamma = kPZ[0], beta1 = kPZ[1], beta2 = kPZ[2], au = kPZ[3], bu = kPZ[4],
               cu = kPZ[5], du = kPZ[6];
  const double rat1 = (7.0 / 6.0) * beta1, rat2 = (4.0 / 3.0) * beta2, third = 1.0 / 3.0;
  double ex = 0.0, ec = 0.0, mu = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double r = rho[i];
    double v = 0.0;
    if (r > 0.0) {
      double rs = cbrt(3.0 / (4.0 * M_PI * r));
      double sq = sqrt(rs);
      double xfact = -cbrt(3.0 * r / M_PI);
      double cfact, mufact;
      if (rs >= 1.0) {
        double cf1 = 1.0 + beta1 * sq + beta2 * rs;
        double cf2 = 1.0 + rat1 * sq + rat2 * rs;
        cfact = gamma / cf1;
        mufact = cfact * (cf2 / cf1);
      } else {
        double lnrs = log(rs);
        cfact = au * lnrs + bu + cu * rs * lnrs + du * rs;
        mufact = au * lnrs + (bu - third * au) + 2.0 * third * cu * rs * lnrs +
                 third * (2.0 * du - cu) * rs;
      }
      cfact *= corr;
      mufact *= corr;
      ex += xfact * r;
      ec += cfact * r;
      v = xfact + mufact;
      mu += v * r;
    }
    vxc[i] = v;
  }
  double a = block_sum(0.75 * ex + ec, red);
  double b = block_sum(mu, red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

struct Atoms {
  int natm, ntyp;
  const int* typ;      // [natm]
  const double* frac;  // [natm][3] fractional coordinates (hmati R)
  const double* q;     // [ntyp]
  const double* vps;   // [ntyp][4][nspl]
  const double* gzvps; // [ntyp]
  int nspl;
  double gmin, dg;
  int kxm, kym, kzm;   // phase-table extents
  const double2* ex;   // [kxm+1][natm]      e^{i 2pi kx s_x}
  const double2* ey;   // [2kym+1][natm]     ky in [-kym, kym]
  const double2* ez;   // [2kzm+1][natm]
  const double2* ezt;  // [natm][2kzm+1], atoms in type order
  const int* rank;     // atom -> type-ordered position
  int tstart[CPSTEP_MAX_TYPES + 1];
};

__global__ void k_phase(const double* __restrict__ frac, int natm, int kxm, int kym, int kzm,
                        const int* __restrict__ rank, double2* __restrict__ ex,
                        double2* __restrict__ ey, double2* __restrict__ ez,
                        double2* __restrict__ ezt) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natm) return;
  const double tpi = 2.0 * M_PI;
  for (int k = 0; k <= kxm; ++k) {
    double s, c;
    sincos(tpi * k * frac[3 * a], &s, &c);
    ex[(size_t)k * natm + a] = make_double2(c, s);
  }
  for (int k = -kym; k <= kym; ++k) {
    double s, c;
    sincos(tpi * k * frac[3 * a + 1], &s, &c);
    ey[(size_t)(k + kym) * natm + a] = make_double2(c, s);
  }
  double2* zt = ezt + (size_t)rank[a] * (2 * kzm + 1);
  for (int k = -kzm; k <= kzm; ++k) {
    double s, c;
    sincos(tpi * k * frac[3 * a + 2], &s, &c);
    ez[(size_t)(k + kzm) * natm + a] = make_double2(c, s);
    zt[k + kzm] = make_double2(c, s);
  }
}

// fractional coordinates s = hmati R from Cartesian positions
__global__ void k_frac(const double* __restrict__ pos, const double* __restrict__ hmati, int natm,
                       double* __restrict__ frac) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natm) return;
  const double* R = pos + 3 * a;
  for (int d = 0; d < 3; ++d)
    frac[3 * a + d] = hmati[d] * R[0] + hmati[d + 3] * R[1] + hmati[d + 6] * R[2];
}

__device__ __forceinline__ double2 phase(const Atoms& A, int a, int kx, int ky, int kz) {
  double2 x = A.ex[(size_t)kx * A.natm + a];
  double2 y = A.ey[(size_t)(ky + A.kym) * A.natm + a];
  double2 z = A.ez[(size_t)(kz + A.kzm) * A.natm + a];
  double2 xy = make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
  return make_double2(xy.x * z.x - xy.y * z.y, xy.x * z.y + xy.y * z.x);
}

// spline value / vol of type t at g (CP_get_vpsnow, cp_hart_ext.C:459-471)
__device__ __forceinline__ double vps_at(const Atoms& A, int t, double g, double rvol) {
  int iii = (int)((g - A.gmin) / A.dg + 1.0);
  iii = min(iii, A.nspl);
  iii = max(iii, 1);
  double h = g - ((double)(iii - 1) * A.dg + A.gmin);
  const double* v = A.vps + (size_t)t * 4 * A.nspl + (iii - 1);
  return (((v[3 * A.nspl] * h + v[2 * A.nspl]) * h + v[A.nspl]) * h + v[0]) * rvol;
}

// Structure factors along z-lines.  The density sphere is packed line by line
// (all kz of one (kx, ky) contiguous), and e^{iG.R} = [e^{i2pi kx sx} e^{i2pi ky sy}]
// e^{i2pi kz sz}: the bracket is formed once per line and atom (in shared
// memory, type order) and each point of the line multiplies it by the atom's
// z phase.  The reference advances the structure factor along kz the same way
// (ei_inc recursion, cp_hart_ext.C:150-210); the tables keep every phase exact.
//
// One block per line, one thread per point (lines longer than the block loop).
// rhog_t: transformed density (sum rho e^{+iGr} vol/N = conj of the reference
// rho(G)); writes conj(vks) for the G->R kernels, the per-point force terms
// and per-line energy partials [nlines][3].
constexpr int HT = 128;
constexpr int kMaxAtoms = 1024;  // the force pass holds at most 4 atoms per thread of 256
__global__ void __launch_bounds__(HT)
k_hart_lines(const double2* __restrict__ rhog_t, const int* __restrict__ line_off, int nlines,
             const int* __restrict__ kx, const int* __restrict__ ky, const int* __restrict__ kz,
             int npts, const double* __restrict__ hmati, double vol, double ecut4, double alp,
             Atoms A, double2* __restrict__ vg_t, double4* __restrict__ fterm,
             double* __restrict__ part) {
  extern __shared__ double2 su[];  // [natm] line phases, type order
  __shared__ double red[32];
  const double tpi = 2.0 * M_PI, rvol = 1.0 / vol, fpi = 4.0 * M_PI;
  const double falp2 = 4.0 * alp * alp;
  const int l = blockIdx.x;
  const int off = line_off[l], end = (l + 1 < nlines) ? line_off[l + 1] : npts;
  const int a = kx[off], b = ky[off];
  const int nz = 2 * A.kzm + 1;
  for (int i = threadIdx.x; i < A.natm; i += HT) {
    double2 x = A.ex[(size_t)a * A.natm + i];
    double2 y = A.ey[(size_t)(b + A.kym) * A.natm + i];
    su[A.rank[i]] = make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
  }
  __syncthreads();
  double eh = 0.0, ee = 0.0, ew = 0.0;
  const double gx0 = tpi * (a * hmati[0] + b * hmati[1]);
  const double gy0 = tpi * (a * hmati[3] + b * hmati[4]);
  const double gz0 = tpi * (a * hmati[6] + b * hmati[7]);
  for (int p = off + threadIdx.x; p < end; p += HT) {
    const int c = kz[p];
    double gx = gx0 + tpi * c * hmati[2];
    double gy = gy0 + tpi * c * hmati[5];
    double gz = gz0 + tpi * c * hmati[8];
    double g2 = gx * gx + gy * gy + gz * gz;
    double2 out = make_double2(0.0, 0.0);
    double4 ft = make_double4(0.0, 0.0, 0.0, 0.0);
    if (g2 <= ecut4 && g2 != 0.0) {
      double w = (a == 0) ? 1.0 : 2.0;
      double2 r = rhog_t[p];
      r.y = -r.y;  // reference rho(G)
      double hart = fpi / (g2 * vol);
      eh += 0.5 * hart * (r.x * r.x + r.y * r.y) * w;
      double g = sqrt(g2);
      double2 vext = make_double2(0.0, 0.0), sewd = make_double2(0.0, 0.0);
      const double2* zc = A.ezt + (c + A.kzm);
      for (int t = 0; t < A.ntyp; ++t) {
        double2 st = make_double2(0.0, 0.0);
#pragma unroll 4
        for (int i = A.tstart[t]; i < A.tstart[t + 1]; ++i) {
          double2 u = su[i];
          double2 z = zc[(size_t)i * nz];
          st.x += u.x * z.x - u.y * z.y;
          st.y += u.x * z.y + u.y * z.x;
        }
        double vt = vps_at(A, t, g, rvol);
        double qt = A.q[t];
        vext.x += vt * st.x;
        vext.y += vt * st.y;
        sewd.x += qt * st.x;
        sewd.y += qt * st.y;
      }
      double ewdf = fpi * exp(-g2 / falp2) / (g2 * vol);
      ew += 0.5 * ewdf * (sewd.x * sewd.x + sewd.y * sewd.y) * w;
      ee += (r.x * vext.x - r.y * vext.y) * w;
      // vks = rho*hart + conj(vext); store conj(vks)
      out = make_double2(r.x * hart + vext.x, -(r.y * hart - vext.y));
      ft = make_double4(r.x * w, -r.y * w, sewd.x * ewdf * w, sewd.y * ewdf * w);
    }
    vg_t[p] = out;
    fterm[p] = ft;
  }
  double s1 = block_sum(eh, red);
  double s2 = block_sum(ee, red);
  double s3 = block_sum(ew, red);
  if (threadIdx.x == 0) {
    part[3 * l] = s1;
    part[3 * l + 1] = s2;
    part[3 * l + 2] = s3;
  }
}

// The same pass with the z phase advanced along the line instead of read per
// point (the reference's ei_inc recursion, cp_hart_ext.C:150-210): needs the
// points of every line at consecutive kz.  A group of HG lanes owns a line;
// lane j owns points HPL j .. HPL j + HPL - 1 of each HG HPL-point segment.
// Per atom (type order) a lane reads the phase at its first kz and
// e^{i2pi sz}, then multiplies along its points; the loads of four atoms are
// issued together.  Each lane's per-type sums are in registers; the energy
// partials of the line are summed over its group.
constexpr int HG = 32, HPL = 4, HWARPS = 4, HBATCH = 4;
__global__ void __launch_bounds__(32 * HWARPS)
k_hart_lines_rec(const double2* __restrict__ rhog_t, const int* __restrict__ line_off,
                 int nlines, const int* __restrict__ kx, const int* __restrict__ ky,
                 const int* __restrict__ kz, int npts, const double* __restrict__ hmati,
                 double vol, double ecut4, double alp, Atoms A, double2* __restrict__ vg_t,
                 double4* __restrict__ fterm, double* __restrict__ part) {
  extern __shared__ double2 su_all[];  // [groups][natm] line phases, type order
  const double tpi = 2.0 * M_PI, rvol = 1.0 / vol, fpi = 4.0 * M_PI;
  const double falp2 = 4.0 * alp * alp;
  const int lane = threadIdx.x & 31, grp = threadIdx.x / HG, j = lane & (HG - 1);
  const int ngrp = (32 / HG) * HWARPS;
  double2* su = su_all + (size_t)grp * A.natm;
  const int nz = 2 * A.kzm + 1;
  // every group walks lines l = blockIdx.x * ngrp + grp, + gridDim.x * ngrp, ...;
  // the trip count is the same for the two groups of a warp (their shuffles)
  for (int lb = blockIdx.x * ngrp; lb < nlines; lb += gridDim.x * ngrp) {
    const int l = lb + grp;
    const bool live = l < nlines;
    const int off = live ? line_off[l] : 0;
    const int end = live ? ((l + 1 < nlines) ? line_off[l + 1] : npts) : 0;
    const int a = live ? kx[off] : 0, b = live ? ky[off] : 0;
    __syncwarp();
    if (live)
      for (int i = j; i < A.natm; i += HG) {
        const int at = i;  // atom index; its phase goes to its type-ordered slot
        double2 x = A.ex[(size_t)a * A.natm + at];
        double2 y = A.ey[(size_t)(b + A.kym) * A.natm + at];
        su[A.rank[at]] = make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
      }
    __syncwarp();
    double eh = 0.0, ee = 0.0, ew = 0.0;
    const double gx0 = tpi * (a * hmati[0] + b * hmati[1]);
    const double gy0 = tpi * (a * hmati[3] + b * hmati[4]);
    const double gz0 = tpi * (a * hmati[6] + b * hmati[7]);
    for (int s0 = off; s0 < end; s0 += HG * HPL) {
      const int p0 = s0 + HPL * j;            // this lane's first point
      const int np = max(0, min(HPL, end - p0));
      const int c0 = np > 0 ? kz[p0] : 0;
      double2 vext[HPL], sewd[HPL];
#pragma unroll
      for (int k = 0; k < HPL; ++k) vext[k] = sewd[k] = make_double2(0.0, 0.0);
      double g[HPL];
#pragma unroll
      for (int k = 0; k < HPL; ++k) {
        const int c = c0 + k;
        const double gx = gx0 + tpi * c * hmati[2], gy = gy0 + tpi * c * hmati[5],
                     gz = gz0 + tpi * c * hmati[8];
        g[k] = gx * gx + gy * gy + gz * gz;  // g^2 here, g below
      }
      if (np > 0) {
        for (int t = 0; t < A.ntyp; ++t) {
          double2 st[HPL];
#pragma unroll
          for (int k = 0; k < HPL; ++k) st[k] = make_double2(0.0, 0.0);
          const int ie = A.tstart[t + 1];
          for (int i0 = A.tstart[t]; i0 < ie; i0 += HBATCH) {
            double2 z[HBATCH], inc[HBATCH], u[HBATCH];
#pragma unroll
            for (int q = 0; q < HBATCH; ++q) {
              const bool in = i0 + q < ie;
              const double2* zr = A.ezt + (size_t)(in ? i0 + q : i0) * nz;
              z[q] = in ? zr[c0 + A.kzm] : make_double2(0.0, 0.0);
              inc[q] = zr[1 + A.kzm];
              u[q] = su[in ? i0 + q : i0];
            }
#pragma unroll
            for (int q = 0; q < HBATCH; ++q) {  // atoms in order: the sums keep it
              double2 ph = make_double2(u[q].x * z[q].x - u[q].y * z[q].y,
                                        u[q].x * z[q].y + u[q].y * z[q].x);
#pragma unroll
              for (int k = 0; k < HPL; ++k) {
                st[k].x += ph.x;
                st[k].y += ph.y;
                ph = make_double2(ph.x * inc[q].x - ph.y * inc[q].y,
                                  ph.x * inc[q].y + ph.y * inc[q].x);
              }
            }
          }
          const double qt = A.q[t];
#pragma unroll
          for (int k = 0; k < HPL; ++k) {
            const double vt = (k < np && g[k] != 0.0) ? vps_at(A, t, sqrt(g[k]), rvol) : 0.0;
            vext[k].x += vt * st[k].x;
            vext[k].y += vt * st[k].y;
            sewd[k].x += qt * st[k].x;
            sewd[k].y += qt * st[k].y;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < HPL; ++k) {
        if (k >= np) break;
        const int p = p0 + k;
        const double g2 = g[k];
        double2 out = make_double2(0.0, 0.0);
        double4 ft = make_double4(0.0, 0.0, 0.0, 0.0);
        if (g2 <= ecut4 && g2 != 0.0) {
          const double w = (a == 0) ? 1.0 : 2.0;
          double2 r = rhog_t[p];
          r.y = -r.y;  // reference rho(G)
          const double hart = fpi / (g2 * vol);
          eh += 0.5 * hart * (r.x * r.x + r.y * r.y) * w;
          const double ewdf = fpi * exp(-g2 / falp2) / (g2 * vol);
          ew += 0.5 * ewdf * (sewd[k].x * sewd[k].x + sewd[k].y * sewd[k].y) * w;
          ee += (r.x * vext[k].x - r.y * vext[k].y) * w;
          out = make_double2(r.x * hart + vext[k].x, -(r.y * hart - vext[k].y));
          ft = make_double4(r.x * w, -r.y * w, sewd[k].x * ewdf * w, sewd[k].y * ewdf * w);
        }
        vg_t[p] = out;
        fterm[p] = ft;
      }
    }
#pragma unroll
    for (int o = HG / 2; o > 0; o >>= 1) {
      eh += __shfl_xor_sync(0xffffffffu, eh, o, HG);
      ee += __shfl_xor_sync(0xffffffffu, ee, o, HG);
      ew += __shfl_xor_sync(0xffffffffu, ew, o, HG);
    }
    if (live && j == 0) {
      part[3 * l] = eh;
      part[3 * l + 1] = ee;
      part[3 * l + 2] = ew;
    }
  }
}

// G = 0 (cp_hart_ext.C:345-368); single thread
__global__ void k_hart_g0(const double2* __restrict__ rhog_t, int izero, double vol, Atoms A,
                          double2* __restrict__ vg_t, double* __restrict__ eext) {
  double v = 0.0;
  for (int i = 0; i < A.natm; ++i) v += A.gzvps[A.typ[i]];
  v /= vol;
  vg_t[izero] = make_double2(v, 0.0);
  *eext += v * rhog_t[izero].x;
}

// Local + Ewald forces on the atoms, line by line: for line (kx, ky) and atom
// a with type t, with T_t(G) the per-point term and u_a the line phase,
//   F_a += sum_kz g(G) Im(u_a e^{i2pi kz sz_a} conj T_t(G))
//        = g0 Im(u_a P_a) + (2pi hmati col z) Im(u_a Q_a),
//   P_a = sum_kz e^{i2pi kz sz_a} conj T_t,  Q_a = sum_kz kz e^{i2pi kz sz_a} conj T_t,
// g = g0 + kz (2pi hmati col z) being linear along the line.  A block (one
// thread per atom) walks lines blockIdx.x, +gridDim.x, ...; T_t of the line's
// points is staged in shared memory [ntyp][lmax] with kz beside it.
// Writes fpart[block][natm][3].
template <bool REC>
__global__ void k_local_forces_lines(const double4* __restrict__ fterm,
                                     const int* __restrict__ line_off, int nlines,
                                     const int* __restrict__ kx, const int* __restrict__ ky,
                                     const int* __restrict__ kz, int npts,
                                     const double* __restrict__ hmati, double vol, Atoms A,
                                     int lmax, double* __restrict__ fpart) {
  extern __shared__ double2 sT[];  // [ntyp][lmax] conj T, then int kz[lmax]
  int* skz = reinterpret_cast<int*>(sT + (size_t)A.ntyp * lmax);
  const double tpi = 2.0 * M_PI, rvol = 1.0 / vol;
  const double cx = tpi * hmati[2], cy = tpi * hmati[5], cz = tpi * hmati[8];
  double f[4][3] = {};  // up to 4 atoms per thread
  const int nper = (A.natm + blockDim.x - 1) / blockDim.x;
  for (int l = blockIdx.x; l < nlines; l += gridDim.x) {
    const int off = line_off[l], end = (l + 1 < nlines) ? line_off[l + 1] : npts;
    const int a = kx[off], b = ky[off];
    const double g0x = tpi * (a * hmati[0] + b * hmati[1]);
    const double g0y = tpi * (a * hmati[3] + b * hmati[4]);
    const double g0z = tpi * (a * hmati[6] + b * hmati[7]);
    for (int c0 = off; c0 < end; c0 += lmax) {
      const int len = min(lmax, end - c0);
      __syncthreads();
      for (int i = threadIdx.x; i < len; i += blockDim.x) {
        const int p = c0 + i;
        const int c = kz[p];
        skz[i] = c;
        double4 ft = fterm[p];
        double gx = g0x + c * cx, gy = g0y + c * cy, gz = g0z + c * cz;
        double g = sqrt(gx * gx + gy * gy + gz * gz);
        for (int t = 0; t < A.ntyp; ++t) {
          double vt = (ft.x != 0.0 || ft.y != 0.0) ? vps_at(A, t, g, rvol) : 0.0;
          double qt = A.q[t];
          sT[(size_t)t * lmax + i] = make_double2(ft.x * vt + ft.z * qt, -(ft.y * vt + ft.w * qt));
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int at = threadIdx.x + k * blockDim.x;
        if (k < nper && at < A.natm) {
          const int t = A.typ[at];
          double2 x = A.ex[(size_t)a * A.natm + at];
          double2 y = A.ey[(size_t)(b + A.kym) * A.natm + at];
          double2 u = make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
          const double2* T = sT + (size_t)t * lmax;
          double px = 0.0, py = 0.0, qx = 0.0, qy = 0.0;
          // REC: kz runs up by one along the line, so e^{i2pi kz sz} is
          // advanced by e^{i2pi sz} (the reference's ei_inc recursion)
          double2 e = REC ? A.ez[(size_t)(skz[0] + A.kzm) * A.natm + at] : make_double2(0.0, 0.0);
          const double2 inc = REC ? A.ez[(size_t)(1 + A.kzm) * A.natm + at] : e;
#pragma unroll 4
          for (int i = 0; i < len; ++i) {
            const int c = skz[i];
            if (!REC) e = A.ez[(size_t)(c + A.kzm) * A.natm + at];
            double2 tt = T[i];
            double rx = e.x * tt.x - e.y * tt.y;
            double ry = e.x * tt.y + e.y * tt.x;
            px += rx;
            py += ry;
            qx += c * rx;
            qy += c * ry;
            if (REC) e = make_double2(e.x * inc.x - e.y * inc.y, e.x * inc.y + e.y * inc.x);
          }
          double ip = u.x * py + u.y * px;  // Im(u P)
          double iq = u.x * qy + u.y * qx;  // Im(u Q)
          f[k][0] += g0x * ip + cx * iq;
          f[k][1] += g0y * ip + cy * iq;
          f[k][2] += g0z * ip + cz * iq;
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int at = threadIdx.x + k * blockDim.x;
    if (k < nper && at < A.natm) {
      double* o = fpart + ((size_t)blockIdx.x * A.natm + at) * 3;
      o[0] = f[k][0]; o[1] = f[k][1]; o[2] = f[k][2];
    }
  }
}

// out[c] = scale * sum_r part[r][c]; one block per column, fixed order.
// ---------------------------------------------------------------------------
// The EES form of the pass (cp_eext_ees_opt; CPLOCAL::eesAtmBsplineRgrp,
// eesPackGridRchare, eesHartEextGchare, eesEwaldGchare, eesAtmForceRchare,
// cp_hart_ext.C:641-1470).  The reference spreads each type's atoms onto the
// EES grid with their B-splines, transforms the grid to G, forms
// S_t(G) b(G) and the energies per point, transforms the per-type and Ewald
// terms back and gathers the forces through the B-spline derivatives.  The
// spread grid of one atom is a tensor product of three 1-D stencils, so its
// transform at G is the product of three 1-D sums, and with b(G) separable
// too, S_t(G) b(G) = sum_{a in t} t_x[a](kx) t_y[a](ky) t_z[a](kz): the same
// form as the explicit structure factor with the exact phases replaced by
// the tables of EesLocal.  k_hart_lines runs on those tables unchanged; the
// gather becomes, per atom, sum_G Re(T(G) D_a(G)) with D_a the derivative
// tables' products (k_eloc_forces_lines).  No 3-D grid or transform is formed.

// t_d / dt_d of every (atom, axis, k): the 8 stencil terms of one axis
__global__ void k_eloc_tables(const int* __restrict__ ig, const double* __restrict__ mn,
                              const double* __restrict__ dmn, int natm, int ngrid, int kxm,
                              int kym, int kzm, const double2* __restrict__ bden,
                              const int* __restrict__ rank, double2* __restrict__ tx,
                              double2* __restrict__ ty, double2* __restrict__ tz,
                              double2* __restrict__ dtx, double2* __restrict__ dty,
                              double2* __restrict__ dtz, double2* __restrict__ tzt) {
  const int nx = kxm + 1, ny = 2 * kym + 1, nz = 2 * kzm + 1;
  const int per = nx + ny + nz;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)natm * per) return;
  const int a = (int)(i / per);
  const int r = (int)(i % per);
  int d, k, slot;
  if (r < nx) {
    d = 0; slot = r; k = r;
  } else if (r < nx + ny) {
    d = 1; slot = r - nx; k = slot - kym;
  } else {
    d = 2; slot = r - nx - ny; k = slot - kzm;
  }
  const int* g = ig + ((size_t)a * 3 + d) * kNlInterp;
  const double* m = mn + ((size_t)a * 3 + d) * kNlInterp;
  const double* dm = dmn + ((size_t)a * 3 + d) * kNlInterp;
  double sr = 0.0, si = 0.0, dr = 0.0, di = 0.0;
#pragma unroll
  for (int j = 0; j < kNlInterp; ++j) {
    long long t = ((long long)k * g[j]) % ngrid;
    if (t < 0) t += ngrid;
    double sn, cs;
    sincospi(2.0 * (double)t / (double)ngrid, &sn, &cs);
    sr += m[j] * cs;
    si += m[j] * sn;
    dr += dm[j] * cs;
    di += dm[j] * sn;
  }
  const double2 b = bden[((k % ngrid) + ngrid) % ngrid];
  const double2 tv = make_double2(sr * b.x - si * b.y, sr * b.y + si * b.x);
  const double2 dv = make_double2(dr * b.x - di * b.y, dr * b.y + di * b.x);
  const size_t o = (size_t)slot * natm + a;
  if (d == 0) {
    tx[o] = tv;
    dtx[o] = dv;
  } else if (d == 1) {
    ty[o] = tv;
    dty[o] = dv;
  } else {
    tz[o] = tv;
    dtz[o] = dv;
    tzt[(size_t)rank[a] * nz + slot] = tv;
  }
}

// G = 0 (eesHartEextGchare :1175-1205): vext(0) = sum_a gzvps/vol Re(S b)(0)
__global__ void k_eloc_g0(const double2* __restrict__ rhog_t, int izero, double vol, Atoms A,
                          double2* __restrict__ vg_t, double* __restrict__ eext) {
  double v = 0.0;
  for (int a = 0; a < A.natm; ++a) {
    const double2 x = A.ex[a];
    const double2 y = A.ey[(size_t)A.kym * A.natm + a];
    const double2 z = A.ez[(size_t)A.kzm * A.natm + a];
    const double xyr = x.x * y.x - x.y * y.y, xyi = x.x * y.y + x.y * y.x;
    v += A.gzvps[A.typ[a]] * (xyr * z.x - xyi * z.y);
  }
  v /= vol;
  vg_t[izero] = make_double2(v, 0.0);
  *eext += v * rhog_t[izero].x;
}

// Atom forces of the EES form, line by line as k_local_forces_lines: with T
// the per-point term (local and Ewald, as there) and, for atom a on line
// (kx, ky), u0 = t_x t_y, ux = dt_x t_y, uy = t_x dt_y,
//   F_a = -N sum_kz Re(T(G) [(h_r0 ux + h_r1 uy) t_z(kz) + h_r2 u0 dt_z(kz)])
// per Cartesian row r of hmati: the dMn_x/y/z of eesAtmBsplineRgrp IV
// (dMn grid hmati) summed against the back-transformed terms.
struct ElocD {
  const double2 *dtx, *dty, *dtz;
  double grid;
};
__global__ void k_eloc_forces_lines(const double4* __restrict__ fterm,
                                    const int* __restrict__ line_off, int nlines,
                                    const int* __restrict__ kx, const int* __restrict__ ky,
                                    const int* __restrict__ kz, int npts,
                                    const double* __restrict__ hmati, double vol, Atoms A,
                                    ElocD D, int lmax, double* __restrict__ fpart) {
  extern __shared__ double2 sT[];  // [ntyp][lmax] T, then int kz[lmax]
  int* skz = reinterpret_cast<int*>(sT + (size_t)A.ntyp * lmax);
  const double tpi = 2.0 * M_PI, rvol = 1.0 / vol;
  double f[4][3] = {};
  const int nper = (A.natm + blockDim.x - 1) / blockDim.x;
  for (int l = blockIdx.x; l < nlines; l += gridDim.x) {
    const int off = line_off[l], end = (l + 1 < nlines) ? line_off[l + 1] : npts;
    const int a = kx[off], b = ky[off];
    const double g0x = tpi * (a * hmati[0] + b * hmati[1]);
    const double g0y = tpi * (a * hmati[3] + b * hmati[4]);
    const double g0z = tpi * (a * hmati[6] + b * hmati[7]);
    for (int c0 = off; c0 < end; c0 += lmax) {
      const int len = min(lmax, end - c0);
      __syncthreads();
      for (int i = threadIdx.x; i < len; i += blockDim.x) {
        const int p = c0 + i;
        const int c = kz[p];
        skz[i] = c;
        double4 ft = fterm[p];
        double gx = g0x + c * tpi * hmati[2], gy = g0y + c * tpi * hmati[5];
        double gz = g0z + c * tpi * hmati[8];
        double g = sqrt(gx * gx + gy * gy + gz * gz);
        for (int t = 0; t < A.ntyp; ++t) {
          double vt = (ft.x != 0.0 || ft.y != 0.0) ? vps_at(A, t, g, rvol) : 0.0;
          double qt = A.q[t];
          sT[(size_t)t * lmax + i] = make_double2(ft.x * vt + ft.z * qt, -(ft.y * vt + ft.w * qt));
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int at = threadIdx.x + k * blockDim.x;
        if (k < nper && at < A.natm) {
          const int t = A.typ[at];
          const double2 x = A.ex[(size_t)a * A.natm + at];
          const double2 y = A.ey[(size_t)(b + A.kym) * A.natm + at];
          const double2 dx = D.dtx[(size_t)a * A.natm + at];
          const double2 dy = D.dty[(size_t)(b + A.kym) * A.natm + at];
          const double2 u0 = make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
          const double2 ux = make_double2(dx.x * y.x - dx.y * y.y, dx.x * y.y + dx.y * y.x);
          const double2 uy = make_double2(x.x * dy.x - x.y * dy.y, x.x * dy.y + x.y * dy.x);
          const double2* T = sT + (size_t)t * lmax;
          double px = 0.0, py = 0.0, qx = 0.0, qy = 0.0;
#pragma unroll 4
          for (int i = 0; i < len; ++i) {
            const int cz = skz[i] + A.kzm;
            const double2 z = A.ez[(size_t)cz * A.natm + at];
            const double2 dz = D.dtz[(size_t)cz * A.natm + at];
            const double2 tt = T[i];
            px += tt.x * z.x - tt.y * z.y;
            py += tt.x * z.y + tt.y * z.x;
            qx += tt.x * dz.x - tt.y * dz.y;
            qy += tt.x * dz.y + tt.y * dz.x;
          }
#pragma unroll
          for (int r = 0; r < 3; ++r) {
            const double h0 = hmati[3 * r], h1 = hmati[3 * r + 1], h2 = hmati[3 * r + 2];
            const double wx = h0 * ux.x + h1 * uy.x, wy = h0 * ux.y + h1 * uy.y;
            const double re = (wx * px - wy * py) + h2 * (u0.x * qx - u0.y * qy);
            f[k][r] -= D.grid * re;
          }
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int at = threadIdx.x + k * blockDim.x;
    if (k < nper && at < A.natm) {
      double* o = fpart + ((size_t)blockIdx.x * A.natm + at) * 3;
      o[0] = f[k][0]; o[1] = f[k][1]; o[2] = f[k][2];
    }
  }
}

__global__ void k_sum_cols(const double* __restrict__ part, int nrow, int ncol,
                           double* __restrict__ out, double scale) {
  __shared__ double red[32];
  const int c = blockIdx.x;
  double s = 0.0;
  for (int r = threadIdx.x; r < nrow; r += blockDim.x) s += part[(size_t)r * ncol + c];
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[c] = s * scale;
}

__global__ void k_add(double* __restrict__ a, const double* __restrict__ b, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] += b[i];
}

__global__ void k_conj_scale(const double2* __restrict__ in, double2* __restrict__ out, int n,
                             double s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_double2(in[i].x * s, -in[i].y * s);
}

}  // namespace rho

// ===========================================================================


namespace rho {

// ---- BLYP (Becke 88 exchange gradient correction + LYP correlation)

// becke_gcx_lda (cp_becke.C:44-73): the spin density rho/2, |grad|^2/4
__device__ void becke_gcx(double rho, double g2, double& f, double& dfdn, double& dfdg) {
  const double beta = 0.0042;  // cp_grad_rho_ctrl.C:53
  rho *= 0.5;
  g2 *= 0.25;
  const double r13 = cbrt(rho), r43 = rho * r13;
  const double x = sqrt(g2) / r43;
  const double root = sqrt(1.0 + x * x);
  const double asinch = log(x + root);
  const double bterm = 1.0 + 6.0 * beta * x * asinch;
  const double bx = x * x / bterm, bxx = x / bterm;
  const double bpx = 2.0 * bxx - 6.0 * beta * bxx * bxx * (asinch + x / root);
  f = -2.0 * beta * r43 * bx;
  dfdn = -beta * ((4.0 / 3.0) * r13 * (bx - x * bpx));
  dfdg = -beta * bpx;
}

// lyp_gcc (cp_becke.C:121-170)
__device__ void lyp_gcc(double rho, double g2, double& f, double& dfdn, double& dfdg) {
  const double a = 0.049180, b = 0.1320, c = 0.25330, d = 0.3490;
  const double cf = 0.30 * 9.570780000627304;  // 0.3 (3 pi^2)^{2/3}
  const double drho = sqrt(g2);
  const double r13 = cbrt(rho);                 // rho^{1/3}
  const double rm13 = 1.0 / r13;                // rho^{-1/3}
  const double rm43 = rm13 / rho;               // rho^{-4/3}
  const double rm113 = rm13 * rm13 / (rho * rho * rho);  // rho^{-11/3}
  const double den = 1.0 + d * rm13, den2 = den * den;
  const double cexp = exp(-c * rm13);
  const double omega = cexp * rm113 / den;
  double br = (d * rm43 + den * (c * rm43 - 11.0 / rho)) / 3.0;
  const double domega = omega * br / den;
  const double delta = c * rm13 + d * rm13 / den;
  br = (d * rm13 - den) * d * rm43 / den2;
  const double ddelta = (-c * rm43 + br) / 3.0;
  const double rho2 = rho * rho;
  const double term1 = -a * rho / den;
  const double br1 = ((5.0 - 7.0 / 6.0 * delta) / 3.0) * g2;
  const double r83 = rho2 * r13 * r13;          // rho^{8/3}
  const double br2 = 4.0 * cf * r83 + br1;
  const double br3 = (0.250 * br2 - 11.0 * g2 / 24.0) * rho2;
  const double term2 = -a * b * omega * br3;
  const double arho = 0.250 * br2 - 11.0 * g2 / 24.0;
  const double darho = 0.250 * (32.0 * cf * (rho * r13 * r13) / 3.0 - 7.0 / 18.0 * ddelta * g2);
  const double dprho = 2.0 * arho * rho + darho * rho2;
  const double dterm1 = -a * (1.0 + (4.0 / 3.0) * d * rm13) / den2;
  const double dterm2 = -a * b * (domega * br3 + omega * dprho);
  f = term1 + term2;
  dfdn = dterm1 + dterm2;
  dfdg = -a * b * omega * (0.50 * ((5.0 - 7.0 / 6.0 * delta) / 3.0) - 11.0 / 12.0) * rho2 * drho;
}

// CP_getGGAFunctional's point loop (cp_grad_rho_ctrl.C:81-176): vks += df/drho,
// g <- unit(grad rho) df/d|grad rho| in place, block partials of ex + ec
__global__ void k_gga(const double* __restrict__ rho, double* __restrict__ gx,
                      double* __restrict__ gy, double* __restrict__ gz, double* __restrict__ vks,
                      size_t n, double rho_cut, double heali, double* __restrict__ part) {
  __shared__ double red[32];
  double e = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double r = rho[i];
    double ux = 0.0, uy = 0.0, uz = 0.0;
    if (r > rho_cut) {
      const double x = gx[i], y = gy[i], z = gz[i];
      const double g2 = x * x + y * y + z * z;
      double rsw = (r - rho_cut) * heali;
      rsw = fmin(fmax(rsw, 0.0), 1.0);
      const double srho = rsw * rsw * (3.0 - 2.0 * rsw);
      const double dsrho = 6.0 * rsw * (1.0 - rsw) * heali;
      double fx, dfx, dgx, fc, dfc, dgc;
      becke_gcx(r, g2, fx, dfx, dgx);
      lyp_gcc(r, g2, fc, dfc, dgc);
      dfx = dfx * srho + fx * dsrho;
      dfc = dfc * srho + fc * dsrho;
      e += (fx + fc) * srho;
      vks[i] += dfx + dfc;
      if (g2 > 0.0) {
        const double s = (dgx + dgc) * srho / sqrt(g2);
        ux = x * s;
        uy = y * s;
        uz = z * s;
      }
    }
    gx[i] = ux;
    gy[i] = uy;
    gz[i] = uz;
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) part[blockIdx.x] = e;
}

// E_GGA = sum * scale -> energies[EXC_GGA] (and added to EXC when asked)
__global__ void k_gga_energy(const double* __restrict__ part, int nblk, double scale,
                             int add_to_exc, double* __restrict__ energies) {
  __shared__ double red[32];
  double e = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) e += part[i];
  e = block_sum(e, red);
  if (threadIdx.x == 0) {
    energies[CPSTEP_E_EXC_GGA] = e * scale;
    if (add_to_exc) energies[CPSTEP_E_EXC] += e * scale;
  }
}

__device__ __forceinline__ void gvec(const double* hmati, int a, int b, int c, double (&g)[3]) {
  const double tpi = 2.0 * M_PI;
#pragma unroll
  for (int d = 0; d < 3; ++d)
    g[d] = tpi * ((double)a * hmati[3 * d] + (double)b * hmati[3 * d + 1] +
                  (double)c * hmati[3 * d + 2]);
}

// The transformed density held here is conj of the reference's rho(G) and the
// G -> r transform sums c(G) e^{-iG.r}: the gradient's input is then
// -i g_d (transformed rho) / vol, as in divRhoVksGspace (times -i g, the
// backward FFTs scaled 1/vol).  out[d][p], d = x, y, z.
__global__ void k_grad_g(const double2* __restrict__ rhog, const int* __restrict__ kx,
                         const int* __restrict__ ky, const int* __restrict__ kz, int np,
                         const double* __restrict__ hmati, double inv_vol,
                         double2* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  double g[3];
  gvec(hmati, kx[p], ky[p], kz[p], g);
  const double2 v = rhog[p];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    out[(size_t)d * np + p] = make_double2(g[d] * v.y * inv_vol, -g[d] * v.x * inv_vol);
}

// White-Bird: w(G) = -i g . u(G) (acceptWhiteByrd), u transformed with 1/N
__global__ void k_div_g(const double2* __restrict__ u, const int* __restrict__ kx,
                        const int* __restrict__ ky, const int* __restrict__ kz, int np,
                        const double* __restrict__ hmati, double2* __restrict__ w) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  double g[3];
  gvec(hmati, kx[p], ky[p], kz[p], g);
  double sx = 0.0, sy = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double2 v = u[(size_t)d * np + p];
    sx += g[d] * v.x;
    sy += g[d] * v.y;
  }
  w[p] = make_double2(sy, -sx);
}

__global__ void k_sub(double* __restrict__ a, const double* __restrict__ b, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] -= b[i];
}

}  // namespace rho

static int upload_i(int** d, const std::vector<int>& h) {
  CPSTEP_CUDA_TRY(cudaMalloc(d, sizeof(int) * std::max<size_t>(1, h.size())));
  CPSTEP_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
  return CPSTEP_OK;
}
static int upload_d(double** d, const std::vector<double>& h) {
  CPSTEP_CUDA_TRY(cudaMalloc(d, sizeof(double) * std::max<size_t>(1, h.size())));
  CPSTEP_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
  return CPSTEP_OK;
}

int rho_init(cpstep_ctx* c, double box_len, double ecut_ry) {
  std::vector<int> kx, ky, kz, runs;
  int rc = cpstep_density_layout(box_len, ecut_ry, c->nx, kx, ky, kz, runs);
  if (rc) {
    cpstep_set_error("density sphere does not fit the %d grid", c->nx);
    return rc;
  }
  int nl = (int)runs.size() / 14;
  std::vector<int> off(nl), nneg(nl), npos(nl), zneg(nl), zpos(nl), xy(nl);
  int kxmax = 0;
  for (int l = 0; l < nl; ++l) {
    const int* rn = runs.data() + 14 * l;
    const int* rp = rn + 7;
    off[l] = rn[3]; nneg[l] = rn[4]; npos[l] = rp[4];
    zneg[l] = rn[2] + (c->nz - rn[6]);
    zpos[l] = rp[2];
    xy[l] = rp[0] | (rp[1] << 16);
    kxmax = std::max(kxmax, rp[0]);
  }
  int np = (int)kx.size();
  // consecutive kz along every line: the Hartree / local passes then advance
  // the z phase by one multiplication per point
  {
    bool ok = true;
    for (int l = 0; l < nl && ok; ++l) {
      const int e = l + 1 < nl ? off[l + 1] : np;
      for (int q = off[l]; q + 1 < e; ++q)
        if (kz[q + 1] != kz[q] + 1) ok = false;
    }
    c->rg.kz_runs = ok ? 1 : 0;
  }
  std::vector<double> g2(np), wpt(np);
  const double* hi = c->hmati;
  for (int i = 0; i < np; ++i) {
    double a = kx[i], b = ky[i], cc = kz[i];
    double gx = (a * hi[0] + b * hi[1] + cc * hi[2]) * 2.0 * M_PI;
    double gy = (a * hi[3] + b * hi[4] + cc * hi[5]) * 2.0 * M_PI;
    double gz = (a * hi[6] + b * hi[7] + cc * hi[8]) * 2.0 * M_PI;
    g2[i] = gx * gx + gy * gy + gz * gz;
    wpt[i] = kx[i] == 0 ? 1.0 : 2.0;
    if (kx[i] == 0 && ky[i] == 0 && kz[i] == 0) c->rho_izero = i;
  }
  RhoGeom& r = c->rg;
  r.npts = np;
  r.nlines = nl;
  r.nlpad = (nl + 3) & ~3;
  r.nplane_x = kxmax + 1;
  if ((rc = upload_i(&r.line_off, off)) || (rc = upload_i(&r.line_nneg, nneg)) ||
      (rc = upload_i(&r.line_npos, npos)) || (rc = upload_i(&r.line_zneg, zneg)) ||
      (rc = upload_i(&r.line_zpos, zpos)) || (rc = upload_i(&r.line_xy, xy)) ||
      (rc = upload_i(&r.kx, kx)) || (rc = upload_i(&r.ky, ky)) || (rc = upload_i(&r.kz, kz)) ||
      (rc = upload_d(&r.g2, g2)) || (rc = upload_d(&r.wpt, wpt)))
    return rc;
  size_t pen = (size_t)c->nz * r.nlpad * sizeof(double2);
  CPSTEP_CUDA_TRY(cudaMalloc(&r.pen_a, pen));
  CPSTEP_CUDA_TRY(cudaMalloc(&r.pen_b, pen));
  CPSTEP_CUDA_TRY(cudaMalloc(&r.rhog, sizeof(double2) * np));
  CPSTEP_CUDA_TRY(cudaMalloc(&r.vg, sizeof(double2) * np));
  CPSTEP_CUDA_TRY(cudaMalloc(&r.fterm, sizeof(double4) * np));
  size_t nr = (size_t)c->nx * c->ny * c->nz;
  CPSTEP_CUDA_TRY(cudaMalloc(&r.vhl, sizeof(double) * nr));
  r.nblk_xc = 4 * c->num_sms;
  r.nblk_h = nl;  // k_hart_lines: one block per line
  CPSTEP_CUDA_TRY(cudaMalloc(&r.part, sizeof(double) * (2 * r.nblk_xc + 3 * r.nblk_h + 8)));
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_energies, sizeof(double) * CPSTEP_NENERGY));
  CPSTEP_CUDA_TRY(cudaMemset(c->d_energies, 0, sizeof(double) * CPSTEP_NENERGY));
  return CPSTEP_OK;
}

void rho_free(cpstep_ctx* c) {
  RhoGeom& r = c->rg;
  cudaFree(r.line_off); cudaFree(r.line_nneg); cudaFree(r.line_npos); cudaFree(r.line_zneg);
  cudaFree(r.line_zpos); cudaFree(r.line_xy); cudaFree(r.kx); cudaFree(r.ky); cudaFree(r.kz);
  cudaFree(r.g2); cudaFree(r.wpt); cudaFree(r.pen_a); cudaFree(r.pen_b); cudaFree(r.rhog);
  cudaFree(r.vg); cudaFree(r.fterm); cudaFree(r.vhl); cudaFree(r.part);
  cudaFree(c->d_gga_r); cudaFree(c->d_gga_g);
  c->d_gga_r = nullptr;
  c->d_gga_g = nullptr;
  cudaFree(c->d_energies);
  eesloc_free(c);
  AtomData& a = c->atoms;
  cudaFree(a.typ); cudaFree(a.frac); cudaFree(a.q); cudaFree(a.vps); cudaFree(a.gzvps);
  cudaFree(a.ex); cudaFree(a.ey); cudaFree(a.ez); cudaFree(a.ezt); cudaFree(a.rank);
  cudaFree(a.fpart); cudaFree(a.pos);
}

FftJob rho_job(const cpstep_ctx* c) {
  FftJob j;
  const RhoGeom& r = c->rg;
  j.g.nx = c->nx; j.g.ny = c->ny; j.g.nz = c->nz;
  j.g.nlines = r.nlines; j.g.nlpad = r.nlpad; j.g.nplane_x = r.nplane_x; j.g.npts = r.npts;
  j.g.line_off = r.line_off; j.g.line_nneg = r.line_nneg; j.g.line_npos = r.line_npos;
  j.g.line_zneg = r.line_zneg; j.g.line_zpos = r.line_zpos; j.g.line_xy = r.line_xy;
  j.g.g2 = r.g2; j.g.wpt = r.wpt;
  j.pen_a = r.pen_a;
  j.pen_b = r.pen_b;
  return j;
}

static int eesloc_alloc(cpstep_ctx* c);

int atoms_set(cpstep_ctx* c, int natm, int ntyp, const int* typ, const double* pos,
              const double* q, int nspl, double gmin, double dg, const double* vps,
              const double* gzvps, double alp_ewd) {
  AtomData& a = c->atoms;
  cudaFree(a.typ); cudaFree(a.frac); cudaFree(a.q); cudaFree(a.vps); cudaFree(a.gzvps);
  cudaFree(a.ex); cudaFree(a.ey); cudaFree(a.ez); cudaFree(a.ezt); cudaFree(a.rank);
  cudaFree(a.fpart); cudaFree(a.pos);
  a = AtomData();
  if (ntyp > CPSTEP_MAX_TYPES || natm > rho::kMaxAtoms) {
    cpstep_set_error("atoms: %d types / %d atoms exceed the limits %d / %d", ntyp, natm,
                     CPSTEP_MAX_TYPES, rho::kMaxAtoms);
    return CPSTEP_ERR_ARG;
  }
  std::vector<int> t(typ, typ + natm);
  for (int v : t)
    if (v < 0 || v >= ntyp) {
      cpstep_set_error("atoms: type index out of range");
      return CPSTEP_ERR_ARG;
    }
  // type order (stable): rank[atom], tstart[type]
  std::vector<int> cnt(ntyp + 1, 0), rank(natm);
  for (int v : t) ++cnt[v + 1];
  for (int k = 0; k < ntyp; ++k) cnt[k + 1] += cnt[k];
  for (int k = 0; k <= ntyp; ++k) a.tstart[k] = cnt[k];
  {
    std::vector<int> next(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < natm; ++i) rank[i] = next[t[i]]++;
  }
  std::vector<double> frac(3 * (size_t)natm);
  const double* hi = c->hmati;  // s = hmati R (column-major hmati)
  for (int i = 0; i < natm; ++i) {
    const double* R = pos + 3 * i;
    for (int d = 0; d < 3; ++d)
      frac[3 * i + d] = hi[d] * R[0] + hi[d + 3] * R[1] + hi[d + 6] * R[2];
  }
  int rc;
  if ((rc = upload_i(&a.typ, t)) || (rc = upload_i(&a.rank, rank)) ||
      (rc = upload_d(&a.frac, frac)) ||
      (rc = upload_d(&a.q, std::vector<double>(q, q + ntyp))) ||
      (rc = upload_d(&a.vps, std::vector<double>(vps, vps + (size_t)ntyp * 4 * nspl))) ||
      (rc = upload_d(&a.gzvps, std::vector<double>(gzvps, gzvps + ntyp))) ||
      (rc = upload_d(&a.pos, std::vector<double>(pos, pos + 3 * (size_t)natm))))
    return rc;
  a.h_q.resize(natm);
  for (int i = 0; i < natm; ++i) a.h_q[i] = q[t[i]];
  a.natm = natm;
  a.ntyp = ntyp;
  a.nspl = nspl;
  a.gmin = gmin;
  a.dg = dg;
  a.alp_ewd = alp_ewd;
  a.kxm = c->nx / 2;
  a.kym = c->ny / 2;
  a.kzm = c->nz / 2;
  CPSTEP_CUDA_TRY(cudaMalloc(&a.ex, sizeof(double2) * (a.kxm + 1) * natm));
  CPSTEP_CUDA_TRY(cudaMalloc(&a.ey, sizeof(double2) * (2 * a.kym + 1) * natm));
  CPSTEP_CUDA_TRY(cudaMalloc(&a.ez, sizeof(double2) * (2 * a.kzm + 1) * natm));
  CPSTEP_CUDA_TRY(cudaMalloc(&a.ezt, sizeof(double2) * (2 * a.kzm + 1) * natm));
  a.nfblk = std::max(1, std::min(c->rg.nlines, 8 * c->num_sms));  // line partials per block
  CPSTEP_CUDA_TRY(cudaMalloc(&a.fpart, sizeof(double) * 3 * (size_t)natm * a.nfblk));
  rho::k_phase<<<cdiv(natm, 128), 128, 0, c->stream>>>(a.frac, natm, a.kxm, a.kym, a.kzm, a.rank,
                                                        a.ex, a.ey, a.ez, a.ezt);
  CPSTEP_LAUNCH_CHECK();
  if (!c->d_hmati) CPSTEP_CUDA_TRY(cudaMalloc(&c->d_hmati, sizeof(double) * 9));
  CPSTEP_CUDA_TRY(cudaMemcpy(c->d_hmati, c->hmati, sizeof(double) * 9, cudaMemcpyHostToDevice));
  if (c->eloc.on) return eesloc_alloc(c);  // the EES form's tables follow the atoms
  return CPSTEP_OK;
}

static rho::Atoms atoms_view(const cpstep_ctx* c) {
  const AtomData& a = c->atoms;
  rho::Atoms A;
  A.natm = a.natm; A.ntyp = a.ntyp; A.typ = a.typ; A.frac = a.frac; A.q = a.q; A.vps = a.vps;
  A.gzvps = a.gzvps; A.nspl = a.nspl; A.gmin = a.gmin; A.dg = a.dg;
  A.kxm = a.kxm; A.kym = a.kym; A.kzm = a.kzm; A.ex = a.ex; A.ey = a.ey; A.ez = a.ez;
  A.ezt = a.ezt; A.rank = a.rank;
  for (int k = 0; k <= CPSTEP_MAX_TYPES; ++k) A.tstart[k] = a.tstart[k];
  return A;
}

// New atom positions (host, natm x 3): queued H2D copy, fractional
// coordinates and phase tables on the context's stream.
int atoms_set_positions(cpstep_ctx* c, const double* h_pos) {
  AtomData& a = c->atoms;
  if (a.natm <= 0) {
    cpstep_set_error("set_positions: no atoms set");
    return CPSTEP_ERR_STATE;
  }
  if (!a.pos) CPSTEP_CUDA_TRY(cudaMalloc(&a.pos, sizeof(double) * 3 * a.natm));
  CPSTEP_CUDA_TRY(cudaMemcpyAsync(a.pos, h_pos, sizeof(double) * 3 * a.natm,
                                  cudaMemcpyHostToDevice, c->stream));
  rho::k_frac<<<cdiv(a.natm, 128), 128, 0, c->stream>>>(a.pos, c->d_hmati, a.natm, a.frac);
  CPSTEP_LAUNCH_CHECK();
  rho::k_phase<<<cdiv(a.natm, 128), 128, 0, c->stream>>>(a.frac, a.natm, a.kxm, a.kym, a.kzm,
                                                          a.rank, a.ex, a.ey, a.ez, a.ezt);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// new positions from device memory (the atom integrator's output)
int atoms_set_positions_dev(cpstep_ctx* c, const double* d_pos) {
  AtomData& a = c->atoms;
  if (a.natm <= 0 || !a.pos) {
    cpstep_set_error("set_positions: no atoms set");
    return CPSTEP_ERR_STATE;
  }
  if (d_pos != a.pos)
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(a.pos, d_pos, sizeof(double) * 3 * a.natm,
                                    cudaMemcpyDeviceToDevice, c->stream));
  rho::k_frac<<<cdiv(a.natm, 128), 128, 0, c->stream>>>(a.pos, c->d_hmati, a.natm, a.frac);
  CPSTEP_LAUNCH_CHECK();
  rho::k_phase<<<cdiv(a.natm, 128), 128, 0, c->stream>>>(a.frac, a.natm, a.kxm, a.kym, a.kzm,
                                                          a.rank, a.ex, a.ey, a.ez, a.ezt);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// E_xc, muxc -> energies[EXC], [MUXC]; vxc written to out
int rho_xc(cpstep_ctx* c, const double* rho_r, double* vxc, double* energies) {
  size_t nr = (size_t)c->nx * c->ny * c->nz;
  RhoGeom& r = c->rg;
  rho::k_xc<<<r.nblk_xc, 256, 0, c->stream>>>(rho_r, vxc, nr,
                                              c->xc == CPSTEP_XC_BLYP ? 0.0 : 1.0, r.part);
  CPSTEP_LAUNCH_CHECK();
  rho::k_sum_cols<<<2, 256, 0, c->stream>>>(r.part, r.nblk_xc, 2, energies + CPSTEP_E_EXC,
                                            c->vol / (double)nr);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// rho(r) -> transformed density (conj of the reference rho(G)) in r.rhog
int rho_r2g(cpstep_ctx* c, const double* rho_r) {
  FftJob j = rho_job(c);
  double scale = c->vol / ((double)c->nx * c->ny * c->nz);
  return c->ops64.r2g(c, j, rho_r, reinterpret_cast<double*>(c->rg.rhog), 1, scale);
}

// CP_getGGAFunctional on given gradients (overwritten with the u terms)
int rho_gga_functional(cpstep_ctx* c, const double* rho_r, double* gx, double* gy, double* gz,
                       double* vks_r, double* energies, int add_to_exc) {
  const size_t nr = (size_t)c->nx * c->ny * c->nz;
  RhoGeom& r = c->rg;
  const double rho_cut = 0.1 * c->gga_cut, heali = 1.0 / (3.9 * c->gga_cut);
  rho::k_gga<<<r.nblk_xc, 256, 0, c->stream>>>(rho_r, gx, gy, gz, vks_r, nr, rho_cut, heali,
                                               r.part);
  CPSTEP_LAUNCH_CHECK();
  rho::k_gga_energy<<<1, 256, 0, c->stream>>>(r.part, r.nblk_xc, c->vol / (double)nr,
                                              add_to_exc, energies);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// BLYP gradient correction after rho_r2g (r.rhog holds the transformed
// density): gradients, the functional, the White-Bird term subtracted from vks
int rho_gga(cpstep_ctx* c, const double* rho_r, double* vks_r, double* energies) {
  if (!c->d_gga_r || !c->d_gga_g) {
    cpstep_set_error("gga: BLYP scratch not allocated (cpstep_set_xc)");
    return CPSTEP_ERR_STATE;
  }
  const size_t nr = (size_t)c->nx * c->ny * c->nz;
  RhoGeom& r = c->rg;
  FftJob j = rho_job(c);
  const int np = r.npts;
  double* gr = c->d_gga_r;
  double2* gg = c->d_gga_g;
  rho::k_grad_g<<<cdiv(np, 256), 256, 0, c->stream>>>(r.rhog, r.kx, r.ky, r.kz, np, c->d_hmati,
                                                      1.0 / c->vol, gg);
  CPSTEP_LAUNCH_CHECK();
  for (int d = 0; d < 3; ++d)
    if (int rc = c->ops64.g2r(c, j, reinterpret_cast<const double*>(gg + (size_t)d * np),
                              gr + d * nr, 1))
      return rc;
  if (int rc = rho_gga_functional(c, rho_r, gr, gr + nr, gr + 2 * nr, vks_r, energies, 1))
    return rc;
  for (int d = 0; d < 3; ++d)  // u scaled 1/N on the way (whiteByrdFFT)
    if (int rc = c->ops64.r2g(c, j, gr + d * nr, reinterpret_cast<double*>(gg + (size_t)d * np),
                              1, 1.0 / (double)nr))
      return rc;
  rho::k_div_g<<<cdiv(np, 256), 256, 0, c->stream>>>(gg, r.kx, r.ky, r.kz, np, c->d_hmati,
                                                     gg + 3 * (size_t)np);
  CPSTEP_LAUNCH_CHECK();
  if (int rc = c->ops64.g2r(c, j, reinterpret_cast<const double*>(gg + 3 * (size_t)np), r.vhl, 1))
    return rc;
  rho::k_sub<<<2 * c->num_sms, 256, 0, c->stream>>>(vks_r, r.vhl, nr);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

void eesloc_free(cpstep_ctx* c) {
  EesLocal& e = c->eloc;
  cudaFree(e.ig); cudaFree(e.mn); cudaFree(e.dmn); cudaFree(e.bden);
  cudaFree(e.tx); cudaFree(e.ty); cudaFree(e.tz); cudaFree(e.dtx); cudaFree(e.dty);
  cudaFree(e.dtz); cudaFree(e.tzt);
  e = EesLocal();
}

// buffers of the EES form for the context's atoms and sphere extents
static int eesloc_alloc(cpstep_ctx* c) {
  EesLocal& e = c->eloc;
  const AtomData& a = c->atoms;
  const int ng = e.ngrid, natm = a.natm;
  cudaFree(e.ig); cudaFree(e.mn); cudaFree(e.dmn);
  cudaFree(e.tx); cudaFree(e.ty); cudaFree(e.tz); cudaFree(e.dtx); cudaFree(e.dty);
  cudaFree(e.dtz); cudaFree(e.tzt);
  const size_t nb = (size_t)natm * 3 * kNlInterp;
  const size_t nx = (size_t)(a.kxm + 1) * natm, ny = (size_t)(2 * a.kym + 1) * natm;
  const size_t nz = (size_t)(2 * a.kzm + 1) * natm;
  CPSTEP_CUDA_TRY(cudaMalloc(&e.ig, sizeof(int) * nb));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.mn, sizeof(double) * nb));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.dmn, sizeof(double) * nb));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.tx, sizeof(double2) * nx));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.dtx, sizeof(double2) * nx));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.ty, sizeof(double2) * ny));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.dty, sizeof(double2) * ny));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.tz, sizeof(double2) * nz));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.dtz, sizeof(double2) * nz));
  CPSTEP_CUDA_TRY(cudaMalloc(&e.tzt, sizeof(double2) * nz));
  e.natm = natm;
  (void)ng;
  return CPSTEP_OK;
}

// cpstep_set_local_ees: on = 1 computes the pass in the EES form on an
// ngrid^3 grid with B-splines of order n_interp (kNlInterp only), on = 0
// returns to the explicit structure factors.
int eesloc_set(cpstep_ctx* c, int on, int ngrid, int n_interp) {
  if (!on) {
    eesloc_free(c);
    return CPSTEP_OK;
  }
  if (c->atoms.natm <= 0) {
    cpstep_set_error("set_local_ees: set the atoms first (cpstep_set_atoms)");
    return CPSTEP_ERR_STATE;
  }
  if (n_interp != kNlInterp || ngrid < n_interp) {
    cpstep_set_error("set_local_ees: B-spline order %d on a %d grid (order %d is built, grid >= "
                     "order)", n_interp, ngrid, kNlInterp);
    return CPSTEP_ERR_ARG;
  }
  eesloc_free(c);
  EesLocal& e = c->eloc;
  e.ngrid = ngrid;
  std::vector<double> br, bi;
  ees_bspline_weights(n_interp, ngrid, br, bi);
  std::vector<double2> h(ngrid);
  for (int m = 0; m < ngrid; ++m) h[m] = make_double2(br[m], bi[m]);
  CPSTEP_CUDA_TRY(cudaMalloc(&e.bden, sizeof(double2) * ngrid));
  CPSTEP_CUDA_TRY(cudaMemcpy(e.bden, h.data(), sizeof(double2) * ngrid, cudaMemcpyHostToDevice));
  if (int rc = eesloc_alloc(c)) return rc;
  e.on = 1;  // published last: the pass reads the form from here
  return CPSTEP_OK;
}

// the EES form of rho_hart
static int eesloc_hart(cpstep_ctx* c, double* energies, double* force) {
  RhoGeom& r = c->rg;
  EesLocal& e = c->eloc;
  const AtomData& ad = c->atoms;
  if (e.natm != ad.natm)
    if (int rc = eesloc_alloc(c)) return rc;
  const int natm = ad.natm;
  if (int rc = ees_bspline_launch(c, ad.frac, natm, e.ngrid, e.ig, e.mn, e.dmn)) return rc;
  const long long nt = (long long)natm * ((ad.kxm + 1) + (2 * ad.kym + 1) + (2 * ad.kzm + 1));
  rho::k_eloc_tables<<<(unsigned)((nt + 127) / 128), 128, 0, c->stream>>>(
      e.ig, e.mn, e.dmn, natm, e.ngrid, ad.kxm, ad.kym, ad.kzm, e.bden, ad.rank, e.tx, e.ty,
      e.tz, e.dtx, e.dty, e.dtz, e.tzt);
  CPSTEP_LAUNCH_CHECK();
  rho::Atoms A = atoms_view(c);
  A.ex = e.tx; A.ey = e.ty; A.ez = e.tz; A.ezt = e.tzt;
  const double ecut4 = 8.0 * (0.5 * c->ecut_ry);
  double* hp = r.part + 2 * r.nblk_xc;
  const size_t hsm = sizeof(double2) * (size_t)natm;
  if (hsm > 48 * 1024)
    CPSTEP_CUDA_TRY(cudaFuncSetAttribute(rho::k_hart_lines,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm));
  rho::k_hart_lines<<<r.nlines, rho::HT, hsm, c->stream>>>(
      r.rhog, r.line_off, r.nlines, r.kx, r.ky, r.kz, r.npts, c->d_hmati, c->vol, ecut4,
      ad.alp_ewd, A, r.vg, r.fterm, hp);
  CPSTEP_LAUNCH_CHECK();
  rho::k_sum_cols<<<3, 256, 0, c->stream>>>(hp, r.nlines, 3, energies + CPSTEP_E_HART, 1.0);
  CPSTEP_LAUNCH_CHECK();
  if (c->rho_izero >= 0) {
    rho::k_eloc_g0<<<1, 1, 0, c->stream>>>(r.rhog, c->rho_izero, c->vol, A, r.vg,
                                           energies + CPSTEP_E_EXT);
    CPSTEP_LAUNCH_CHECK();
  }
  if (force) {
    const int per = cdiv(natm, 256);
    const int nthr = std::max(32, cdiv(cdiv(natm, per), 32) * 32);
    const int lmax = c->nz + 1;
    const size_t fsm = (sizeof(double2) * ad.ntyp + sizeof(int)) * (size_t)lmax;
    if (fsm > 48 * 1024)
      CPSTEP_CUDA_TRY(cudaFuncSetAttribute(rho::k_eloc_forces_lines,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)fsm));
    rho::ElocD D{e.dtx, e.dty, e.dtz, (double)e.ngrid};
    rho::k_eloc_forces_lines<<<ad.nfblk, nthr, fsm, c->stream>>>(
        r.fterm, r.line_off, r.nlines, r.kx, r.ky, r.kz, r.npts, c->d_hmati, c->vol, A, D, lmax,
        ad.fpart);
    CPSTEP_LAUNCH_CHECK();
    rho::k_sum_cols<<<3 * natm, 256, 0, c->stream>>>(ad.fpart, ad.nfblk, 3 * natm, force, 1.0);
    CPSTEP_LAUNCH_CHECK();
  }
  return CPSTEP_OK;
}

// Hartree + local + Ewald from r.rhog: conj(vks) in r.vg, energies, force terms
int rho_hart(cpstep_ctx* c, double* energies, double* force) {
  RhoGeom& r = c->rg;
  if (c->atoms.natm <= 0) {
    cpstep_set_error("hart_eext: no atoms set (cpstep_set_atoms)");
    return CPSTEP_ERR_STATE;
  }
  if (c->eloc.on) return eesloc_hart(c, energies, force);
  rho::Atoms A = atoms_view(c);
  double ecut4 = 8.0 * (0.5 * c->ecut_ry);
  double* hp = r.part + 2 * r.nblk_xc;
  if (r.kz_runs) {
    const size_t hsm = sizeof(double2) * (size_t)c->atoms.natm * (32 / rho::HG) * rho::HWARPS;
    if (hsm > 48 * 1024)
      CPSTEP_CUDA_TRY(cudaFuncSetAttribute(rho::k_hart_lines_rec,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)hsm));
    const int nb = std::min(cdiv(r.nlines, (32 / rho::HG) * rho::HWARPS), 8 * c->num_sms);
    rho::k_hart_lines_rec<<<nb, 32 * rho::HWARPS, hsm, c->stream>>>(
        r.rhog, r.line_off, r.nlines, r.kx, r.ky, r.kz, r.npts, c->d_hmati, c->vol, ecut4,
        c->atoms.alp_ewd, A, r.vg, r.fterm, hp);
  } else {
    const size_t hsm = sizeof(double2) * (size_t)c->atoms.natm;
    if (hsm > 48 * 1024)
      CPSTEP_CUDA_TRY(cudaFuncSetAttribute(rho::k_hart_lines,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)hsm));
    rho::k_hart_lines<<<r.nlines, rho::HT, hsm, c->stream>>>(
        r.rhog, r.line_off, r.nlines, r.kx, r.ky, r.kz, r.npts, c->d_hmati, c->vol, ecut4,
        c->atoms.alp_ewd, A, r.vg, r.fterm, hp);
  }
  CPSTEP_LAUNCH_CHECK();
  rho::k_sum_cols<<<3, 256, 0, c->stream>>>(hp, r.nlines, 3, energies + CPSTEP_E_HART, 1.0);
  CPSTEP_LAUNCH_CHECK();
  if (c->rho_izero >= 0) {
    rho::k_hart_g0<<<1, 1, 0, c->stream>>>(r.rhog, c->rho_izero, c->vol, A, r.vg,
                                           energies + CPSTEP_E_EXT);
    CPSTEP_LAUNCH_CHECK();
  }
  if (force) {
    const int natm = c->atoms.natm;
    const int per = cdiv(natm, 256);  // atoms per thread, <= 4 (kMaxAtoms)
    const int nt = std::max(32, cdiv(cdiv(natm, per), 32) * 32);
    const int lmax = c->nz + 1;
    const size_t fsm = (sizeof(double2) * c->atoms.ntyp + sizeof(int)) * (size_t)lmax;
    auto kf = r.kz_runs ? rho::k_local_forces_lines<true> : rho::k_local_forces_lines<false>;
    if (fsm > 48 * 1024)
      CPSTEP_CUDA_TRY(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)fsm));
    kf<<<c->atoms.nfblk, nt, fsm, c->stream>>>(r.fterm, r.line_off, r.nlines, r.kx, r.ky, r.kz,
                                               r.npts, c->d_hmati, c->vol, A, lmax,
                                               c->atoms.fpart);
    CPSTEP_LAUNCH_CHECK();
    rho::k_sum_cols<<<3 * natm, 256, 0, c->stream>>>(c->atoms.fpart, c->atoms.nfblk, 3 * natm,
                                                     force, 1.0);
    CPSTEP_LAUNCH_CHECK();
  }
  return CPSTEP_OK;
}

// V_KS(r) = vxc (already in vks_r) + sum_G vks(G) e^{iGr}
int rho_vks_r(cpstep_ctx* c, double* vks_r) {
  FftJob j = rho_job(c);
  size_t nr = (size_t)c->nx * c->ny * c->nz;
  if (int rc = c->ops64.g2r(c, j, reinterpret_cast<const double*>(c->rg.vg), c->rg.vhl, 1))
    return rc;
  rho::k_add<<<2 * c->num_sms, 256, 0, c->stream>>>(vks_r, c->rg.vhl, nr);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// helpers for the ABI entries that exchange reference-convention arrays
int rho_conj_scale(cpstep_ctx* c, const double* in, double* out, int n, double s) {
  rho::k_conj_scale<<<cdiv(n, 256), 256, 0, c->stream>>>(
      reinterpret_cast<const double2*>(in), reinterpret_cast<double2*>(out), n, s);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}
