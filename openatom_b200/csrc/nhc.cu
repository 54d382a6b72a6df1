// The isokinetic Nose-Hoover chain thermostat of the CP coefficients
// (ISOKIN_OPT = 1), wrapped around the velocity Verlet of step.cu.
//
//   CPINTEGRATE::initCPNHC          src_piny_physics_v1.0/abinito_physics/cp_integrate/
//                                   cp_isokin.C:45-141
//   CPINTEGRATE::cp_isoNHC_update   cp_isokin.C:150-311 (set_yosh :320-388)
//   CPINTEGRATE::CP_integrate_dyn / cp_evolve_vel / get_fictKE
//                                   cp_integrate/cp_dynamics.C:22-256
//
// One chain set per state (the reference with one G-space chare per state):
// the state's non-redundant coefficients in the reference's chare order (G=0,
// the unique Gx=0 points, the rest; each in packed order) are cut into nck
// chunks, each with num chains of length 2.  The thermostat only rescales the
// velocities of a chunk, so a step is three passes:
//   k_nhc_ekin    kick of the previous step (iteration > 1) and the chunk
//                 kinetic energies sum m |v|^2 (deterministic block partials);
//   k_nhc_update  one thread per (state, chunk): the applyorder-2 update on
//                 that energy (iteration > 1), the fictitious KE and the NHC
//                 energies of get_fictKE, the applyorder-1 update; two scales;
//   k_nhc_apply   v = ((v + kick) s2) s1 + kick, psi += v dt (the element
//                 order of cp_evolve_vel's two calls).
// The chunk energy after a scale is s^2 times the energy before it (the
// reference sums the scaled velocities again; the two differ by rounding).
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.cuh"

namespace nhc {

constexpr int kMaxNum = 8;
constexpr int kMaxNck = 8;

struct Par {
  int num, nck, nres, nyosh;
  double kT, m0, m1;
  double c1[kMaxNum];   // -4 v0 / (a4 mNHC[1]): the double-well force factor
  double a2[kMaxNum];
  double gkt[kMaxNck];  // degFreeSplt[k] * kT
  double w[9];          // Yoshida weights times dt / nres
};

__global__ void __launch_bounds__(256, 4) k_nhc_ekin(const double2* __restrict__ v, const double2* __restrict__ f,
                           const double* __restrict__ cmass, const int* __restrict__ cls,
                           const signed char* __restrict__ ck, int npts, int span, double dt,
                           int first_in, const int* __restrict__ skip, int nck,
                           double* __restrict__ part) {
  constexpr int U = 2;  // points per thread and pass, loaded before any is used
  __shared__ double red[32];
  const int first = first_in && !(skip && *skip);
  const int s = blockIdx.y;
  const int p0 = blockIdx.x * span, p1 = min(npts, p0 + span);
  const double dt2 = 0.5 * dt;
  const int B = blockDim.x;
  double acc[kMaxNck];
#pragma unroll
  for (int k = 0; k < kMaxNck; ++k) acc[k] = 0.0;
  const double2* vs = v + (size_t)s * npts;
  const double2* fs = f + (size_t)s * npts;
  for (int pb = p0 + threadIdx.x; pb < p1; pb += U * B) {
    int c[U];
    double2 vv[U], ff[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int p = pb + u * B;
      c[u] = p < p1 ? cls[p] : 0;
      vv[u] = c[u] ? vs[p] : make_double2(0.0, 0.0);
      ff[u] = (c[u] && first) ? fs[p] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (c[u] == 0) continue;
      const int p = pb + u * B;
      const double m = cmass[p];
      if (c[u] == 1) { vv[u].y = 0.0; ff[u].y = 0.0; }
      if (first) {
        const double fm = dt2 / m;
        vv[u].x += ff[u].x * fm;
        vv[u].y += ff[u].y * fm;
      }
      const double e = (vv[u].x * vv[u].x + vv[u].y * vv[u].y) * (c[u] == 2 ? 2.0 * m : m);
      const int k = ck[p];
#pragma unroll
      for (int q = 0; q < kMaxNck; ++q) acc[q] += (q == k) ? e : 0.0;
    }
  }
#pragma unroll
  for (int q = 0; q < kMaxNck; ++q) {
    if (q >= nck) break;
    const double t = block_sum(acc[q], red);
    if (threadIdx.x == 0) part[((size_t)s * gridDim.x + blockIdx.x) * nck + q] = t;
  }
}

// h and hdot of one chain's velocity update (cp_isokin.C:216-235 / :266-285);
// 1/kT, 1/sqrt(ffdot) and 1/hdot as reciprocals, cosh and sinh from e^arg and
// e^-arg above arg = 1/8 (below it sinh itself: e - 1/e would cancel).  The
// update is a serial chain of 2 x nres x nyosh of these per chunk, so its
// time is the latency of one thread's dependent FP64 operations.
__device__ __forceinline__ void hh_step(double f0, double f1, double& v0, double& v1,
                                        const Par& P, double ikT, double w4) {
  const double ffdot = (f0 * f0 * P.m0 + f1 * f1 * P.m1) * ikT;
  const double pfdot = (f0 * v0 * P.m0 + f1 * v1 * P.m1) * ikT;
  double h, hdot;
  if (ffdot * w4 * w4 > 1.0e-10) {
    const double ifr = rsqrt(ffdot);
    const double fr = ffdot * ifr;
    const double arg = fr * w4;
    const double e = exp(arg), ie = exp(-arg);  // independent: no dependent reciprocal
    const double ch = 0.5 * (e + ie);
    const double sh = arg < 0.125 ? sinh(arg) : 0.5 * (e - ie);
    h = pfdot * ifr * ifr * (ch - 1.0) + ifr * sh;
    hdot = pfdot * ifr * sh + ch;
  } else {
    h = (((ffdot * pfdot / 24.0 * w4 + ffdot / 6.0) * w4 + 0.50 * pfdot) * w4 + 1.0) * w4;
    hdot = ((ffdot * pfdot / 6.0 * w4 + ffdot / 2.0) * w4 + pfdot) * w4 + 1.0;
  }
  const double ihd = 1.0 / hdot;
  v0 = (v0 + f0 * h) * ihd;
  v1 = (v1 + f1 * h) * ihd;
}

// cp_isoNHC_update (cp_isokin.C:150-311) for one chunk of NUM chains, all in
// registers: returns the velocity scale; x, xp, vn are [NUM][2].
template <int NUM>
__device__ double iso_update(double ekin, double gkt, const Par& P, double (&x)[NUM][2],
                             double (&xp)[NUM][2], double (&vn)[NUM][2]) {
  const double ikT = 1.0 / P.kT, im0 = 1.0 / P.m0;
  double f[NUM][2];
#pragma unroll
  for (int i = 0; i < NUM; ++i) {
    xp[i][0] = 0.0;
    const double q = xp[i][1];
    f[i][0] = (ekin - gkt) * im0;
    f[i][1] = P.c1[i] * (q * (q * q - P.a2[i]));
  }
  double scale = 1.0;
  for (int ir = 0; ir < P.nres; ++ir) {
    for (int iy = 0; iy < P.nyosh; ++iy) {
      const double w2 = P.w[iy] * 0.5, w4 = P.w[iy] * 0.25;
      double vsum = 0.0;
#pragma unroll
      for (int i = 0; i < NUM; ++i) {
        hh_step(f[i][0], f[i][1], vn[i][0], vn[i][1], P, ikT, w4);
        vsum += vn[i][0];
      }
      const double aa = exp(-w4 * vsum);
      scale *= aa;
      ekin *= aa * aa;
#pragma unroll
      for (int i = 0; i < NUM; ++i) {
        x[i][0] += P.kT * vn[i][0] * w2;
        x[i][1] += vn[i][0] * (ekin - gkt) * w2;
        xp[i][1] += vn[i][1] * w2;
      }
      scale *= aa;
      ekin *= aa * aa;
#pragma unroll
      for (int i = 0; i < NUM; ++i) {
        const double q = xp[i][1];
        f[i][0] = (ekin - gkt) * im0;
        f[i][1] = P.c1[i] * (q * (q * q - P.a2[i]));
        hh_step(f[i][0], f[i][1], vn[i][0], vn[i][1], P, ikT, w4);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NUM; ++i) {
    const double en = P.m0 * vn[i][0] * vn[i][0] + P.m1 * vn[i][1] * vn[i][1];
    const double sc = sqrt(P.kT / en);
    vn[i][0] *= sc;
    vn[i][1] *= sc;
  }
  return scale;
}

// one thread per (state, chunk); eout[t] = {ekin, ekinNHC (x2), potNHC} at
// the time of get_fictKE; scale[t] = {s2, s1}
template <int NUM>
__global__ void k_nhc_update(Par P, const double* __restrict__ part, int nsplit, int nstates,
                             int first_in, const int* __restrict__ skip,
                             double* __restrict__ x, double* __restrict__ xp,
                             double* __restrict__ vn, double* __restrict__ scale,
                             double* __restrict__ eout) {
  const int first = first_in && !(skip && *skip);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nstates * P.nck) return;
  const int s = t / P.nck, k = t % P.nck;
  double ekin = 0.0;
  for (int q = 0; q < nsplit; ++q) ekin += part[((size_t)s * nsplit + q) * P.nck + k];
  double xl[NUM][2], xpl[NUM][2], vl[NUM][2];
  const size_t o = (size_t)t * NUM * 2;
#pragma unroll
  for (int i = 0; i < NUM; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      xl[i][j] = x[o + 2 * i + j];
      xpl[i][j] = xp[o + 2 * i + j];
      vl[i][j] = vn[o + 2 * i + j];
    }
  double s2 = 1.0;
  if (first) {
    s2 = iso_update<NUM>(ekin, P.gkt[k], P, xl, xpl, vl);
    ekin *= s2 * s2;
  }
  double ekn = 0.0, pot = 0.0;
#pragma unroll
  for (int i = 0; i < NUM; ++i) {
    ekn += P.m0 * vl[i][0] * vl[i][0] + P.m1 * vl[i][1] * vl[i][1];
    pot += xl[i][0] + xl[i][1];
  }
  eout[3 * t] = ekin;
  eout[3 * t + 1] = ekn;
  eout[3 * t + 2] = pot;
  const double s1 = iso_update<NUM>(ekin, P.gkt[k], P, xl, xpl, vl);
#pragma unroll
  for (int i = 0; i < NUM; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      x[o + 2 * i + j] = xl[i][j];
      xp[o + 2 * i + j] = xpl[i][j];
      vn[o + 2 * i + j] = vl[i][j];
    }
  scale[2 * t] = s2;
  scale[2 * t + 1] = s1;
}

// fict KE, NHC kinetic energy and NHC potential, summed in a fixed order
__global__ void k_nhc_sum(const double* __restrict__ eout, int n, double* __restrict__ fict,
                          double* __restrict__ enhc) {
  __shared__ double red[32];
  double a = 0.0, b = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    a += eout[3 * i];
    b += eout[3 * i + 1];
    c += eout[3 * i + 2];
  }
  a = block_sum(a, red);
  b = block_sum(b, red);
  c = block_sum(c, red);
  if (threadIdx.x == 0) {
    if (fict) *fict = 0.5 * a;
    if (enhc) {
      enhc[0] = 0.5 * b;
      enhc[1] = c;
    }
  }
}

// grid (point blocks, states): U points per thread, all loads issued first
__global__ void __launch_bounds__(256, 3) k_nhc_apply(double2* __restrict__ psi, double2* __restrict__ v,
                            const double2* __restrict__ f, const double* __restrict__ cmass,
                            const int* __restrict__ cls, const signed char* __restrict__ ck,
                            const double* __restrict__ scale, int nck, int npts, int nstates,
                            double dt, int first_in, const int* __restrict__ skip) {
  constexpr int U = 4;
  const int first = first_in && !(skip && *skip);
  const double dt2 = 0.5 * dt;
  const int s = blockIdx.y;
  const int B = blockDim.x;
  const int pb = blockIdx.x * U * B + threadIdx.x;
  const size_t row = (size_t)s * npts;
  const double2* sc2 = reinterpret_cast<const double2*>(scale) + (size_t)s * nck;
  int c[U];
  double2 vv[U], ff[U], a[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int p = pb + u * B;
    c[u] = p < npts ? cls[p] : 0;
    if (c[u]) {
      vv[u] = v[row + p];
      ff[u] = f[row + p];
      a[u] = psi[row + p];
    }
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (c[u] == 0) continue;
    const int p = pb + u * B;
    const double2 sc = sc2[ck[p]];
    const double fm = dt2 / cmass[p];
    double2 w = vv[u], g = ff[u];
    if (c[u] == 1) { w.y = 0.0; g.y = 0.0; }
    if (first) {
      w.x += g.x * fm;
      w.y += g.y * fm;
      if (c[u] == 1) w.y = 0.0;
      w.x *= sc.x;
      w.y *= sc.x;
    }
    w.x *= sc.y;
    w.y *= sc.y;
    w.x += g.x * fm;
    w.y += g.y * fm;
    if (c[u] == 1) w.y = 0.0;
    v[row + p] = w;
    a[u].x += w.x * dt;
    a[u].y += w.y * dt;
    psi[row + p] = a[u];
  }
}

// set_yosh (cp_isokin.C:320-388), unscaled
void yosh(int nyosh, double* w) {
  switch (nyosh) {
    case 1: w[0] = 1.0; break;
    case 3: {
      const double t = std::pow(2.0, 1.0 / 3.0);
      w[0] = 1.0 / (2.0 - t); w[1] = -t / (2.0 - t); w[2] = 1.0 / (2.0 - t);
      break;
    }
    case 5: {
      const double p2 = 1.0 / (4.0 - std::pow(4.0, 1.0 / 3.0));
      w[0] = w[1] = w[3] = w[4] = p2; w[2] = 1.0 - 4.0 * p2;
      break;
    }
    case 7:
      w[0] = w[6] = 0.784513610477560;
      w[1] = w[5] = 0.235573213359357;
      w[2] = w[4] = -1.17767998417887;
      w[3] = 1.0 - 2.0 * (w[0] + w[1] + w[2]);
      break;
    default:  // 9
      w[0] = w[8] = 0.192;
      w[1] = w[7] = 0.554910818409783619692725006662999;
      w[2] = w[6] = 0.124659619941888644216504240951585;
      w[3] = w[5] = -0.843182063596933505315033808282941;
      w[4] = 1.0 - 2.0 * (w[0] + w[1] + w[2] + w[3]);
      break;
  }
}

}  // namespace nhc

void nhc_yosh(int nyosh, double* w) { nhc::yosh(nyosh, w); }

void nhc_free(cpstep_ctx* c) {
  CpNhc& t = c->nhc;
  cudaFree(t.d_ck); cudaFree(t.d_x); cudaFree(t.d_xp); cudaFree(t.d_vn);
  cudaFree(t.d_part); cudaFree(t.d_scale); cudaFree(t.d_eout);
  t = CpNhc();
}

// initCPNHC (cp_isokin.C:45-141) for every state, the chunk map in chare
// order, and the default chain state x = xp = 0, v = (sqrt(kT/m0), 0).
int nhc_set(cpstep_ctx* c, double te_ext, double tau_fs, int num, int nck, int nres, int nyosh) {
  nhc_free(c);
  if (!(te_ext > 0.0)) return CPSTEP_OK;  // thermostat off
  if (num < 1 || num > nhc::kMaxNum || nck < 1 || nck > nhc::kMaxNck || nres < 1 ||
      !(nyosh == 1 || nyosh == 3 || nyosh == 5 || nyosh == 7 || nyosh == 9) || !(tau_fs > 0.0)) {
    cpstep_set_error("set_cp_thermostat: num in 1..%d, nck in 1..%d, nres >= 1, "
                     "nyosh in {1,3,5,7,9}, tau > 0", nhc::kMaxNum, nhc::kMaxNck);
    return CPSTEP_ERR_ARG;
  }
  const int np = c->npts;
  std::vector<int> cls(np);
  CPSTEP_CUDA_TRY(cudaMemcpy(cls.data(), c->d_cls, sizeof(int) * np, cudaMemcpyDeviceToHost));
  std::vector<int> order;
  for (int want = 1; want <= 3; ++want)
    for (int p = 0; p < np; ++p)
      if (cls[p] == want) order.push_back(p);
  const int ncoef = (int)order.size();
  int nzero = 0;
  for (int p = 0; p < np; ++p) nzero += cls[p] == 1;
  if (nck > ncoef) {
    cpstep_set_error("set_cp_thermostat: %d chunks for %d coefficients", nck, ncoef);
    return CPSTEP_ERR_ARG;
  }
  CpNhc& t = c->nhc;
  // t.on is published last: a failed allocation or copy leaves the thermostat
  // off (the buffers made so far are released by the next nhc_free)
  t.num = num; t.nck = nck; t.nres = nres; t.nyosh = nyosh;
  const double kT = te_ext / 315777.0, tau = tau_fs / 0.0241888;  // BOLTZ, TIME_CONV
  const double degfree = (double)(2 * ncoef - nzero), pre = tau * tau * kT;
  t.kT = kT;
  t.m[0] = pre * degfree / nck;
  t.m[1] = 2.5 * pre;
  for (int i = 0; i < num; ++i) {
    const double frac = (double)(num + i + 5) / (double)(num + 5);
    t.v0[i] = 0.8 * kT * frac;
    t.a2[i] = 1.6 * (0.8 * frac);
    t.a4[i] = t.a2[i] * t.a2[i];
  }
  std::vector<signed char> ck(np, -1);
  const int div = ncoef / nck, rem = ncoef % nck;
  for (int k = 0; k < nck; ++k) {
    const int nstr = div * k + (k >= rem ? rem : k), nnow = div + (k < rem ? 1 : 0);
    for (int i = nstr; i < nstr + nnow; ++i) ck[order[i]] = (signed char)k;
    t.dfs[k] = 2.0 * nnow - (k == 0 ? nzero : 0);
  }
  const size_t nch = (size_t)c->nstates * nck * num * 2;
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_ck, np));
  CPSTEP_CUDA_TRY(cudaMemcpy(t.d_ck, ck.data(), np, cudaMemcpyHostToDevice));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_x, sizeof(double) * nch));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_xp, sizeof(double) * nch));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_vn, sizeof(double) * nch));
  std::vector<double> zero(nch, 0.0), vn(nch, 0.0);
  for (size_t q = 0; q < nch; q += 2) vn[q] = std::sqrt(kT / t.m[0]);
  CPSTEP_CUDA_TRY(cudaMemcpy(t.d_x, zero.data(), sizeof(double) * nch, cudaMemcpyHostToDevice));
  CPSTEP_CUDA_TRY(cudaMemcpy(t.d_xp, zero.data(), sizeof(double) * nch, cudaMemcpyHostToDevice));
  CPSTEP_CUDA_TRY(cudaMemcpy(t.d_vn, vn.data(), sizeof(double) * nch, cudaMemcpyHostToDevice));
  // enough (state, span) blocks for two waves; spans of whole 256-point rows
  // one wave of (state, span) blocks at 8 blocks of 256 threads per SM
  t.nsplit = std::max(1, std::min((np + 255) / 256, (8 * c->num_sms) / c->nstates));
  t.span = (np + t.nsplit - 1) / t.nsplit;
  t.nsplit = (np + t.span - 1) / t.span;
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_part, sizeof(double) * (size_t)c->nstates * t.nsplit * nck));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_scale, sizeof(double) * 2 * (size_t)c->nstates * nck));
  CPSTEP_CUDA_TRY(cudaMalloc(&t.d_eout, sizeof(double) * 3 * (size_t)c->nstates * nck));
  t.on = 1;
  return CPSTEP_OK;
}

int nhc_state(cpstep_ctx* c, int set, double* h_x, double* h_xp, double* h_vn) {
  CpNhc& t = c->nhc;
  if (!t.on) {
    cpstep_set_error("cp_thermostat_state: the thermostat is off");
    return CPSTEP_ERR_STATE;
  }
  const size_t b = sizeof(double) * (size_t)c->nstates * t.nck * t.num * 2;
  double* d[3] = {t.d_x, t.d_xp, t.d_vn};
  double* h[3] = {h_x, h_xp, h_vn};
  for (int q = 0; q < 3; ++q) {
    if (!h[q]) continue;
    if (set)
      CPSTEP_CUDA_TRY(cudaMemcpyAsync(d[q], h[q], b, cudaMemcpyHostToDevice, c->stream));
    else
      CPSTEP_CUDA_TRY(cudaMemcpyAsync(h[q], d[q], b, cudaMemcpyDeviceToHost, c->stream));
  }
  CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CPSTEP_OK;
}

int nhc_integrate(cpstep_ctx* c, const double* force, double* psi, double* vpsi, double dt,
                  int iteration, double* d_fict_ke, double* d_enhc, const int* d_skip_half) {
  CpNhc& t = c->nhc;
  nhc::Par P;
  P.num = t.num; P.nck = t.nck; P.nres = t.nres; P.nyosh = t.nyosh;
  P.kT = t.kT; P.m0 = t.m[0]; P.m1 = t.m[1];
  for (int i = 0; i < nhc::kMaxNum; ++i) {
    P.a2[i] = t.a2[i];
    P.c1[i] = i < t.num ? -(4.0 * t.v0[i] / (t.a4[i] * t.m[1])) : 0.0;
  }
  for (int k = 0; k < nhc::kMaxNck; ++k) P.gkt[k] = t.dfs[k] * t.kT;
  double w[9] = {0};
  nhc::yosh(t.nyosh, w);
  for (int i = 0; i < 9; ++i) P.w[i] = w[i] * (dt / t.nres);
  const int first = iteration > 1 ? 1 : 0;
  double2* p = reinterpret_cast<double2*>(psi);
  double2* v = reinterpret_cast<double2*>(vpsi);
  const double2* f = reinterpret_cast<const double2*>(force);
  nhc::k_nhc_ekin<<<dim3(t.nsplit, c->nstates), 256, 0, c->stream>>>(
      v, f, c->d_cmass, c->d_cls, t.d_ck, c->npts, t.span, dt, first, d_skip_half, t.nck,
      t.d_part);
  CPSTEP_LAUNCH_CHECK();
  const int nt = c->nstates * t.nck;
  const dim3 ug((nt + 31) / 32), ub(32);
#define NHC_UPDATE(N)                                                                        \
  nhc::k_nhc_update<N><<<ug, ub, 0, c->stream>>>(P, t.d_part, t.nsplit, c->nstates, first,  \
                                                 d_skip_half, t.d_x, t.d_xp, t.d_vn, t.d_scale, t.d_eout)
  switch (t.num) {
    case 1: NHC_UPDATE(1); break;
    case 2: NHC_UPDATE(2); break;
    case 3: NHC_UPDATE(3); break;
    case 4: NHC_UPDATE(4); break;
    case 5: NHC_UPDATE(5); break;
    case 6: NHC_UPDATE(6); break;
    case 7: NHC_UPDATE(7); break;
    default: NHC_UPDATE(8); break;
  }
#undef NHC_UPDATE
  CPSTEP_LAUNCH_CHECK();
  if (d_fict_ke || d_enhc) {
    nhc::k_nhc_sum<<<1, 256, 0, c->stream>>>(t.d_eout, nt, d_fict_ke, d_enhc);
    CPSTEP_LAUNCH_CHECK();
  }
  nhc::k_nhc_apply<<<dim3(cdiv(c->npts, 4 * 256), c->nstates), 256, 0, c->stream>>>(
      p, v, f, c->d_cmass, c->d_cls, t.d_ck,
                                                       t.d_scale, t.nck, c->npts, c->nstates,
                                                       dt, first, d_skip_half);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}
