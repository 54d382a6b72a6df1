// EES non-local pseudopotential (Euler exponential spline, Kleinman-Bylander
// s and p channels) for every state on one GPU.
//
//   set-up                       eesSetEesWghtGgrp / get_bspline_wght1d / eesSplProjectorGgrp
//                                (src_piny_physics_v1.0/abinito_physics/cp_nonlocal/
//                                cp_ees_nonlocal.C:60-240, interface/cp_ewald/set_cp_ewald.C:1237-1322)
//   atom B-splines               eesAtmBsplineRgrp  cp_ees_nonlocal.C:256-580
//   projector x psi, NL G->R     eesProjGchare / eesYlmOnD :594-1236, doNlFFTGtoR (fftCache.C)
//   Z matrix, energy, forces     eesZmatRchare :1238-1346, eesEnergyAtmForcRchare :1480-1700
//   scatter, NL R->G, psi force  eesEnergyAtmForcRchare, doNlFFTRtoG, eesPsiForcGspace :2000-2064
//
// The reference runs one (state, channel) per chare pair with the NL grid
// split into planes; here one channel at a time runs for all states: K1 with
// the projector (conj(dyp psi)), a plane kernel that finishes the G->R
// transform in shared memory and forms each atom's per-plane sums, a small
// kernel for Z, E_NL, the atom forces and the scaled Z, a plane kernel that
// scatters Z Mn and starts the R->G transform, and K4 adding the psi force.
// The projector dyp depends on the cell only and is formed once at set-up.
#include <algorithm>
#include <cmath>
#include <vector>
#include "ctx.cuh"
#include "tc_sm100.cuh"

namespace ees {

// eesAtmBsplineRgrp I-III for one atom and axis: grid indices, M_n and dM_n.
__global__ void k_nl_bspline(const double* __restrict__ frac, int natm, int nkf,
                             int* __restrict__ ig, double* __restrict__ mn,
                             double* __restrict__ dmn) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natm) return;
  constexpr int n_interp = kNlInterp;
  const double grid = (double)nkf;
  for (int d = 0; d < 3; ++d) {
    double t = frac[3 * a + d];
    const double xm = t - 0.5;
    t -= (double)(int)(xm >= 0.0 ? xm + 0.5 : xm - 0.5);  // NINT, SIMP_NINT form
    t = (t == 1.0) ? 0.0 : t;
    t = t * grid;
    const int it = (int)t;
    const double fr = t - (double)it;
    double u[n_interp], m[n_interp], dm[n_interp];
    int* igo = ig + ((size_t)a * 3 + d) * n_interp;
#pragma unroll
    for (int j = 1; j <= n_interp; ++j) {
      u[j - 1] = fr + (double)(j - 1);
      int idx = it - (j - 2);
      idx = (idx > 0) ? idx : nkf + idx;
      idx = (idx <= nkf) ? idx : idx - nkf;
      igo[j - 1] = min(max(idx, 1), nkf) - 1;  // in [1, nkf] already; kept as a bound
      m[j - 1] = 0.0;
      dm[j - 1] = 0.0;
    }
    m[0] = 1.0 - fabs(u[0] - 1.0);
    m[1] = 1.0 - fabs(u[1] - 1.0);
#pragma unroll
    for (int n = 3; n <= n_interp; ++n) {
      const double rn = (double)n, rn1 = 1.0 / (double)(n - 1);
#pragma unroll
      for (int j = n; j >= 2; --j) m[j - 1] = (u[j - 1] * m[j - 1] + (rn - u[j - 1]) * m[j - 2]) * rn1;
      m[0] = u[0] * m[0] * rn1;
      if (n == n_interp - 1) {
        dm[0] = m[0];
#pragma unroll
        for (int j = 2; j <= n_interp; ++j) dm[j - 1] = m[j - 1] - m[j - 2];
      }
    }
    double* mo = mn + ((size_t)a * 3 + d) * n_interp;
    double* dmo = dmn + ((size_t)a * 3 + d) * n_interp;
#pragma unroll
    for (int j = 0; j < n_interp; ++j) {
      mo[j] = m[j];
      dmo[j] = dm[j];
    }
  }
}

// Per (type, plane) lists of the atoms with an interpolation plane there, in
// atom order (so the scatter of the R->G kernel adds in a fixed order).
// One warp per (type, plane): 32 atoms per step, ballot + prefix count keep
// the atom order.
__global__ void k_nl_planes(const int* __restrict__ typ, const int* __restrict__ ig, int natm,
                            int ntyp, int nkf, int* __restrict__ plist,
                            int* __restrict__ pcount) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= ntyp * nkf) return;
  const int t = i / nkf, z = i - t * nkf;
  int* out = plist + (size_t)i * natm;
  int n = 0;
  for (int a0 = 0; a0 < natm; a0 += 32) {
    const int a = a0 + lane;
    int jc = -1;
    if (a < natm && typ[a] == t) {
      const int* c = ig + ((size_t)a * 3 + 2) * kNlInterp;
#pragma unroll
      for (int k = 0; k < kNlInterp; ++k)
        if (c[k] == z) jc = k;
    }
    const unsigned m = __ballot_sync(0xffffffffu, jc >= 0);
    if (jc >= 0) out[n + __popc(m & ((1u << lane) - 1u))] = a | (jc << 16);
    n += __popc(m);
  }
  if (lane == 0) pcount[i] = n;
}

// Stencil tables of one (type, plane) (NlAtoms): for every atom slot e of the
// plane's list and point q = jb*8 + ja, its cell and nl_point's products;
// then the gather list that lets the R->G kernel form each touched cell's
// sum of Z Mn with one thread per cell, adding the atoms in list order as a
// serial scatter would.  One block per (plane, type); shared memory: two ints
// per plane cell (counts, then fill cursors).
constexpr int TABTHREADS = 256;
}  // namespace ees
constexpr int kNlGridMax = 160;
namespace ees {
struct TabDims {
  int cap[CPSTEP_MAX_TYPES];
  long long off[CPSTEP_MAX_TYPES];
};
__global__ void __launch_bounds__(TABTHREADS)
k_nl_table(NlAtoms A, int nkf, TabDims d, int* __restrict__ tcell, NlVal* __restrict__ tval,
           int* __restrict__ gcell, int* __restrict__ goff, int* __restrict__ gent,
           int* __restrict__ gcount) {
  extern __shared__ int tab_smem[];
  const int z = blockIdx.x, t = blockIdx.y;
  const int ncell = nkf * nkf;
  int* cnt = tab_smem;           // [ncell]
  int* cur = tab_smem + ncell;   // [ncell]
  const int cap = d.cap[t];
  const size_t base = (size_t)d.off[t] + (size_t)z * cap;
  const size_t gbase = (size_t)d.off[t] + (size_t)t * nkf + (size_t)z * (cap + 1);
  const int* pl = A.plist + ((size_t)t * nkf + z) * A.natm;
  const int npl = A.pcount[t * nkf + z];
  for (int i = threadIdx.x; i < ncell; i += TABTHREADS) cnt[i] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < npl * 64; i += TABTHREADS) {
    const int e = i >> 6, q = i & 63, ja = q & 7, jb = q >> 3;
    const int a = pl[e] & 0xffff, jc = pl[e] >> 16;
    const int* ig = A.ig + (size_t)a * 3 * kNlInterp;
    const int cell = ig[kNlInterp + jb] * nkf + ig[ja];
    NlVal v;
    nl_point(A, a, ja, jb, jc, v.mn, v.dx, v.dy, v.dz);
    tcell[base + i] = cell;
    tval[base + i] = v;
    atomicAdd(&cnt[cell], 1);
  }
  __syncthreads();
  // compact the touched cells in increasing order: each thread a contiguous
  // range of cells, then a block scan of (touched cells, entries)
  __shared__ int wsum_c[TABTHREADS / 32], wsum_e[TABTHREADS / 32];
  const int per = (ncell + TABTHREADS - 1) / TABTHREADS;
  const int c0 = threadIdx.x * per, c1 = min(ncell, c0 + per);
  int nc = 0, ne = 0;
  for (int c = c0; c < c1; ++c) {
    nc += cnt[c] > 0;
    ne += cnt[c];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int ic = nc, ie = ne;  // inclusive warp scans
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int uc = __shfl_up_sync(0xffffffffu, ic, o), ue = __shfl_up_sync(0xffffffffu, ie, o);
    if (lane >= o) {
      ic += uc;
      ie += ue;
    }
  }
  if (lane == 31) {
    wsum_c[warp] = ic;
    wsum_e[warp] = ie;
  }
  __syncthreads();
  int pc = ic - nc, pe = ie - ne;  // exclusive within the warp
  for (int w = 0; w < warp; ++w) {
    pc += wsum_c[w];
    pe += wsum_e[w];
  }
  for (int c = c0; c < c1; ++c) {
    const int k = cnt[c];
    if (k > 0) {
      gcell[base + pc] = c;
      goff[gbase + pc] = pe;
      cur[c] = pe;
      ++pc;
      pe += k;
    }
  }
  if (threadIdx.x == TABTHREADS - 1) {
    gcount[t * nkf + z] = pc;
    goff[gbase + pc] = pe;  // = npl * 64
  }
  __syncthreads();
  // entries in atom-slot order: an atom's 64 cells are distinct
  for (int e = 0; e < npl; ++e) {
    if (threadIdx.x < 64) {
      const int i = e * 64 + threadIdx.x;
      const int cell = tcell[base + i];
      gent[base + cur[cell]] = i;
      cur[cell] += 1;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// G-space evaluation of the same sums (mixed contexts, tensor cores).  With
// F(r) the C2R transform of proj = conj(dyp psi), Parseval turns the grid sums
// of an atom's stencil into sums over the packed points:
//   sum_r M(r) F(r) = sum_p wpt_p Re(proj(p) S(p)),   S(p) = s_a(kx) s_b(ky) s_c(kz),
//   s_d(k) = sum_j M_d[j] exp(-2 pi i k ig_d[j] / nkf)
// (the B-spline factors of eesAtmBsplineRgrp), and the scatter + R2C of the
// psi force into pg(p) = sum_atoms zs conj(S(p)).  The dMn sums take the
// derivative factors in one axis at a time, combined with hmati as nl_point
// does.

// separable transforms [atom][axis][Mn, dMn][k + km], k in [-km, km]
__global__ void k_ees_sep(const int* __restrict__ ig, const double* __restrict__ mn,
                          const double* __restrict__ dmn, int natm, int nkf, int km,
                          double2* __restrict__ sep) {
  const int nk = 2 * km + 1;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)natm * 6 * nk) return;
  const int kk = (int)(i % nk);
  const long long rest = i / nk;
  const int m = (int)(rest % 2), d = (int)((rest / 2) % 3), a = (int)(rest / 6);
  const int k = kk - km;
  const int* g = ig + ((size_t)a * 3 + d) * kNlInterp;
  const double* f = (m ? dmn : mn) + ((size_t)a * 3 + d) * kNlInterp;
  double re = 0.0, im = 0.0;
#pragma unroll
  for (int j = 0; j < kNlInterp; ++j) {
    long long t = ((long long)k * g[j]) % nkf;
    if (t < 0) t += nkf;
    double sn, cs;
    sincospi(2.0 * (double)t / (double)nkf, &sn, &cs);
    re += f[j] * cs;
    im -= f[j] * sn;
  }
  sep[i] = make_double2(re, im);
}

struct TypeDims {
  int tstart[CPSTEP_MAX_TYPES + 1];
  long long svoff[CPSTEP_MAX_TYPES];
  long long tsoff[CPSTEP_MAX_TYPES];  // first S row of the type in tsc / tinv
  long long bloff[CPSTEP_MAX_TYPES];  // byte offset of the type's S-row levels
};

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Bounds of |S| of the rows (v, a) of every atom from the per-axis maxima of
// its separable transforms: |S| is their product, the gradient rows are
// bounded by the triangle inequality.  tsc = pow2_scale(bound) scales the
// row's FP16 levels, tinv = 1 / tsc; smax[t] gets the largest Mn-row bound of
// the type (float bits of a non-negative value, atomicMax).  One warp per atom.
__global__ void k_ees_bound(const double2* __restrict__ sep, int natm, int km,
                            const int* __restrict__ typ, const int* __restrict__ rank,
                            TypeDims td, NlAtoms A, float* __restrict__ tsc,
                            float* __restrict__ tinv, unsigned int* __restrict__ smax) {
  const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (a >= natm) return;
  const int nk = 2 * km + 1;
  const double2* T = sep + (size_t)a * 6 * nk;
  double m[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double mx = 0.0;
    for (int k = lane; k < nk; k += 32) {
      const double2 v = T[q * nk + k];
      mx = fmax(mx, hypot(v.x, v.y));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    m[q] = mx;
  }
  if (lane == 0) {
    const int t = typ[a];
    const int nt = td.tstart[t + 1] - td.tstart[t], al = rank[a] - td.tstart[t];
    double b[4];
    b[0] = m[0] * m[2] * m[4];
    const double* h = A.hmati;
    for (int v = 0; v < 3; ++v) {
      const double h0 = fabs(h[3 * v] * A.grid), h1 = fabs(h[3 * v + 1] * A.grid),
                   h2 = fabs(h[3 * v + 2] * A.grid);
      b[v + 1] = m[1] * m[2] * m[4] * h0 + m[0] * m[3] * m[4] * h1 + m[0] * m[2] * m[5] * h2;
    }
    for (int v = 0; v < 4; ++v) {
      const float sc = tc::pow2_scale((float)b[v]);
      tsc[td.tsoff[t] + v * nt + al] = sc;
      tinv[td.tsoff[t] + v * nt + al] = 1.f / sc;
    }
    atomicMax(smax + t, __float_as_uint((float)b[0]));
  }
}

// S matrices, 4 points per thread: the Mn rows in FP32 (row a of the type, for
// the psi force) and every row (v natm_t + a, v = Mn, d/dx, d/dy, d/dz) as
// scaled FP16 levels in the pre-split image (nsp K steps per 128-row tile)
// for the sums.  Lane i of a warp is the atom of type-order rank 8 y + (i & 7)
// (y = blockIdx.y) at point quad (i >> 3) of the warp: the 8 atoms' 16-byte
// pieces of a K half are one 128-byte core matrix when their rows are 8-aligned.
__global__ void __launch_bounds__(256) k_ees_smat(
    const double2* __restrict__ sep, const int* __restrict__ kx, const int* __restrict__ ky,
    const int* __restrict__ kz, int npts, int km, const int* __restrict__ typ,
    const int* __restrict__ order, int natm, TypeDims td, NlAtoms A, long long ld_s,
    float* __restrict__ sv, const float* __restrict__ tsc, uint8_t* __restrict__ blv, int nsp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ra = blockIdx.y * 8 + (lane & 7);
  const int p0 = 4 * ((blockIdx.x * 8 + warp) * 4 + (lane >> 3));
  if (ra >= natm || p0 >= npts) return;
  const int a = order[ra];
  const int t = typ[a];
  const int nt = td.tstart[t + 1] - td.tstart[t], al = ra - td.tstart[t];
  const int nk = 2 * km + 1;
  const double2* T = sep + (size_t)a * 6 * nk;
  const double* h = A.hmati;
  const double g = A.grid;
  float lv[4][8];
  float* base = sv + td.svoff[t] + (size_t)al * ld_s;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int p = p0 + e;
    if (p < npts) {
      const int ix = kx[p] + km, iy = ky[p] + km, iz = kz[p] + km;
      const double2 sa = T[0 * nk + ix], da = T[1 * nk + ix];
      const double2 sb = T[2 * nk + iy], db = T[3 * nk + iy];
      const double2 sc = T[4 * nk + iz], dc = T[5 * nk + iz];
      const double2 sbc = cm(sb, sc);
      const double2 S = cm(sa, sbc);
      const double2 at = cm(da, sbc), bt = cm(sa, cm(db, sc)), ct = cm(cm(sa, sb), dc);
      lv[0][2 * e] = (float)S.x;
      lv[0][2 * e + 1] = (float)S.y;
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        const double h0 = h[3 * v] * g, h1 = h[3 * v + 1] * g, h2 = h[3 * v + 2] * g;
        lv[v + 1][2 * e] = (float)(at.x * h0 + bt.x * h1 + ct.x * h2);
        lv[v + 1][2 * e + 1] = (float)(at.y * h0 + bt.y * h1 + ct.y * h2);
      }
    } else {
#pragma unroll
      for (int v = 0; v < 4; ++v) lv[v][2 * e] = lv[v][2 * e + 1] = 0.f;
    }
  }
  if (p0 + 3 < npts) {
    *reinterpret_cast<float4*>(base + 2 * p0) = make_float4(lv[0][0], lv[0][1], lv[0][2], lv[0][3]);
    *reinterpret_cast<float4*>(base + 2 * p0 + 4) =
        make_float4(lv[0][4], lv[0][5], lv[0][6], lv[0][7]);
  } else {
    for (int e = 0; p0 + e < npts; ++e)
      reinterpret_cast<float2*>(base)[p0 + e] = make_float2(lv[0][2 * e], lv[0][2 * e + 1]);
  }
  // reals 2 p0 .. 2 p0 + 7: K step p0 / 8, half (p0 / 4) & 1
  uint8_t* bt0 = blv + td.bloff[t];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int j = v * nt + al;
    tc::split_store_h(bt0 + ((size_t)(j >> 7) * nsp + (p0 >> 3)) * (2 * tc::CM_TILE) +
                          tc::core_off(j & 127, 8 * ((p0 >> 2) & 1)),
                      lv[v], tsc[td.tsoff[t] + j]);
  }
}

// Z, E_NL, scaled Z and atom forces of one type from its G-space sums
// C(s, ch jp + v nt + a) (column-major, ld = nstates): as k_nl_zmat.
__global__ void k_ees_zglue(const double* __restrict__ C, int nstates, int nt, int nch,
                            const int* __restrict__ chan, const double* __restrict__ vnc,
                            const int* __restrict__ order, int t0, int natm,
                            const double* __restrict__ occ, double* __restrict__ zt, int ldz,
                            double* __restrict__ enl_s, double* __restrict__ fnl,
                            unsigned int* __restrict__ zmax) {
  __shared__ double red[32];
  const int s = blockIdx.x;
  const double w = occ[s];
  const int jp = 4 * nt;
  double e = 0.0;
  float zm = 0.f;  // largest |scaled Z| (float bits into *zmax, as k_ees_smat)
  for (int al = threadIdx.x; al < nt; al += blockDim.x) {
    const int atom = order[t0 + al];
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    for (int ch = 0; ch < nch; ++ch) {
      const double vn = vnc[chan[ch]];
      const double* cc = C + ((size_t)ch * jp + al) * nstates + s;
      const double z = cc[0];
      const double dx = cc[(size_t)nt * nstates], dy = cc[(size_t)2 * nt * nstates];
      const double dz = cc[(size_t)3 * nt * nstates];
      e += z * z * vn * w;
      const double zsc = z * (2.0 * vn * w);
      zt[(size_t)s * ldz + ch * nt + al] = zsc;
      zm = fmaxf(zm, (float)fabs(zsc));
      f0 -= dx * zsc;
      f1 -= dy * zsc;
      f2 -= dz * zsc;
    }
    double* f = fnl + ((size_t)s * natm + atom) * 3;
    f[0] += f0;
    f[1] += f1;
    f[2] += f2;
  }
  for (int o = 16; o > 0; o >>= 1) zm = fmaxf(zm, __shfl_xor_sync(0xffffffffu, zm, o));
  if ((threadIdx.x & 31) == 0 && zm > 0.f) atomicMax(zmax, __float_as_uint(zm));
  e = block_sum(e, red);
  if (threadIdx.x == 0) enl_s[s] += e;
}

// Z_a = sum over the atom's planes, E_NL += Z^2 vn occ, Z <- 2 vn occ Z,
// F_a -= Z sum P dMn (eesEnergyAtmForcRchare :1545-1560, :1596-1600).
// One block per state; atoms of the channel's type.
__global__ void k_nl_zmat(const double* __restrict__ zpart, NlAtoms A, int ctype, double vn,
                          const double* __restrict__ occ, double* __restrict__ zs,
                          double* __restrict__ enl_s, double* __restrict__ fnl) {
  __shared__ double red[32];
  const int s = blockIdx.x;
  const double w = occ[s];
  double e = 0.0;
  for (int a = threadIdx.x; a < A.natm; a += blockDim.x) {
    if (A.typ[a] != ctype) continue;
    const double* zp = zpart + ((size_t)s * A.natm + a) * kNlInterp * 4;
    double z = 0.0, dx = 0.0, dy = 0.0, dz = 0.0;
#pragma unroll
    for (int jc = 0; jc < kNlInterp; ++jc) {
      z += zp[4 * jc];
      dx += zp[4 * jc + 1];
      dy += zp[4 * jc + 2];
      dz += zp[4 * jc + 3];
    }
    e += z * z * vn * w;
    const double zsc = z * (2.0 * vn * w);
    zs[(size_t)s * A.natm + a] = zsc;
    double* f = fnl + ((size_t)s * A.natm + a) * 3;
    f[0] -= dx * zsc;
    f[1] -= dy * zsc;
    f[2] -= dz * zsc;
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) enl_s[s] += e;
}

// energies[E_NL] = sum_s enl_s[s]; fatm[a][k] += sum_s fnl[s][a][k] (fixed order)
__global__ void k_nl_finish(const double* __restrict__ enl_s, const double* __restrict__ fnl,
                            int nstates, int natm, double* __restrict__ energies,
                            double* __restrict__ fatm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && energies) {
    double e = 0.0;
    for (int s = 0; s < nstates; ++s) e += enl_s[s];
    energies[CPSTEP_E_NL] = e;
  }
  if (fatm && i < 3 * natm) {
    double f = 0.0;
    for (int s = 0; s < nstates; ++s) f += fnl[(size_t)s * 3 * natm + i];
    fatm[i] += f;
  }
}

}  // namespace ees

// ===========================================================================
// host side

namespace {

// get_bspline_wght1d (set_cp_ewald.C:1237-1322): the complex 1/b(m) factors
// for m = 0 .. ngrid-1 of the order-n_interp cardinal B-spline.
void bspline_wght1d(int n_interp, int ngrid, std::vector<double>& br, std::vector<double>& bi) {
  std::vector<double> mnk(n_interp + 1, 0.0), uk(n_interp + 1, 0.0);
  mnk[1] = 1.0;
  uk[1] = 1.0;
  for (int k = 2; k <= n_interp; ++k) uk[k] = (double)k;
  for (int n = 3; n <= n_interp; ++n) {
    const double rn = (double)n, rn1 = 1.0 / (double)(n - 1);
    for (int k = n; k >= 2; --k) mnk[k] = (uk[k] * mnk[k] + (rn - uk[k]) * mnk[k - 1]) * rn1;
    mnk[1] = uk[1] * mnk[1] * rn1;
  }
  const double grid = (double)ngrid;
  const double tpi_n = 2.0 * M_PI / grid;
  br.assign(ngrid, 0.0);
  bi.assign(ngrid, 0.0);
  for (int m = 0; m < ngrid; ++m) {
    double r = 0.0, i = 0.0;
    for (int k = 1; k <= n_interp - 1; ++k) {
      const double arg = tpi_n * (double)((k - 1) * m);
      r += cos(arg) * mnk[k];
      i += sin(arg) * mnk[k];
    }
    const double arg = 2.0 * M_PI * (double)(n_interp - 1) / grid * (double)m;
    const double nr = cos(arg), ni = sin(arg);
    const double den = r * r + i * i;
    br[m] = (nr * r + ni * i) / den;
    bi[m] = (ni * r - nr * i) / den;
  }
}

template <typename T>
int upload_tw_n(int n, void** dst) {
  std::vector<cplx<T>> h(n);
  for (int m = 0; m < n; ++m) {
    double a = -2.0 * M_PI * (double)m / (double)n;
    h[m] = mk<T>((T)cos(a), (T)sin(a));
  }
  CPSTEP_CUDA_TRY(cudaMalloc(dst, sizeof(cplx<T>) * n));
  CPSTEP_CUDA_TRY(cudaMemcpy(*dst, h.data(), sizeof(cplx<T>) * n, cudaMemcpyHostToDevice));
  return CPSTEP_OK;
}

int wrap(int v, int n) { return v < 0 ? v + n : v; }

}  // namespace

void ees_bspline_weights(int n_interp, int ngrid, std::vector<double>& br,
                         std::vector<double>& bi) {
  bspline_wght1d(n_interp, ngrid, br, bi);
}

int ees_bspline_launch(cpstep_ctx* c, const double* frac, int natm, int nkf, int* ig, double* mn,
                       double* dmn) {
  ees::k_nl_bspline<<<cdiv(natm, 128), 128, 0, c->stream>>>(frac, natm, nkf, ig, mn, dmn);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

void nl_free(cpstep_ctx* c) {
  NlData& n = c->nl;
  cudaFree(n.dyp); cudaFree(n.line_zneg); cudaFree(n.line_zpos); cudaFree(n.line_xy);
  cudaFree(n.pen_a); cudaFree(n.pen_b); cudaFree(n.tw); cudaFree(n.ig); cudaFree(n.mn);
  cudaFree(n.dmn); cudaFree(n.zpart); cudaFree(n.zs); cudaFree(n.enl_s); cudaFree(n.fnl);
  cudaFree(n.tcell); cudaFree(n.tval); cudaFree(n.gcell); cudaFree(n.goff); cudaFree(n.gent);
  cudaFree(n.gcount);
  cudaFree(n.sep); cudaFree(n.sv); cudaFree(n.d_order); cudaFree(n.d_tch); cudaFree(n.d_vn);
  cudaFree(n.csum); cudaFree(n.zt);
  for (auto d : n.tdyp) cudaFree(d);
  n.tdyp.clear();
  cudaFree(n.d_hmax);
  n.d_hmax = nullptr;
  cudaFree(n.blv);
  cudaFree(n.tsc);
  cudaFree(n.tinv);
  cudaFree(n.alv);
  cudaFree(n.pf_z);
  cudaFree(n.pf_st);
  n.pf_z = n.pf_st = nullptr;
  n.pf_zbytes = n.pf_stbytes = 0;
  n.blv = n.alv = nullptr;
  n.tsc = n.tinv = nullptr;
  n.alv_bytes = 0;
  n.sep = nullptr; n.sv = nullptr; n.d_order = nullptr; n.d_tch = nullptr; n.d_vn = nullptr;
  n.csum = nullptr; n.zt = nullptr; n.gspace_ok = 0;
  cudaFree(n.plist); cudaFree(n.pcount);
  n = NlData();
}

int nl_set(cpstep_ctx* c, int nkf, int n_interp, int nchan, const int* ch_type, const int* ch_l,
           const int* ch_m, const double* vnl, const double* gz0, const double* vnorm) {
  const AtomData& at = c->atoms;
  if (at.natm <= 0) {
    cpstep_set_error("set_nonlocal: call cpstep_set_atoms first");
    return CPSTEP_ERR_STATE;
  }
  if (n_interp != kNlInterp || nkf < n_interp || nchan <= 0) {
    cpstep_set_error("set_nonlocal: n_interp must be %d, nkf >= n_interp, nchan > 0", kNlInterp);
    return CPSTEP_ERR_ARG;
  }
  if (nkf > kNlGridMax) {  // the stencil-table kernel keeps two ints per plane cell in shared memory
    cpstep_set_error("set_nonlocal: NL grid %d above %d", nkf, kNlGridMax);
    return CPSTEP_ERR_ARG;
  }
  for (int k = 0; k < nchan; ++k) {
    if (ch_type[k] < 0 || ch_type[k] >= at.ntyp || ch_l[k] < 0 || ch_l[k] > 1 ||
        ch_m[k] < -ch_l[k] || ch_m[k] > ch_l[k]) {
      cpstep_set_error("set_nonlocal: channel %d (type %d, l %d, m %d) not supported (s, p)", k,
                       ch_type[k], ch_l[k], ch_m[k]);
      return CPSTEP_ERR_ARG;
    }
  }
  // the state sphere must fit the NL grid: |k| < nkf / 2 on every axis
  int km = 0;
  for (int p = 0; p < c->npts; ++p)
    km = std::max(km, std::max(std::abs(c->h_kx[p]), std::max(std::abs(c->h_ky[p]),
                                                               std::abs(c->h_kz[p]))));
  if (2 * km >= nkf) {
    cpstep_set_error("set_nonlocal: NL grid %d too small for |k| <= %d", nkf, km);
    return CPSTEP_ERR_ARG;
  }
  StateFftOps ops;
  if (!statefft_lookup(c->precision, nkf, &ops)) {
    cpstep_set_error("set_nonlocal: NL grid size %d not built into libcpstep", nkf);
    return CPSTEP_ERR_ARG;
  }
  if (ops.nl_smem(c->nplane_x) > 227 * 1024) {
    cpstep_set_error("set_nonlocal: NL plane of %d x %d does not fit shared memory in this "
                     "precision", nkf, nkf);
    return CPSTEP_ERR_ARG;
  }
  nl_free(c);
  sf_free(c);  // the structure-factor path and this one exclude each other
  NlData& n = c->nl;
  n.nkf = nkf;
  n.nchan = nchan;
  n.ops = ops;
  n.natm = at.natm;
  n.ch_type.assign(ch_type, ch_type + nchan);
  n.ch_vn.resize(nchan);
  for (int k = 0; k < nchan; ++k) n.ch_vn[k] = vnorm[k] / c->vol;
  // NL-grid line tables from the state lines
  const int nl = c->nlines;
  std::vector<int> zneg(nl), zpos(nl), xy(nl);
  for (int l = 0; l < nl; ++l) {
    const int off = c->h_line_off[l];
    const int end = (l + 1 < nl) ? c->h_line_off[l + 1] : c->npts;
    int nneg = 0;
    while (off + nneg < end && c->h_kz[off + nneg] < 0) ++nneg;
    zneg[l] = nneg > 0 ? wrap(c->h_kz[off], nkf) : 0;
    zpos[l] = (off + nneg < end) ? wrap(c->h_kz[off + nneg], nkf) : 0;
    xy[l] = wrap(c->h_kx[off], nkf) | (wrap(c->h_ky[off], nkf) << 16);
  }
  auto up = [&](int** d, const std::vector<int>& h) -> int {
    CPSTEP_CUDA_TRY(cudaMalloc(d, sizeof(int) * h.size()));
    CPSTEP_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
    return CPSTEP_OK;
  };
  int rc;
  if ((rc = up(&n.line_zneg, zneg)) || (rc = up(&n.line_zpos, zpos)) || (rc = up(&n.line_xy, xy)))
    return rc;
  // projector dyp per channel and point (eesSetEesWghtGgrp, eesYlmOnD, eesProjGchare)
  std::vector<double> br, bi;
  bspline_wght1d(n_interp, nkf, br, bi);
  const double fpi = 4.0 * M_PI;
  const double y00 = 1.0 / sqrt(fpi), y10 = sqrt(3.0 / fpi), y11 = sqrt(1.5 / fpi) * sqrt(2.0);
  const double* h = c->hmati;
  const double tpi = 2.0 * M_PI;
  std::vector<double2> dyp((size_t)nchan * c->npts);
  for (int p = 0; p < c->npts; ++p) {
    const int ka = c->h_kx[p], kb = c->h_ky[p], kc = c->h_kz[p];
    const int ia = wrap(ka, nkf), ib = wrap(kb, nkf), ic = wrap(kc, nkf);
    double abr = br[ia] * br[ib] - bi[ia] * bi[ib];
    double abi = bi[ia] * br[ib] + br[ia] * bi[ib];
    double dre = abr * br[ic] - abi * bi[ic];
    double dim = abi * br[ic] + abr * bi[ic];
    const bool g0 = (ka == 0 && kb == 0 && kc == 0);
    if (g0) {
      dre = br[0] * br[0] * br[0];
      dim = 0.0;
    }
    const double xk = (ka * h[0] + kb * h[1] + kc * h[2]) * tpi;
    const double yk = (ka * h[3] + kb * h[4] + kc * h[5]) * tpi;
    const double zk = (ka * h[6] + kb * h[7] + kc * h[8]) * tpi;
    const double g = sqrt(xk * xk + yk * yk + zk * zk);
    int iii = (int)((g - at.gmin) / at.dg + 1.0);
    iii = std::min(iii, at.nspl);
    iii = std::max(iii, 1);
    double hh = g - ((double)(iii - 1) * at.dg + at.gmin);
    if (g < 1.0e-12) {
      hh = 0.0;
      iii = 1;
    }
    for (int k = 0; k < nchan; ++k) {
      double yr, yi;
      if (ch_l[k] == 0) {
        yr = dre * y00;
        yi = dim * y00;
      } else if (g != 0.0) {
        double y;
        if (ch_m[k] == 0) {
          y = y10 * (zk / g);
        } else {
          const double gs = sqrt(xk * xk + yk * yk);
          const double ph = (ch_m[k] == 1) ? (gs == 0.0 ? 1.0 : xk / gs)
                                           : (gs == 0.0 ? 0.0 : yk / gs);
          y = y11 * (gs / g) * ph;
        }
        yr = -dim * y;
        yi = dre * y;
      } else {
        yr = yi = 0.0;
      }
      double2 v;
      if (g0) {
        v = (ch_l[k] == 0) ? make_double2(yr * gz0[k], 0.0) : make_double2(0.0, 0.0);
      } else {
        const double* t = vnl + (size_t)k * 4 * at.nspl + (iii - 1);
        const double vnow =
            ((t[3 * at.nspl] * hh + t[2 * at.nspl]) * hh + t[at.nspl]) * hh + t[0];
        v = make_double2(yr * vnow, yi * vnow);
      }
      dyp[(size_t)k * c->npts + p] = v;
    }
  }
  CPSTEP_CUDA_TRY(cudaMalloc(&n.dyp, sizeof(double2) * dyp.size()));
  CPSTEP_CUDA_TRY(cudaMemcpy(n.dyp, dyp.data(), sizeof(double2) * dyp.size(),
                             cudaMemcpyHostToDevice));
  const bool fp64 = c->precision == CPSTEP_PREC_FP64;
  if ((rc = fp64 ? upload_tw_n<double>(nkf, &n.tw) : upload_tw_n<float>(nkf, &n.tw))) return rc;
  const size_t csz = fp64 ? sizeof(cplx<double>) : sizeof(cplx<float>);
  const size_t pen = (size_t)c->nstates * nkf * c->nlpad * csz;
  CPSTEP_CUDA_TRY(cudaMalloc(&n.pen_a, pen));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.pen_b, pen));
  const size_t na = (size_t)at.natm;
  CPSTEP_CUDA_TRY(cudaMalloc(&n.ig, sizeof(int) * na * 3 * kNlInterp));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.mn, sizeof(double) * na * 3 * kNlInterp));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.dmn, sizeof(double) * na * 3 * kNlInterp));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.plist, sizeof(int) * (size_t)at.ntyp * nkf * na));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.pcount, sizeof(int) * (size_t)at.ntyp * nkf));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.zpart, sizeof(double) * c->nstates * na * kNlInterp * 4));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.zs, sizeof(double) * c->nstates * na));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.enl_s, sizeof(double) * c->nstates));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.fnl, sizeof(double) * c->nstates * na * 3));
  // stencil tables: 64 entries per atom of the type on each plane at most
  n.tab_cap.assign(at.ntyp, 0);
  n.tab_off.assign(at.ntyp, 0);
  size_t tot = 0;
  for (int t = 0; t < at.ntyp; ++t) {
    n.tab_off[t] = tot;
    n.tab_cap[t] = 64 * (at.tstart[t + 1] - at.tstart[t]);
    tot += (size_t)nkf * n.tab_cap[t];
  }
  const size_t tot1 = std::max<size_t>(tot, 1);
  CPSTEP_CUDA_TRY(cudaMalloc(&n.tcell, sizeof(int) * tot1));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.tval, sizeof(NlVal) * tot1));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.gcell, sizeof(int) * tot1));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.gent, sizeof(int) * tot1));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.goff, sizeof(int) * (tot + (size_t)at.ntyp * nkf)));
  CPSTEP_CUDA_TRY(cudaMalloc(&n.gcount, sizeof(int) * (size_t)at.ntyp * nkf));
  // G-space form (mixed contexts): channels per type, S matrices, scratch
  n.km = km;
  n.tch.assign(at.ntyp, {});
  for (int k = 0; k < nchan; ++k) n.tch[ch_type[k]].push_back(k);
  n.gspace_ok = c->precision == CPSTEP_PREC_MIXED;
  for (int t = 0; t < at.ntyp; ++t) n.gspace_ok = n.gspace_ok && n.tch[t].size() <= 4;
  if (n.gspace_ok) {
    n.ld_s = (long long)((2 * (size_t)c->npts + 3) / 4 * 4);
    n.sv_off.assign(at.ntyp, 0);
    long long tot = 0;
    size_t csz = 1, zsz = 1;
    for (int t = 0; t < at.ntyp; ++t) {
      const int nt = at.tstart[t + 1] - at.tstart[t];
      n.sv_off[t] = tot;
      tot += 4LL * nt * n.ld_s;
      csz = std::max(csz, (size_t)n.tch[t].size() * 4 * nt * c->nstates);
      zsz = std::max(zsz, (size_t)c->nstates * (((size_t)n.tch[t].size() * nt + 1) / 2 * 2));
    }
    CPSTEP_CUDA_TRY(cudaMalloc(&n.sv, sizeof(float) * (size_t)std::max(tot, 4LL)));
    CPSTEP_CUDA_TRY(cudaMemset(n.sv, 0, sizeof(float) * (size_t)std::max(tot, 4LL)));
    CPSTEP_CUDA_TRY(cudaMalloc(&n.sep, sizeof(double2) * na * 6 * (2 * (size_t)km + 1)));
    CPSTEP_CUDA_TRY(cudaMalloc(&n.csum, sizeof(double) * csz));
    n.zt_slot = zsz;  // two types at a time
    CPSTEP_CUDA_TRY(cudaMalloc(&n.zt, sizeof(double) * 2 * zsz));
    n.tdyp.assign(at.ntyp, nullptr);
    n.tdmax.assign(at.ntyp, 0.f);
    n.tdmax_c.assign(at.ntyp, std::vector<float>(4, 0.f));
    n.ld_d32 = (c->npts + 1) / 2 * 2;
    CPSTEP_CUDA_TRY(cudaMalloc(&n.d_hmax, sizeof(float) * 2 * std::max(1, at.ntyp)));
    std::vector<int> htch((size_t)at.ntyp * 4, -1);
    for (int t = 0; t < at.ntyp; ++t) {
      const size_t nc = n.tch[t].size();
      if (!nc) continue;
      // FP32 copies, rows padded to an even number of points (16-byte rows)
      const size_t ld = n.ld_d32;
      CPSTEP_CUDA_TRY(cudaMalloc(&n.tdyp[t], sizeof(float2) * nc * ld));
      std::vector<double2> hd(c->npts);
      std::vector<float2> hf(nc * ld, make_float2(0.f, 0.f));
      for (size_t k = 0; k < nc; ++k) {
        htch[(size_t)t * 4 + k] = n.tch[t][k];
        CPSTEP_CUDA_TRY(cudaMemcpy(hd.data(), n.dyp + (size_t)n.tch[t][k] * c->npts,
                                   sizeof(double2) * c->npts, cudaMemcpyDeviceToHost));
        for (int q = 0; q < c->npts; ++q) {
          hf[k * ld + q] = make_float2((float)hd[q].x, (float)hd[q].y);
          n.tdmax[t] = std::max(n.tdmax[t], (float)std::hypot(hd[q].x, hd[q].y));
          n.tdmax_c[t][k] = std::max(n.tdmax_c[t][k], (float)std::hypot(hd[q].x, hd[q].y));
        }
      }
      CPSTEP_CUDA_TRY(cudaMemcpy(n.tdyp[t], hf.data(), sizeof(float2) * nc * ld,
                                 cudaMemcpyHostToDevice));
    }
    // FP16 levels of the S rows (zero past each type's rows and past K, never
    // written there), their scales, and the A operand of the sums
    {
      const int K = 2 * c->npts;
      n.blv_off.assign(at.ntyp, 0);
      n.tsoff.assign(at.ntyp, 0);
      size_t bl = 0;
      long long ts = 0;
      int nchmax = 1;
      for (int t = 0; t < at.ntyp; ++t) {
        const int nt = at.tstart[t + 1] - at.tstart[t];
        n.blv_off[t] = bl;
        n.tsoff[t] = ts;
        bl += ees_lv_bytes(std::max(1, 4 * nt), K);
        ts += 4LL * nt;
        nchmax = std::max(nchmax, (int)n.tch[t].size());
      }
      CPSTEP_CUDA_TRY(cudaMalloc(&n.blv, bl));
      CPSTEP_CUDA_TRY(cudaMemset(n.blv, 0, bl));
      CPSTEP_CUDA_TRY(cudaMalloc(&n.tsc, sizeof(float) * (size_t)std::max(1LL, ts)));
      CPSTEP_CUDA_TRY(cudaMalloc(&n.tinv, sizeof(float) * (size_t)std::max(1LL, ts)));
      n.alv_bytes = ees_lv_bytes(nchmax * c->nstates, K);  // per type; two types at a time
      CPSTEP_CUDA_TRY(cudaMalloc(&n.alv, 2 * n.alv_bytes));
      int ntmax = 1;
      for (int t = 0; t < at.ntyp; ++t) ntmax = std::max(ntmax, at.tstart[t + 1] - at.tstart[t]);
      n.pf_zbytes = ees_pf_zbytes(c->nstates, ntmax);
      n.pf_stbytes = ees_pf_stbytes(c->npts, ntmax);
      CPSTEP_CUDA_TRY(cudaMalloc(&n.pf_z, 2 * n.pf_zbytes));  // two types at a time
      CPSTEP_CUDA_TRY(cudaMalloc(&n.pf_st, 2 * n.pf_stbytes));
    }
    CPSTEP_CUDA_TRY(cudaMalloc(&n.d_tch, sizeof(int) * htch.size()));
    CPSTEP_CUDA_TRY(cudaMemcpy(n.d_tch, htch.data(), sizeof(int) * htch.size(),
                               cudaMemcpyHostToDevice));
    CPSTEP_CUDA_TRY(cudaMalloc(&n.d_vn, sizeof(double) * nchan));
    CPSTEP_CUDA_TRY(cudaMemcpy(n.d_vn, n.ch_vn.data(), sizeof(double) * nchan,
                               cudaMemcpyHostToDevice));
    std::vector<int> hrank(na), horder(na);
    CPSTEP_CUDA_TRY(cudaMemcpy(hrank.data(), at.rank, sizeof(int) * na, cudaMemcpyDeviceToHost));
    for (int a = 0; a < (int)na; ++a) horder[hrank[a]] = a;
    CPSTEP_CUDA_TRY(cudaMalloc(&n.d_order, sizeof(int) * na));
    CPSTEP_CUDA_TRY(cudaMemcpy(n.d_order, horder.data(), sizeof(int) * na,
                               cudaMemcpyHostToDevice));
  }
  n.on = 1;
  return CPSTEP_OK;
}

// The EES pass in G space (see k_ees_sep): per type, the forward sums as one
// tensor-core product of psi with conj(dyp) S, the glue, and the psi force as
// one back-multiply with the same matrix.
static int ees_gspace_run(cpstep_ctx* c, const double* psi, const double* occ, double* fpsi,
                          double* energies, double* fatm) {
  NlData& n = c->nl;
  const int S = c->nstates, natm = n.natm, ntyp = c->atoms.ntyp;
  ees::k_nl_bspline<<<cdiv(natm, 128), 128, 0, c->stream>>>(c->atoms.frac, natm, n.nkf, n.ig,
                                                            n.mn, n.dmn);
  CPSTEP_LAUNCH_CHECK();
  const long long nsep = (long long)natm * 6 * (2 * n.km + 1);
  ees::k_ees_sep<<<(unsigned)((nsep + 255) / 256), 256, 0, c->stream>>>(n.ig, n.mn, n.dmn, natm,
                                                                         n.nkf, n.km, n.sep);
  CPSTEP_LAUNCH_CHECK();
  ees::TypeDims td{};
  for (int t = 0; t <= ntyp; ++t) td.tstart[t] = c->atoms.tstart[t];
  for (int t = 0; t < ntyp; ++t) {
    td.svoff[t] = n.sv_off[t];
    td.tsoff[t] = n.tsoff[t];
    td.bloff[t] = (long long)n.blv_off[t];
  }
  NlAtoms A{};
  for (int k = 0; k < 9; ++k) A.hmati[k] = c->hmati[k];
  A.grid = (double)n.nkf;
  // bounds of |S| (the FP16 scales of the S rows' levels) and the largest |Z|
  // entry per type (the psi force's)
  CPSTEP_CUDA_TRY(cudaMemsetAsync(n.d_hmax, 0, sizeof(float) * 2 * ntyp, c->stream));
  unsigned int* smax_u = reinterpret_cast<unsigned int*>(n.d_hmax);
  unsigned int* zmax_u = smax_u + ntyp;
  ees::k_ees_bound<<<cdiv(32 * natm, 256), 256, 0, c->stream>>>(
      n.sep, natm, n.km, c->atoms.typ, c->atoms.rank, td, A, n.tsc, n.tinv, smax_u);
  CPSTEP_LAUNCH_CHECK();
  const int nsp_s = cdiv(2 * c->npts, 32) * 2;  // K steps of a pre-split row tile
  ees::k_ees_smat<<<dim3(cdiv(c->npts, 128), cdiv(natm, 8)), 256, 0, c->stream>>>(
      n.sep, c->d_kx, c->d_ky, c->d_kz, c->npts, n.km, c->atoms.typ, n.d_order, natm, td, A,
      n.ld_s, n.sv, n.tsc, n.blv, nsp_s);
  CPSTEP_LAUNCH_CHECK();
  CPSTEP_CUDA_TRY(cudaMemsetAsync(n.enl_s, 0, sizeof(double) * S, c->stream));
  CPSTEP_CUDA_TRY(cudaMemsetAsync(n.fnl, 0, sizeof(double) * S * natm * 3, c->stream));
  // the types with projectors, two at a time: A of both split from one read of psi
  std::vector<int> tl;
  EesForceType ft[2];
  for (int t = 0; t < ntyp; ++t)
    if (!n.tch[t].empty() && c->atoms.tstart[t + 1] > c->atoms.tstart[t]) tl.push_back(t);
  for (size_t q = 0; q < tl.size(); ++q) {
    const int t = tl[q];
    const int nch = (int)n.tch[t].size();
    const int nt = c->atoms.tstart[t + 1] - c->atoms.tstart[t];
    uint8_t* alv = n.alv + (q & 1) * n.alv_bytes;
    if (q % 2 == 0) {
      const int np2 = q + 1 < tl.size() ? 2 : 1;
      const float2* dy[2];
      const float* dm[2];
      int nc[2];
      uint8_t* al[2] = {n.alv, n.alv + n.alv_bytes};
      for (int k = 0; k < np2; ++k) {
        dy[k] = n.tdyp[tl[q + k]];
        dm[k] = n.tdmax_c[tl[q + k]].data();
        nc[k] = (int)n.tch[tl[q + k]].size();
      }
      if (int rc = ees_tc_presplit_a(c, psi, np2, dy, n.ld_d32, nc, dm, al, n.alv_bytes)) return rc;
    }
    if (int rc = ees_tc_sums_pre(c, nch, n.tdmax_c[t].data(), n.blv + n.blv_off[t], 4 * nt,
                                 n.tinv + n.tsoff[t], alv, n.csum))
      return rc;
    const int ldz = (nch * nt + 1) / 2 * 2;
    double* zt = n.zt + (q & 1) * n.zt_slot;
    ees::k_ees_zglue<<<S, 128, 0, c->stream>>>(n.csum, S, nt, nch, n.d_tch + 4 * t, n.d_vn,
                                                n.d_order, c->atoms.tstart[t], natm, occ, zt, ldz,
                                                n.enl_s, n.fnl, zmax_u + t);
    CPSTEP_LAUNCH_CHECK();
    ft[q & 1] = EesForceType{n.sv + n.sv_off[t], n.ld_s, n.tdyp[t], nch, nt, zt, ldz,
                             n.d_hmax + t, n.d_hmax + ntyp + t, n.pf_z + (q & 1) * n.pf_zbytes,
                             n.pf_st + (q & 1) * n.pf_stbytes};
    // the psi force of the pair (F read and written once for both types)
    if (q % 2 == 1 || q + 1 == tl.size())
      if (int rc = ees_tc_force_pre(c, (int)(q % 2) + 1, ft, n.ld_d32, -1.0, fpsi, n.pf_zbytes,
                                    n.pf_stbytes))
        return rc;
  }
  ees::k_nl_finish<<<cdiv(std::max(1, 3 * natm), 128), 128, 0, c->stream>>>(
      n.enl_s, n.fnl, S, natm, energies, fatm);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

int nl_run(cpstep_ctx* c, const double* psi, const double* occ, double* fpsi, double* energies,
           double* fatm) {
  NlData& n = c->nl;
  if (!n.on) {
    cpstep_set_error("ees_nonlocal: call cpstep_set_nonlocal first");
    return CPSTEP_ERR_STATE;
  }
  if (n.natm != c->atoms.natm) {
    cpstep_set_error("ees_nonlocal: atoms changed since cpstep_set_nonlocal");
    return CPSTEP_ERR_STATE;
  }
  if (n.gspace_ok && c->precision == CPSTEP_PREC_MIXED && c->tc_ok && c->tune.ees_gspace)
    return ees_gspace_run(c, psi, occ, fpsi, energies, fatm);
  const int S = c->nstates, natm = n.natm;
  ees::k_nl_bspline<<<cdiv(natm, 128), 128, 0, c->stream>>>(c->atoms.frac, natm, n.nkf, n.ig,
                                                            n.mn, n.dmn);
  CPSTEP_LAUNCH_CHECK();
  const int ntyp = c->atoms.ntyp;
  ees::k_nl_planes<<<cdiv(ntyp * n.nkf, 8), 256, 0, c->stream>>>(c->atoms.typ, n.ig, natm, ntyp,
                                                                  n.nkf, n.plist, n.pcount);
  CPSTEP_LAUNCH_CHECK();
  CPSTEP_CUDA_TRY(cudaMemsetAsync(n.enl_s, 0, sizeof(double) * S, c->stream));
  CPSTEP_CUDA_TRY(cudaMemsetAsync(n.fnl, 0, sizeof(double) * S * natm * 3, c->stream));
  NlJob j;
  j.f.g = c->geom();
  j.f.g.nx = j.f.g.ny = j.f.g.nz = n.nkf;
  j.f.g.line_zneg = n.line_zneg;
  j.f.g.line_zpos = n.line_zpos;
  j.f.g.line_xy = n.line_xy;
  j.f.pen_a = n.pen_a;
  j.f.pen_b = n.pen_b;
  j.tw = n.tw;
  j.A.natm = natm;
  j.A.typ = c->atoms.typ;
  j.A.ig = n.ig;
  j.A.mn = n.mn;
  j.A.dmn = n.dmn;
  for (int k = 0; k < 9; ++k) j.A.hmati[k] = c->hmati[k];
  j.A.grid = (double)n.nkf;
  j.A.plist = n.plist;
  j.A.pcount = n.pcount;
  {
    ees::TabDims d{};
    for (int t = 0; t < ntyp; ++t) {
      d.cap[t] = n.tab_cap[t];
      d.off[t] = (long long)n.tab_off[t];
    }
    const int tsm = (int)(2 * sizeof(int) * (size_t)n.nkf * n.nkf);
    CPSTEP_CUDA_TRY(cudaFuncSetAttribute(ees::k_nl_table,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, tsm));
    ees::k_nl_table<<<dim3(n.nkf, ntyp), ees::TABTHREADS, tsm, c->stream>>>(
        j.A, n.nkf, d, n.tcell, n.tval, n.gcell, n.goff, n.gent, n.gcount);
    CPSTEP_LAUNCH_CHECK();
  }
  const int zt = std::min(1024, std::max(32, cdiv(natm, 32) * 32));
  for (int k = 0; k < n.nchan; ++k) {
    j.ctype = n.ch_type[k];
    const int t = j.ctype;
    j.A.tcap = n.tab_cap[t];
    j.A.tcell = n.tcell + n.tab_off[t];
    j.A.tval = n.tval + n.tab_off[t];
    j.A.gcell = n.gcell + n.tab_off[t];
    j.A.gent = n.gent + n.tab_off[t];
    j.A.goff = n.goff + n.tab_off[t] + (size_t)t * n.nkf;
    j.A.gcount = n.gcount + (size_t)t * n.nkf;
    const double2* dyp = n.dyp + (size_t)k * c->npts;
    int rc;
    if ((rc = n.ops.nl_proj(c, j, psi, dyp, S, n.zpart))) return rc;
    ees::k_nl_zmat<<<S, zt, 0, c->stream>>>(n.zpart, j.A, j.ctype, n.ch_vn[k], occ, n.zs,
                                            n.enl_s, n.fnl);
    CPSTEP_LAUNCH_CHECK();
    if ((rc = n.ops.nl_force(c, j, n.zs, dyp, S, fpsi))) return rc;
  }
  ees::k_nl_finish<<<cdiv(std::max(1, 3 * natm), 128), 128, 0, c->stream>>>(
      n.enl_s, n.fnl, S, natm, energies, fatm);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}
