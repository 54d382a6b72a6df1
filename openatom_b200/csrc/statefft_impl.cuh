// State FFT pipeline for a cubic grid of compile-time size N:
//   packed psi(G) -> z-pencils -> xy planes -> rho(r)
//   V_KS(r).psi(r) -> xy planes -> z-pencils -> packed F(G) (+ kinetic term)
//
// Reference steps (OpenAtom, src_charm_driver/):
//   expandGSpace / z-FFT           fft_slab_ctrl/fftCache.C:460-507, :1133-1159
//   transpose to planes            cp_state_ctrl/CP_State_GSpacePlane.C:1473-1498,
//                                  cp_state_ctrl/CP_State_RealSpacePlane.C:248-268
//   y-FFT, imag flip, x C2R        fft_slab_ctrl/fftCache.C:1167-1243
//   occ*psi^2 and the reduction    cp_state_ctrl/CP_State_RealSpacePlane.C:349-355, :484-500
//   psi*V_KS*occ                   cp_state_ctrl/CP_State_RealSpacePlane.C:580-587
//   x R2C, imag flip, y-FFT        fft_slab_ctrl/fftCache.C:1252-1319
//   z-FFT, packGSpace, -2/N scale  fft_slab_ctrl/fftCache.C:1099-1123, :517-553,
//                                  cp_state_ctrl/CP_State_GSpacePlane.C:1605-1612
//   addForces (x2 off Gx=0)        fft_slab_ctrl/stateSlab.C:240-272
//   CP_eke_calc                    src_piny_physics_v1.0/abinito_physics/cp_nonlocal/cp_eke.C:30-140
//
// On one GPU the Charm++ transposes become the [state][z][line] pencil layout:
// the z-pass writes, for every z, the contiguous run of its lines, and the
// plane pass reads one contiguous row of nlines values per (state, z).  psi(r)
// is never stored: the V.psi pass recomputes it from the pencils, which hold
// 2*nlines*N reals per state against N^3 for psi(r).
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>
#include "ctx.cuh"
#include "fft_shfl.cuh"
#include "fft_p16.cuh"
#include "fft_t20.cuh"

namespace sfft {

constexpr int ZTHREADS = 256;  // z passes: 8 warps, each owns whole z-lines
constexpr int PTHREADS = 512;  // plane passes: 16 warps
constexpr int PWARPS = PTHREADS / 32;

// packed point p -> (line index within the batch, z) by binary search over the
// batch's line offsets held in shared memory.
__device__ __forceinline__ void locate(int p, const int* soff, int nl, const int* snneg,
                                       const int* szneg, const int* szpos, int& li, int& z) {
  int lo = 0, hi = nl - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (soff[mid] <= p) lo = mid; else hi = mid - 1;
  }
  li = lo;
  int q = p - soff[lo];
  z = (q < snneg[lo]) ? szneg[lo] + q : szpos[lo] + (q - snneg[lo]);
}

template <int N>
struct PlaneLd;

template <int N>
struct ZShape {
  static constexpr int LB = std::min(64, std::max(8, 4096 / N));  // lines per block
  static constexpr int LD = PlaneLd<N>::value;
  template <typename T>
  static constexpr size_t bytes() {
    return sizeof(cplx<T>) * (size_t)(N + LB * LD) + sizeof(int) * (4 * LB + 1);
  }
};

// Line stride of the plane columns and row buffers: room for the padded
// stage-1 output of the two-stage warp FFT where N = 16 * M2, else N + 1.
template <int N>
struct PlaneLd {
  static constexpr int value = Fft16Shape<N>::ok ? Fft16Shape<N>::LD : N + 1;
  static constexpr int lines = Fft16Shape<N>::ok ? Fft16Shape<N>::L : 1;  // per warp pass
};

// nl lines of length N at base (stride ld) by the calling warp, up to
// PlaneLd<N>::lines at a time.
// (FP64 keeps the one-line-at-a-time Stockham FFT: the two-stage form needs
// more than the 128 registers a thread of the 512-thread plane kernels has.)
template <typename T, int N, bool INV>
__device__ __forceinline__ void warp_lines(cplx<T>* base, int ld, int nl, const cplx<T>* tw) {
  if constexpr (Fft16Shape<N>::ok && sizeof(T) == 4) {
    constexpr int L = Fft16Shape<N>::L;
    const int lane = threadIdx.x & 31;
    for (int l0 = 0; l0 < nl; l0 += L)
      fft16_lines<T, N, INV>(base + (size_t)l0 * ld, ld, min(L, nl - l0), tw, lane);
  } else {
    for (int l = 0; l < nl; ++l) fft_line_warp<T, N, INV>(base + (size_t)l * ld, tw);
  }
}

// nl lines (stride ld) shared out to all warps of the block in groups.
template <typename T, int N, bool INV>
__device__ __forceinline__ void block_lines(cplx<T>* buf, int ld, int nl, const cplx<T>* tw) {
  constexpr int L = PlaneLd<N>::lines;
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int l0 = warp * L; l0 < nl; l0 += nw * L)
    warp_lines<T, N, INV>(buf + (size_t)l0 * ld, ld, min(L, nl - l0), tw);
}

// Lines c = grp, grp + ngrp, ... (stride ldy) through dif (DIF: natural in,
// permuted out, see shfl_perm) or dit (permuted in, natural out), in place.
template <typename T, int N, bool INV, bool DIF>
__device__ __forceinline__ void shfl_columns(cplx<T>* plane, int ldy, int nplx,
                                             const ShflFft<T, N>& F, const cplx<T>* tw,
                                             int grp, int ngrp) {
  constexpr int NL = ShflCfg<N>::NL, M = ShflCfg<N>::M;
  for (int c0 = 0; c0 < nplx; c0 += ngrp) {
    const int c = c0 + grp;
    const bool act = c < nplx;
    cplx<T> v[M];
    cplx<T>* col = plane + (size_t)(act ? c : 0) * ldy;
#pragma unroll
    for (int k = 0; k < M; ++k) v[k] = act ? col[F.l + NL * k] : mk<T>(0, 0);
    if (DIF) F.template dif<INV>(v, tw); else F.template dit<INV>(v, tw);
    if (act) {
#pragma unroll
      for (int k = 0; k < M; ++k) col[F.l + NL * k] = v[k];
    }
  }
}

// ---------------------------------------------------------------------------
// K1: expand packed psi into z-lines, forward z-FFT, write [s][z][line] pencils
// With mul (EES projector dyp), the line holds conj(mul * psi) instead of psi
// (eesProjGchare, cp_ees_nonlocal.C:705-709).
template <typename T, int N>
__global__ void __launch_bounds__(ZTHREADS)
k_zfft_fwd(const double2* __restrict__ psi, cplx<T>* __restrict__ pen, StateGeom g,
           const cplx<T>* __restrict__ twz, const double2* __restrict__ mul) {
  constexpr int LB = ZShape<N>::LB, LD = ZShape<N>::LD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* buf = tw + N;
  int* soff = reinterpret_cast<int*>(buf + LB * LD);
  int* snneg = soff + LB + 1;
  int* szneg = snneg + LB;
  int* szpos = szneg + LB;
  const int s = blockIdx.y;
  const int l0 = blockIdx.x * LB;
  const int nl = min(LB, g.nlines - l0);
  for (int i = threadIdx.x; i < N; i += ZTHREADS) tw[i] = twz[i];
  for (int i = threadIdx.x; i < LB * LD; i += ZTHREADS) buf[i] = mk<T>(0, 0);
  for (int i = threadIdx.x; i < nl; i += ZTHREADS) {
    soff[i] = g.line_off[l0 + i];
    snneg[i] = g.line_nneg[l0 + i];
    szneg[i] = g.line_zneg[l0 + i];
    szpos[i] = g.line_zpos[l0 + i];
  }
  if (threadIdx.x == 0) soff[nl] = (l0 + nl < g.nlines) ? g.line_off[l0 + nl] : g.npts;
  __syncthreads();
  const int p0 = soff[0], p1 = soff[nl];
  const double2* ps = psi + (size_t)s * g.npts;
  for (int p = p0 + threadIdx.x; p < p1; p += ZTHREADS) {
    int li, z;
    locate(p, soff, nl, snneg, szneg, szpos, li, z);
    double2 v = ps[p];
    if (mul) {
      double2 d = mul[p];
      v = make_double2(d.x * v.x - d.y * v.y, -(d.y * v.x + d.x * v.y));
    }
    buf[li * LD + z] = mk<T>((T)v.x, (T)v.y);
  }
  __syncthreads();
  if constexpr (ShflCfg<N>::ok) {
    ShflFft<T, N> F;
    F.init(tw);
    shfl_columns<T, N, false, true>(buf, LD, nl, F, tw, threadIdx.x / ShflCfg<N>::NL,
                                    ZTHREADS / ShflCfg<N>::NL);  // FFTW_FORWARD along z
  } else {
    block_lines<T, N, false>(buf, LD, nl, tw);  // FFTW_FORWARD along z
  }
  __syncthreads();
  cplx<T>* po = pen + (size_t)s * N * g.nlpad + l0;
  for (int i = threadIdx.x; i < nl * N; i += ZTHREADS) {
    int z = i / nl, li = i - z * nl;
    po[(size_t)z * g.nlpad + li] = buf[li * LD + (ShflCfg<N>::ok ? shfl_perm<N>(z) : z)];
  }
}

// ---------------------------------------------------------------------------
// shared plane helpers.  plane is [nplane_x][LDY] (column kx holds y contiguous)

// The nplx plane columns, shared out to the block's warps in groups.
template <typename T, int N, bool INV>
__device__ __forceinline__ void plane_columns(cplx<T>* plane, int nplx, const cplx<T>* tw) {
  block_lines<T, N, INV>(plane, PlaneLd<N>::value, nplx, tw);
}

template <typename T, int N>
__device__ __forceinline__ void scatter_plane(const cplx<T>* __restrict__ prow, cplx<T>* plane,
                                              const StateGeom& g) {
  constexpr int LDY = PlaneLd<N>::value;
  for (int i = threadIdx.x; i < g.nplane_x * LDY; i += blockDim.x) plane[i] = mk<T>(0, 0);
  __syncthreads();
  for (int l = threadIdx.x; l < g.nlines; l += blockDim.x) {
    int xy = __ldg(g.line_xy + l);
    plane[(xy & 0xffff) * LDY + (xy >> 16)] = prow[l];
  }
  __syncthreads();
}

// The calling warp builds Z = Xa + i Xb for the C2R of rows (ya, ya+1) from the
// y-transformed plane: the reference's imag flip (conj), the Hermitian
// extension to kx > N/2, zero outside the nplane_x columns.
template <typename T, int N>
__device__ __forceinline__ void build_c2r_row(const cplx<T>* plane, cplx<T>* row, int nplx,
                                              int ya) {
  constexpr int LDY = PlaneLd<N>::value;
  for (int k = threadIdx.x & 31; k < N; k += 32) {
    cplx<T> z;
    if (k == 0) {
      z = mk<T>(plane[ya].x, plane[ya + 1].x);
    } else if (k < nplx) {
      cplx<T> a = plane[k * LDY + ya], b = plane[k * LDY + ya + 1];
      z = mk<T>(a.x + b.y, b.x - a.y);  // conj(a) + i conj(b)
    } else if (N - k < nplx) {
      int m = N - k;
      cplx<T> a = plane[m * LDY + ya], b = plane[m * LDY + ya + 1];
      z = mk<T>(a.x - b.y, a.y + b.x);  // a + i b
    } else {
      z = mk<T>(0, 0);
    }
    row[k] = z;
  }
  __syncwarp();
}

// The calling warp splits the spectra of the two real rows held in `row`
// (after the forward x-FFT), applies the imag flip and stores kx < nplane_x
// into plane rows (ya, ya+1).
template <typename T, int N>
__device__ __forceinline__ void extract_r2c_row(const cplx<T>* row, cplx<T>* plane, int nplx,
                                                int ya) {
  constexpr int LDY = PlaneLd<N>::value;
  for (int k = threadIdx.x & 31; k < nplx; k += 32) {
    cplx<T> zk = row[k];
    cplx<T> zm = row[k == 0 ? 0 : N - k];
    // A = (zk + conj zm)/2 ; B = (zk - conj zm)/(2i); stored conjugated
    plane[k * LDY + ya] = mk<T>((T)0.5 * (zk.x + zm.x), (T)0.5 * (zm.y - zk.y));
    plane[k * LDY + ya + 1] = mk<T>((T)0.5 * (zk.y + zm.y), (T)0.5 * (zk.x - zm.x));
  }
  __syncwarp();
}

template <typename T, int N>
struct PShape {
  static constexpr int LDY = PlaneLd<N>::value, LDX = PlaneLd<N>::value;
  static constexpr int E = (N + 31) / 32;               // row elements per lane
  static constexpr int QMAX = std::max(1, 32 / (2 * E));  // row pairs a warp accumulates
  static constexpr int ROWS = std::min(N, 2 * QMAX * PWARPS) & ~1;  // rows per y-split
  static constexpr int RPW = PlaneLd<N>::lines;         // row buffers per warp
  static constexpr size_t LIMIT = 227 * 1024;
  static constexpr size_t bytes(int nplx) {
    return sizeof(cplx<T>) *
           ((size_t)N + (size_t)nplx * LDY + (size_t)PWARPS * RPW * LDX);
  }
};

// ---------------------------------------------------------------------------
// K2: planes -> psi(r).  MODE 0 accumulates occ*psi^2 into per-group FP64
// partial densities held in registers (each warp owns row pairs
// warp, warp+16, ... of the block's y range); MODE 1 writes psi(r) (FP64).
// A warp builds and transforms up to RPW row pairs together.
template <typename T, int N, int MODE>
__global__ void __launch_bounds__(PTHREADS, 1)
k_xy_fwd(const cplx<T>* __restrict__ pen, StateGeom g, const cplx<T>* __restrict__ twx_g,
         const double* __restrict__ occ, int nstates, int spg, int ysplit_rows,
         double* __restrict__ out) {
  constexpr int LDY = PShape<T, N>::LDY, LDX = PShape<T, N>::LDX;
  constexpr int E = PShape<T, N>::E, QMAX = PShape<T, N>::QMAX, RPW = PShape<T, N>::RPW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* plane = tw + N;
  cplx<T>* rows = plane + g.nplane_x * LDY;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  cplx<T>* wrows = rows + (size_t)warp * RPW * LDX;
  const int z = blockIdx.x;
  const int grp = blockIdx.y;
  const int y0 = blockIdx.z * ysplit_rows;
  const int nrows = min(ysplit_rows, N - y0);
  const int npair = nrows / 2;
  const int s0 = grp * spg, s1 = min(nstates, s0 + spg);
  for (int i = threadIdx.x; i < N; i += PTHREADS) tw[i] = twx_g[i];
  double acc[QMAX][2][E];
#pragma unroll
  for (int q = 0; q < QMAX; ++q)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int e = 0; e < E; ++e) acc[q][h][e] = 0.0;
  __syncthreads();
  for (int s = s0; s < s1; ++s) {
    scatter_plane<T, N>(pen + ((size_t)s * N + z) * g.nlpad, plane, g);
    plane_columns<T, N, false>(plane, g.nplane_x, tw);  // FFTW_FORWARD y
    __syncthreads();
    const double w = (MODE == 0) ? occ[s] : 1.0;
    if (MODE == 0) {
#pragma unroll
      for (int q0 = 0; q0 < QMAX; q0 += RPW) {
        int nb = 0;
#pragma unroll
        for (int i = 0; i < RPW; ++i) {
          const int pp = warp + PWARPS * (q0 + i);
          if (q0 + i < QMAX && pp < npair) {
            build_c2r_row<T, N>(plane, wrows + i * LDX, g.nplane_x, y0 + 2 * pp);
            nb = i + 1;
          }
        }
        warp_lines<T, N, true>(wrows, LDX, nb, tw);  // C2R, +i sign
#pragma unroll
        for (int i = 0; i < RPW; ++i) {
          const int q = q0 + i;
          if (q < QMAX && i < nb) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
              int x = lane + 32 * e;
              if (x < N) {
                cplx<T> v = wrows[i * LDX + x];
                acc[q][0][e] += w * (double)v.x * (double)v.x;
                acc[q][1][e] += w * (double)v.y * (double)v.y;
              }
            }
          }
        }
        __syncwarp();
      }
    } else {
      for (int p0 = warp * RPW; p0 < npair; p0 += PWARPS * RPW) {
        const int nb = min(RPW, npair - p0);
#pragma unroll 1
        for (int i = 0; i < nb; ++i)
          build_c2r_row<T, N>(plane, wrows + i * LDX, g.nplane_x, y0 + 2 * (p0 + i));
        warp_lines<T, N, true>(wrows, LDX, nb, tw);  // C2R, +i sign
#pragma unroll 1
        for (int i = 0; i < nb; ++i) {
          const int ya = y0 + 2 * (p0 + i);
          double* o = out + (((size_t)s * N + z) * N + ya) * N;
          for (int x = lane; x < N; x += 32) {
            cplx<T> v = wrows[i * LDX + x];
            o[x] = (double)v.x;
            o[N + x] = (double)v.y;
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
  }
  if (MODE == 0) {
    double* o = out + ((size_t)grp * N + z) * N * N;
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
      int pp = warp + PWARPS * q;
      if (pp < npair) {
        int ya = y0 + 2 * pp;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          int x = lane + 32 * e;
          if (x < N) {
            o[(size_t)ya * N + x] = acc[q][0][e];
            o[(size_t)(ya + 1) * N + x] = acc[q][1][e];
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// K3: MODE 0: pencils -> psi(r) -> psi*V*occ -> planes -> pencils_out
//     MODE 1: real f(r) (FP64, [s][z][y][x]) -> planes -> pencils_out
// Each warp takes up to RPW row pairs at a time (pairs warp*RPW + i, then
// + PWARPS*RPW) through C2R, the product and R2C in its own row buffers.
template <typename T, int N, int MODE>
__global__ void __launch_bounds__(PTHREADS, 1)
k_xy_bwd(const cplx<T>* __restrict__ pen, const double* __restrict__ freal,
         const T* __restrict__ vks, cplx<T>* __restrict__ pen_out, StateGeom g,
         const cplx<T>* __restrict__ twx_g, const double* __restrict__ occ, int nstates,
         int spg) {
  constexpr int LDY = PShape<T, N>::LDY, LDX = PShape<T, N>::LDX, RPW = PShape<T, N>::RPW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* plane = tw + N;
  cplx<T>* rows = plane + g.nplane_x * LDY;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  cplx<T>* wrows = rows + (size_t)warp * RPW * LDX;
  const int z = blockIdx.x;
  const int s0 = blockIdx.y * spg, s1 = min(nstates, s0 + spg);
  for (int i = threadIdx.x; i < N; i += PTHREADS) tw[i] = twx_g[i];
  const T* vplane = (MODE == 0) ? vks + (size_t)z * N * N : nullptr;
  __syncthreads();
  for (int s = s0; s < s1; ++s) {
    if (MODE == 0) {
      scatter_plane<T, N>(pen + ((size_t)s * N + z) * g.nlpad, plane, g);
      plane_columns<T, N, false>(plane, g.nplane_x, tw);
      __syncthreads();
    }
    const T w = (MODE == 0) ? (T)occ[s] : (T)1;
    for (int p0 = warp * RPW; p0 < N / 2; p0 += PWARPS * RPW) {
      const int nb = min(RPW, N / 2 - p0);
      if (MODE == 0) {
#pragma unroll 1
        for (int i = 0; i < nb; ++i)
          build_c2r_row<T, N>(plane, wrows + i * LDX, g.nplane_x, 2 * (p0 + i));
        warp_lines<T, N, true>(wrows, LDX, nb, tw);
#pragma unroll 1
        for (int i = 0; i < nb; ++i) {
          const int ya = 2 * (p0 + i);
          cplx<T>* row = wrows + i * LDX;
          for (int x = lane; x < N; x += 32) {
            cplx<T> v = row[x];
            v.x *= __ldg(vplane + ya * N + x) * w;
            v.y *= __ldg(vplane + (ya + 1) * N + x) * w;
            row[x] = v;
          }
        }
      } else {
        const double* fs = freal + ((size_t)s * N + z) * N * N;
#pragma unroll 1
        for (int i = 0; i < nb; ++i) {
          const int ya = 2 * (p0 + i);
          cplx<T>* row = wrows + i * LDX;
          for (int x = lane; x < N; x += 32)
            row[x] = mk<T>((T)fs[ya * N + x], (T)fs[(ya + 1) * N + x]);
        }
      }
      __syncwarp();
      warp_lines<T, N, false>(wrows, LDX, nb, tw);  // R2C, -i sign
#pragma unroll 1
      for (int i = 0; i < nb; ++i)
        extract_r2c_row<T, N>(wrows + i * LDX, plane, g.nplane_x, 2 * (p0 + i));
    }
    __syncthreads();
    plane_columns<T, N, true>(plane, g.nplane_x, tw);  // FFTW_BACKWARD along y
    __syncthreads();
    cplx<T>* po = pen_out + ((size_t)s * N + z) * g.nlpad;
    for (int l = threadIdx.x; l < g.nlines; l += PTHREADS) {
      int xy = __ldg(g.line_xy + l);
      po[l] = plane[(xy & 0xffff) * LDY + (xy >> 16)];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Plane passes for planes that do not fit in a block's shared memory (the
// density sphere at n = 200 in FP64: 99 columns of 201 complex): the columns
// (y) and the row pairs (x) of K2/K3 MODE 1 in separate launches, the
// y-transformed plane in global memory as [state][z][y][nplane_x].  Same
// transforms, signs and imag flips as k_xy_fwd / k_xy_bwd.
constexpr int SPLIT_THREADS = 256;
constexpr int SPLIT_CW = 8;  // columns per block (one per warp)

// FWD: lines of the plane with x in [x0, x0 + CW) -> forward y-FFT -> tbuf.
// !FWD: tbuf columns -> backward y-FFT -> the lines of those columns.
template <typename T, int N, bool FWD>
__global__ void __launch_bounds__(SPLIT_THREADS)
k_split_cols(const cplx<T>* __restrict__ pen, cplx<T>* __restrict__ pen_out, StateGeom g,
             const cplx<T>* __restrict__ twx_g, cplx<T>* __restrict__ tbuf) {
  constexpr int LDY = PlaneLd<N>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* cols = tw + N;  // [SPLIT_CW][LDY]
  const int z = blockIdx.x, x0 = blockIdx.y * SPLIT_CW, s = blockIdx.z;
  const int nplx = g.nplane_x;
  const int ncol = min(SPLIT_CW, nplx - x0);
  for (int i = threadIdx.x; i < N; i += SPLIT_THREADS) tw[i] = twx_g[i];
  cplx<T>* t0 = tbuf + ((size_t)s * N + z) * N * nplx;
  const size_t prow = ((size_t)s * N + z) * g.nlpad;
  if (FWD) {
    for (int i = threadIdx.x; i < SPLIT_CW * LDY; i += SPLIT_THREADS) cols[i] = mk<T>(0, 0);
    __syncthreads();
    for (int l = threadIdx.x; l < g.nlines; l += SPLIT_THREADS) {
      const int xy = __ldg(g.line_xy + l), x = xy & 0xffff;
      if (x >= x0 && x < x0 + ncol) cols[(x - x0) * LDY + (xy >> 16)] = pen[prow + l];
    }
  } else {
    for (int i = threadIdx.x; i < N * ncol; i += SPLIT_THREADS) {
      const int y = i / ncol, xi = i - y * ncol;
      cols[xi * LDY + y] = t0[(size_t)y * nplx + x0 + xi];
    }
  }
  __syncthreads();
  block_lines<T, N, !FWD>(cols, LDY, ncol, tw);  // FFTW_FORWARD y / FFTW_BACKWARD y
  __syncthreads();
  if (FWD) {
    for (int i = threadIdx.x; i < N * ncol; i += SPLIT_THREADS) {
      const int y = i / ncol, xi = i - y * ncol;
      t0[(size_t)y * nplx + x0 + xi] = cols[xi * LDY + y];
    }
  } else {
    for (int l = threadIdx.x; l < g.nlines; l += SPLIT_THREADS) {
      const int xy = __ldg(g.line_xy + l), x = xy & 0xffff;
      if (x >= x0 && x < x0 + ncol) pen_out[prow + l] = cols[(x - x0) * LDY + (xy >> 16)];
    }
  }
}

// FWD: row pair (ya, ya + 1) from tbuf -> C2R -> real rows of out.
// !FWD: real rows of freal -> R2C -> tbuf.  One warp per row pair.
template <typename T, int N, bool FWD>
__global__ void __launch_bounds__(SPLIT_THREADS)
k_split_rows(const double* __restrict__ freal, double* __restrict__ out, StateGeom g,
             const cplx<T>* __restrict__ twx_g, cplx<T>* __restrict__ tbuf) {
  constexpr int LDX = PlaneLd<N>::value;
  constexpr int NW = SPLIT_THREADS / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  cplx<T>* row = tw + N + (size_t)warp * LDX;
  const int z = blockIdx.x, s = blockIdx.z;
  const int nplx = g.nplane_x;
  for (int i = threadIdx.x; i < N; i += SPLIT_THREADS) tw[i] = twx_g[i];
  __syncthreads();
  const int pp = blockIdx.y * NW + warp;
  if (pp >= N / 2) return;  // no block-wide barrier follows
  const int ya = 2 * pp;
  cplx<T>* t0 = tbuf + ((size_t)s * N + z) * N * nplx;
  const cplx<T>* ra = t0 + (size_t)ya * nplx;
  const cplx<T>* rb = ra + nplx;
  const size_t ro = (((size_t)s * N + z) * N + ya) * N;
  if (FWD) {
    for (int k = lane; k < N; k += 32) {  // as build_c2r_row
      cplx<T> zz;
      if (k == 0) {
        zz = mk<T>(ra[0].x, rb[0].x);
      } else if (k < nplx) {
        const cplx<T> a = ra[k], b = rb[k];
        zz = mk<T>(a.x + b.y, b.x - a.y);
      } else if (N - k < nplx) {
        const cplx<T> a = ra[N - k], b = rb[N - k];
        zz = mk<T>(a.x - b.y, a.y + b.x);
      } else {
        zz = mk<T>(0, 0);
      }
      row[k] = zz;
    }
    __syncwarp();
    fft_line_warp<T, N, true>(row, tw);  // C2R, +i sign
    for (int x = lane; x < N; x += 32) {
      const cplx<T> v = row[x];
      out[ro + x] = (double)v.x;
      out[ro + N + x] = (double)v.y;
    }
  } else {
    for (int x = lane; x < N; x += 32) row[x] = mk<T>((T)freal[ro + x], (T)freal[ro + N + x]);
    __syncwarp();
    fft_line_warp<T, N, false>(row, tw);  // R2C, -i sign
    cplx<T>* wa = t0 + (size_t)ya * nplx;
    cplx<T>* wb = wa + nplx;
    for (int k = lane; k < nplx; k += 32) {  // as extract_r2c_row
      const cplx<T> zk = row[k], zm = row[k == 0 ? 0 : N - k];
      wa[k] = mk<T>((T)0.5 * (zk.x + zm.x), (T)0.5 * (zm.y - zk.y));
      wb[k] = mk<T>((T)0.5 * (zk.y + zm.y), (T)0.5 * (zk.x - zm.x));
    }
  }
}

// ---------------------------------------------------------------------------
// Plane passes with register-resident line FFTs (ShflFft) for the sizes
// ShflCfg<N> lists.  A group of NL lanes owns one column (y) or one row pair
// (x) at a time; only the plane itself is in shared memory.  Columns are
// transformed in place by dif (natural -> the permuted storage shfl_perm) or
// dit (permuted -> natural); rows are built from the plane straight into
// registers and written back to the permuted positions they came from.

template <typename T, int N>
struct SShape {
  static constexpr int LDY = N + 1;
  static constexpr int NL = ShflCfg<N>::NL, M = ShflCfg<N>::M;
  static constexpr int NG = PTHREADS / NL;                 // lane groups per block
  static constexpr int QMAX = (N / 2 + NG - 1) / NG;       // row pairs per group
  static constexpr size_t bytes(int nplx) {
    return sizeof(cplx<T>) * ((size_t)N + (size_t)nplx * LDY);
  }
};

// Row pair (ya, ya+1) of the y-transformed (permuted) plane as the C2R input
// Z = Xa + i Xb in dif order (element x = l + NL k in slot k): the imag flip,
// the Hermitian extension to kx > N/2, zero outside the nplane_x columns.
template <typename T, int N>
__device__ __forceinline__ void shfl_build_row(const cplx<T>* plane, int ldy, int nplx, int ya,
                                               const ShflFft<T, N>& F,
                                               cplx<T> (&v)[ShflCfg<N>::M]) {
  constexpr int NL = ShflCfg<N>::NL, M = ShflCfg<N>::M;
  const int pa = shfl_perm<N>(ya), pb = shfl_perm<N>(ya + 1);
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const int x = F.l + NL * k;
    cplx<T> z = mk<T>(0, 0);
    if (x == 0) {
      z = mk<T>(plane[pa].x, plane[pb].x);
    } else if (x < nplx) {
      const cplx<T> a = plane[x * ldy + pa], b = plane[x * ldy + pb];
      z = mk<T>(a.x + b.y, b.x - a.y);  // conj(a) + i conj(b)
    } else if (N - x < nplx) {
      const int m = N - x;
      const cplx<T> a = plane[m * ldy + pa], b = plane[m * ldy + pb];
      z = mk<T>(a.x - b.y, a.y + b.x);  // a + i b
    }
    v[k] = z;
  }
}

// After dit (forward, R2C) of a row pair: natural Zf[l + NL k] in slot k.
// Split the two real rows' spectra, apply the imag flip and store kx <
// nplane_x at the permuted positions of rows ya, ya+1.
template <typename T, int N>
__device__ __forceinline__ void shfl_extract_row(const cplx<T> (&v)[ShflCfg<N>::M],
                                                 cplx<T>* plane, int ldy, int nplx, int ya,
                                                 const ShflFft<T, N>& F, bool act) {
  constexpr int NL = ShflCfg<N>::NL, M = ShflCfg<N>::M;
  const int pa = shfl_perm<N>(ya), pb = shfl_perm<N>(ya + 1);
  const int src = (NL - F.l) & (NL - 1);
#pragma unroll
  for (int k = 0; k < M; ++k) {
    // Zf[N - kx] with kx = l + NL k: lane NL - l, slot M - 1 - k (l > 0); own slot (M - k) % M (l = 0)
    cplx<T> zm;
    zm.x = __shfl_sync(0xffffffffu, v[M - 1 - k].x, src, NL);
    zm.y = __shfl_sync(0xffffffffu, v[M - 1 - k].y, src, NL);
    if (F.l == 0) zm = v[(M - k) % M];
    const int kx = F.l + NL * k;
    if (act && kx < nplx) {
      const cplx<T> zk = v[k];
      plane[kx * ldy + pa] = mk<T>((T)0.5 * (zk.x + zm.x), (T)0.5 * (zm.y - zk.y));
      plane[kx * ldy + pb] = mk<T>((T)0.5 * (zk.y + zm.y), (T)0.5 * (zk.x - zm.x));
    }
  }
}

// K2 (shuffle form): planes -> psi(r).  MODE 0 accumulates occ psi^2 into the
// group's FP64 registers (row pairs grp, grp + NG, ...), MODE 1 writes psi(r).
template <typename T, int N, int MODE>
__global__ void __launch_bounds__(PTHREADS, 1)
k_xy_fwd_s(const cplx<T>* __restrict__ pen, StateGeom g, const cplx<T>* __restrict__ twx_g,
           const double* __restrict__ occ, int nstates, int spg, double* __restrict__ out) {
  using S = SShape<T, N>;
  constexpr int LDY = S::LDY, NL = S::NL, M = S::M, NG = S::NG, QMAX = S::QMAX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* plane = tw + N;
  const int grp = threadIdx.x / NL;
  const int z = blockIdx.x;
  const int s0 = blockIdx.y * spg, s1 = min(nstates, s0 + spg);
  for (int i = threadIdx.x; i < N; i += PTHREADS) tw[i] = twx_g[i];
  __syncthreads();
  ShflFft<T, N> F;
  F.init(tw);
  double acc[QMAX][2][M];
#pragma unroll
  for (int q = 0; q < QMAX; ++q)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int k = 0; k < M; ++k) acc[q][h][k] = 0.0;
  for (int s = s0; s < s1; ++s) {
    scatter_plane<T, N>(pen + ((size_t)s * N + z) * g.nlpad, plane, g);
    shfl_columns<T, N, false, true>(plane, LDY, g.nplane_x, F, tw, grp, NG);  // FFTW_FORWARD y
    __syncthreads();
    const double w = (MODE == 0) ? occ[s] : 1.0;
    // every lane of a warp runs the shuffles: groups past the last pair
    // transform row 0 and drop the result
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
      const int pp = grp + NG * q;
      const bool act = pp < N / 2;
      const int ya = act ? 2 * pp : 0;
      cplx<T> v[M];
      shfl_build_row<T, N>(plane, LDY, g.nplane_x, ya, F, v);
      F.template dif<true>(v, tw);  // C2R, +i sign
      if (act) {
        if (MODE == 0) {
#pragma unroll
          for (int k = 0; k < M; ++k) {
            acc[q][0][k] += w * (double)v[k].x * (double)v[k].x;
            acc[q][1][k] += w * (double)v[k].y * (double)v[k].y;
          }
        } else {
          double* o = out + (((size_t)s * N + z) * N + ya) * N;
#pragma unroll
          for (int k = 0; k < M; ++k) {
            const int x = F.pos(k);
            o[x] = (double)v[k].x;
            o[N + x] = (double)v[k].y;
          }
        }
      }
    }
    __syncthreads();
  }
  if (MODE == 0) {
    double* o = out + ((size_t)blockIdx.y * N + z) * N * N;
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
      const int pp = grp + NG * q;
      if (pp < N / 2) {
        const int ya = 2 * pp;
#pragma unroll
        for (int k = 0; k < M; ++k) {
          const int x = F.pos(k);
          o[(size_t)ya * N + x] = acc[q][0][k];
          o[(size_t)(ya + 1) * N + x] = acc[q][1][k];
        }
      }
    }
  }
}

// K3 (shuffle form): MODE 0 pencils -> psi(r) -> psi V occ -> pencils_out;
// MODE 1 real f(r) (FP64, [s][z][y][x]) -> pencils_out.
template <typename T, int N, int MODE>
__global__ void __launch_bounds__(PTHREADS, 1)
k_xy_bwd_s(const cplx<T>* __restrict__ pen, const double* __restrict__ freal,
           const T* __restrict__ vks, cplx<T>* __restrict__ pen_out, StateGeom g,
           const cplx<T>* __restrict__ twx_g, const double* __restrict__ occ, int nstates,
           int spg) {
  using S = SShape<T, N>;
  constexpr int LDY = S::LDY, M = S::M, NG = S::NG, NL = S::NL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* plane = tw + N;
  const int grp = threadIdx.x / NL;
  const int z = blockIdx.x;
  const int s0 = blockIdx.y * spg, s1 = min(nstates, s0 + spg);
  for (int i = threadIdx.x; i < N; i += PTHREADS) tw[i] = twx_g[i];
  const T* vplane = (MODE == 0) ? vks + (size_t)z * N * N : nullptr;
  __syncthreads();
  ShflFft<T, N> F;
  F.init(tw);
  for (int s = s0; s < s1; ++s) {
    if (MODE == 0) {
      scatter_plane<T, N>(pen + ((size_t)s * N + z) * g.nlpad, plane, g);
      shfl_columns<T, N, false, true>(plane, LDY, g.nplane_x, F, tw, grp, NG);
      __syncthreads();
    }
    const T w = (MODE == 0) ? (T)occ[s] : (T)1;
    // same trip count for every group of a warp (the shuffles need all lanes)
    for (int p0 = 0; p0 < N / 2; p0 += NG) {
      const int pp = p0 + grp;
      const bool act = pp < N / 2;
      const int ya = act ? 2 * pp : 0;
      cplx<T> v[M];
      if (MODE == 0) {
        shfl_build_row<T, N>(plane, LDY, g.nplane_x, ya, F, v);
        F.template dif<true>(v, tw);  // C2R, +i sign
#pragma unroll
        for (int k = 0; k < M; ++k) {
          const int x = F.pos(k);
          v[k].x *= __ldg(vplane + ya * N + x) * w;
          v[k].y *= __ldg(vplane + (ya + 1) * N + x) * w;
        }
      } else {
        const double* fs = freal + ((size_t)s * N + z) * N * N;
#pragma unroll
        for (int k = 0; k < M; ++k) {
          const int x = F.pos(k);
          v[k] = mk<T>((T)fs[ya * N + x], (T)fs[(ya + 1) * N + x]);
        }
      }
      F.template dit<false>(v, tw);  // R2C, -i sign
      shfl_extract_row<T, N>(v, plane, LDY, g.nplane_x, ya, F, act);
    }
    __syncthreads();
    shfl_columns<T, N, true, false>(plane, LDY, g.nplane_x, F, tw, grp, NG);  // BACKWARD y
    __syncthreads();
    cplx<T>* po = pen_out + ((size_t)s * N + z) * g.nlpad;
    for (int l = threadIdx.x; l < g.nlines; l += PTHREADS) {
      int xy = __ldg(g.line_xy + l);
      po[l] = plane[(xy & 0xffff) * LDY + (xy >> 16)];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Plane passes in the two-stage form (fft_p16.cuh), FP32, N = 32, 64, 128:
// 256 threads, every warp 32 / R line groups of R threads, one line (a
// column or a row pair) per group at a time.  The plane is [nplane_x][LDY]
// with LDY = N + 3; every line group owns a scratch line of SCR = N + N/16
// elements, the exchange buffer of its column and row transforms.  Row pairs
// are built straight from the plane into stride layout (imag flip, Hermitian
// extension), C2R'd by s2b into block layout where V_KS (K3) or the density
// (K2) is applied, and (K3) R2C'd by b2s back into stride layout, where the
// two real rows' spectra are split with one shuffle.
// Bank layout (8-byte elements, a warp access served as two half-warp
// phases): with LDY odd and LDY = N + 3 the column loads, the column stores in
// block order and the row builds put the line groups of a half warp on
// disjoint banks, and with the scratch stride SCR (= R mod 2R) so do the
// exchanges: every one of these warp accesses takes the minimum two
// wavefronts (the column exchange in the plane itself took three to four).
// The blocks split the (plane, state) items evenly, plane-major: block b
// takes items [b I / B, (b + 1) I / B) of I = N S, so all B resident blocks
// (B = blocks per SM x SMs) carry the same work whatever S is.
// K2 runs 512 threads (for N = 128 every line group owns one row pair of the
// plane, so its FP64 accumulators fit the registers), K3 256 threads at two
// blocks per SM.
template <int N, int THREADS_>
struct P16Shape {
  static constexpr int THREADS = THREADS_, NW = THREADS / 32;
  static constexpr int LPW = P16Cfg<N>::LPW, SLOTS = NW * LPW;
  static constexpr int LDY = N + 3;
  static constexpr int SL = P16Cfg<N>::SCR;  // scratch line stride
  // twiddles, plane, scratch lines, pencil-row staging (nlines rounded to 2)
  static constexpr size_t bytes(int nplx, int nlines) {
    return sizeof(cplx<float>) *
           ((size_t)N + (size_t)nplx * LDY + (size_t)SLOTS * SL + (size_t)((nlines + 1) & ~1));
  }
};
constexpr int P16_K2_THREADS = 512, P16_K3_THREADS = 256;

// the pencil row of one (state, z) into the shared staging buffer with
// cp.async (8-byte copies, one group per call): issued while the previous
// state is transformed, waited for by p16_scatter
__device__ __forceinline__ void p16_prefetch(const cplx<float>* __restrict__ prow,
                                             cplx<float>* stage, int nlines) {
  for (int l = threadIdx.x; l < nlines; l += blockDim.x)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(stage + l)),
                 "l"(prow + l)
                 : "memory");
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// zero the plane's N rows of every column and scatter the staged pencil row
template <int N, int LDY>
__device__ __forceinline__ void p16_scatter(const cplx<float>* stage, cplx<float>* plane,
                                            const StateGeom& g) {
  for (int i = threadIdx.x; i < g.nplane_x * LDY; i += blockDim.x) plane[i] = mk<float>(0, 0);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  for (int l = threadIdx.x; l < g.nlines; l += blockDim.x) {
    const int xy = __ldg(g.line_xy + l);
    plane[(xy & 0xffff) * LDY + (xy >> 16)] = stage[l];
  }
  __syncthreads();
}

// y-FFTs of the nplane_x columns in place (natural order in and out), the
// exchange through the line group's own scratch; a warp leaves as soon as no
// column is left for any of its groups, and groups past the last column of a
// round run on their scratch and store nothing.
template <int N, bool INV, bool LEAN>
__device__ __forceinline__ void p16_columns(cplx<float>* plane, int ldy, int nplx,
                                            const P16Fft<float, N, LEAN>& F, cplx<float>* scr,
                                            int slot, int nslots) {
  constexpr int R = P16Cfg<N>::R, LPW = P16Cfg<N>::LPW;
  const int wslot = slot - slot % LPW;  // first slot of this warp
  for (int c0 = 0; c0 < nplx; c0 += nslots) {
    if (c0 + wslot >= nplx) break;  // warp-uniform
    const int c = c0 + slot;
    const bool act = c < nplx;
    cplx<float>* col = plane + (size_t)(act ? c : 0) * ldy;
    cplx<float> v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = act ? col[F.t + R * k] : mk<float>(0.f, 0.f);
    F.template s2b<INV>(v, scr);
    if (act) {
#pragma unroll
      for (int q = 0; q < 16; ++q) col[F.bpos(q)] = v[q];
    }
    __syncwarp();
  }
}

// C2R input of rows (ya, ya+1) in stride layout: Z = conj(Xa) + i conj(Xb) from
// the y-transformed plane, Hermitian-extended to kx > N/2 (as shfl_build_row)
template <int N>
__device__ __forceinline__ void p16_build_row(const cplx<float>* plane, int ldy, int nplx, int ya,
                                              int t, cplx<float> (&v)[16]) {
  constexpr int R = P16Cfg<N>::R;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int x = t + R * k;
    cplx<float> z = mk<float>(0, 0);
    if (x == 0) {
      z = mk<float>(plane[ya].x, plane[ya + 1].x);
    } else if (x < nplx) {
      const cplx<float> a = plane[x * ldy + ya], b = plane[x * ldy + ya + 1];
      z = mk<float>(a.x + b.y, b.x - a.y);
    } else if (N - x < nplx) {
      const int m = N - x;
      const cplx<float> a = plane[m * ldy + ya], b = plane[m * ldy + ya + 1];
      z = mk<float>(a.x - b.y, a.y + b.x);
    }
    v[k] = z;
  }
}

// After b2s (forward) of a row pair: Zf[t + R b] in slot b.  Split the two real
// rows' spectra (partner N - kx: thread R - t, slot 15 - b; thread 0 keeps its
// own slot (16 - b) % 16), imag flip, store kx < nplane_x.  All lanes of the
// warp call it (the shuffle); only act stores.
template <int N>
__device__ __forceinline__ void p16_extract_row(const cplx<float> (&v)[16], cplx<float>* plane,
                                                int ldy, int nplx, int ya, int t, bool act) {
  constexpr int R = P16Cfg<N>::R;
  const int src = (R - t) % R;
#pragma unroll
  for (int b = 0; b < 16; ++b) {
    cplx<float> zm;
    zm.x = __shfl_sync(0xffffffffu, v[15 - b].x, src, R);
    zm.y = __shfl_sync(0xffffffffu, v[15 - b].y, src, R);
    if (t == 0) zm = v[(16 - b) % 16];
    const int kx = t + R * b;
    if (act && kx < nplx) {
      const cplx<float> zk = v[b];
      plane[kx * ldy + ya] = mk<float>(0.5f * (zk.x + zm.x), 0.5f * (zm.y - zk.y));
      plane[kx * ldy + ya + 1] = mk<float>(0.5f * (zk.y + zm.y), 0.5f * (zk.x - zm.x));
    }
  }
}

// items [i0, i1) of block b out of B over I = N S (plane-major: item i is
// plane i / S, state i % S); the density reduction uses the same split
__host__ __device__ __forceinline__ long long p16_item_start(long long items, int b, int nblocks) {
  return items * b / nblocks;
}

// K3 (two-stage form): pencils -> psi(r) -> psi V occ -> pencils_out, over
// the block's (plane, state) items
template <int N>
__global__ void __launch_bounds__(P16_K3_THREADS, 2)
k_xy_bwd_p16(const cplx<float>* __restrict__ pen, const float* __restrict__ vks,
             cplx<float>* __restrict__ pen_out, StateGeom g,
             const cplx<float>* __restrict__ twx_g, const double* __restrict__ occ,
             int nstates) {
  using S = P16Shape<N, P16_K3_THREADS>;
  constexpr int LDY = S::LDY, SLOTS = S::SLOTS, R = P16Cfg<N>::R, LPW = S::LPW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<float>* tw = reinterpret_cast<cplx<float>*>(smem_raw);
  cplx<float>* plane = tw + N;
  const int nplx = g.nplane_x;
  const int slot = (threadIdx.x >> 5) * LPW + (threadIdx.x & 31) / R;
  const int wslot = slot - slot % LPW;
  cplx<float>* scr = plane + (size_t)nplx * LDY + (size_t)slot * S::SL;
  cplx<float>* stage = plane + (size_t)nplx * LDY + (size_t)SLOTS * S::SL;
  const long long items = (long long)N * nstates;
  const long long i0 = p16_item_start(items, blockIdx.x, gridDim.x);
  const long long i1 = p16_item_start(items, blockIdx.x + 1, gridDim.x);
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx_g[i];
  if (i0 < i1)
    p16_prefetch(pen + ((size_t)(i0 % nstates) * N + (size_t)(i0 / nstates)) * g.nlpad, stage,
                 g.nlines);
  __syncthreads();
  P16Fft<float, N> F;
  F.init(tw);
  for (long long it = i0; it < i1; ++it) {
    const int z = (int)(it / nstates), s = (int)(it % nstates);
    p16_scatter<N, LDY>(stage, plane, g);
    if (it + 1 < i1)
      p16_prefetch(pen + ((size_t)((it + 1) % nstates) * N + (size_t)((it + 1) / nstates)) *
                             g.nlpad,
                   stage, g.nlines);
    p16_columns<N, false>(plane, LDY, nplx, F, scr, slot, SLOTS);  // FFTW_FORWARD y
    __syncthreads();
    const float* vplane = vks + (size_t)z * N * N;
    const float w = (float)occ[s];
    for (int p0 = 0; p0 < N / 2; p0 += SLOTS) {
      if (p0 + wslot >= N / 2) break;  // warp-uniform: no row pair left for this warp
      const int pp = p0 + slot;
      const bool act = pp < N / 2;
      const int ya = act ? 2 * pp : 0;
      // V_KS of the two rows at this thread's block-layout positions, loaded
      // (from L2) before the C2R so that the transform covers the latency.
      // Slots m, m + R, ..., m + (H - 1) R (m < R) are the H consecutive
      // positions H t + h + 16 m: one vector load of H floats (H = 2, 4, 8;
      // 4 H t bytes from a row start: aligned).
      float va[16], vb[16];
      constexpr int H = P16Cfg<N>::H;
#pragma unroll
      for (int m = 0; m < R; ++m) {
        const int x0 = F.bpos(m);  // = H t + 16 m
        const float* ra = vplane + ya * N + x0;
        const float* rb = ra + N;
        if constexpr (H == 2) {
          const float2 a = __ldg(reinterpret_cast<const float2*>(ra));
          const float2 b = __ldg(reinterpret_cast<const float2*>(rb));
          va[m] = a.x; va[m + R] = a.y;
          vb[m] = b.x; vb[m + R] = b.y;
        } else {
#pragma unroll
          for (int h4 = 0; h4 < H; h4 += 4) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(ra + h4));
            const float4 b = __ldg(reinterpret_cast<const float4*>(rb + h4));
            va[m + (h4 + 0) * R] = a.x; va[m + (h4 + 1) * R] = a.y;
            va[m + (h4 + 2) * R] = a.z; va[m + (h4 + 3) * R] = a.w;
            vb[m + (h4 + 0) * R] = b.x; vb[m + (h4 + 1) * R] = b.y;
            vb[m + (h4 + 2) * R] = b.z; vb[m + (h4 + 3) * R] = b.w;
          }
        }
      }
      cplx<float> v[16];
      p16_build_row<N>(plane, LDY, nplx, ya, F.t, v);
      F.template s2b<true>(v, scr);  // C2R, +i sign
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        v[q].x *= va[q] * w;
        v[q].y *= vb[q] * w;
      }
      F.template b2s<false>(v, scr);  // R2C, -i sign
      p16_extract_row<N>(v, plane, LDY, nplx, ya, F.t, act);
    }
    __syncthreads();
    p16_columns<N, true>(plane, LDY, nplx, F, scr, slot, SLOTS);  // FFTW_BACKWARD y
    __syncthreads();
    cplx<float>* po = pen_out + ((size_t)s * N + z) * g.nlpad;
    for (int l = threadIdx.x; l < g.nlines; l += blockDim.x) {
      const int xy = __ldg(g.line_xy + l);
      po[l] = plane[(xy & 0xffff) * LDY + (xy >> 16)];
    }
    __syncthreads();
  }
}

// K2 (two-stage form): planes -> occ psi^2 accumulated in FP64 registers over
// the block's items of one plane; each plane the block touches (segment q of
// its item range) gets its own partial density out[b segs + q][y][x].  Every
// row pair of the plane belongs to one line group (PASSES = (N/2) / SLOTS of
// them per group), the slots of its block layout to the group's threads.
template <int N>
__global__ void __launch_bounds__(P16_K2_THREADS, 1)
k_xy_fwd_p16(const cplx<float>* __restrict__ pen, StateGeom g,
             const cplx<float>* __restrict__ twx_g, const double* __restrict__ occ,
             int nstates, int segs, double* __restrict__ out) {
  using S = P16Shape<N, P16_K2_THREADS>;
  constexpr int LDY = S::LDY, SLOTS = S::SLOTS, R = P16Cfg<N>::R, LPW = S::LPW;
  constexpr int PASSES = (N / 2 + SLOTS - 1) / SLOTS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<float>* tw = reinterpret_cast<cplx<float>*>(smem_raw);
  cplx<float>* plane = tw + N;
  const int nplx = g.nplane_x;
  const int slot = (threadIdx.x >> 5) * LPW + (threadIdx.x & 31) / R;
  const int wslot = slot - slot % LPW;
  cplx<float>* scr = plane + (size_t)nplx * LDY + (size_t)slot * S::SL;
  cplx<float>* stage = plane + (size_t)nplx * LDY + (size_t)SLOTS * S::SL;
  const long long items = (long long)N * nstates;
  const long long i0 = p16_item_start(items, blockIdx.x, gridDim.x);
  const long long i1 = p16_item_start(items, blockIdx.x + 1, gridDim.x);
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx_g[i];
  if (i0 < i1)
    p16_prefetch(pen + ((size_t)(i0 % nstates) * N + (size_t)(i0 / nstates)) * g.nlpad, stage,
                 g.nlines);
  __syncthreads();
  P16Fft<float, N, true> F;
  F.init(tw);
  double acc[PASSES][2][16];
#pragma unroll
  for (int q = 0; q < PASSES; ++q)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int k = 0; k < 16; ++k) acc[q][h][k] = 0.0;
  // the partial density of the current plane into its segment, then zero
  auto flush = [&](int seg) {
    double* o = out + ((size_t)blockIdx.x * segs + seg) * N * N;
#pragma unroll
    for (int q = 0; q < PASSES; ++q) {
      const int pp = slot + SLOTS * q;
      if (pp < N / 2) {
        const int ya = 2 * pp;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int x = F.bpos(k);
          o[(size_t)ya * N + x] = acc[q][0][k];
          o[(size_t)(ya + 1) * N + x] = acc[q][1][k];
          acc[q][0][k] = 0.0;
          acc[q][1][k] = 0.0;
        }
      }
    }
  };
  int zc = (int)(i0 / nstates), seg = 0;
  for (long long it = i0; it < i1; ++it) {
    const int z = (int)(it / nstates), s = (int)(it % nstates);
    if (z != zc) {  // block-uniform
      flush(seg);
      zc = z;
      ++seg;
    }
    p16_scatter<N, LDY>(stage, plane, g);
    if (it + 1 < i1)
      p16_prefetch(pen + ((size_t)((it + 1) % nstates) * N + (size_t)((it + 1) / nstates)) *
                             g.nlpad,
                   stage, g.nlines);
    p16_columns<N, false>(plane, LDY, nplx, F, scr, slot, SLOTS);  // FFTW_FORWARD y
    __syncthreads();
    const double w = occ[s];
#pragma unroll
    for (int q = 0; q < PASSES; ++q) {
      if (SLOTS * q + wslot < N / 2) {  // warp-uniform
        const int pp = slot + SLOTS * q;
        const bool act = pp < N / 2;
        const int ya = act ? 2 * pp : 0;
        cplx<float> v[16];
        p16_build_row<N>(plane, LDY, nplx, ya, F.t, v);
        F.template s2b<true>(v, scr);  // C2R, +i sign
        if (act) {
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            acc[q][0][k] += w * (double)v[k].x * (double)v[k].x;
            acc[q][1][k] += w * (double)v[k].y * (double)v[k].y;
          }
        }
      }
    }
    __syncthreads();
  }
  if (i0 < i1) flush(seg);
}

// sum, for every plane z, the partial densities of the blocks whose item
// range touched it (block order: deterministic), scaled
__global__ void k_rho_reduce_items(const double* __restrict__ part, int n, int nstates,
                                   int nblocks, int segs, double scale, double* __restrict__ rho);

// ---------------------------------------------------------------------------
// K3 for N = 200 in the two-stage 20 x 10 form (fft_t20.cuh), FP32: the same
// item split and plane passes as k_xy_bwd_p16, 512 threads (16 warps of three
// 10-thread line groups; lanes 30 and 31 work on a scratch line of their own
// and store nothing), one block per SM.  The plane is [nplane_x][N + 3];
// every line group (and every warp's idle pair) owns a scratch line of
// N + N / 20 elements.
constexpr int T20_K3_THREADS = 512;
struct T20Shape {
  static constexpr int N = 200, R = 10, LPW = 3, NW = T20_K3_THREADS / 32;
  static constexpr int SLOTS = NW * LPW;        // working line groups
  static constexpr int SCRL = NW * (LPW + 1);   // scratch lines (idle pairs included)
  static constexpr int LDY = N + 3;
  static constexpr int SL = T20Cfg::SCR + 2;    // scratch line stride
  static constexpr size_t bytes(int nplx, int nlines) {
    return sizeof(cplx<float>) *
           ((size_t)N + (size_t)nplx * LDY + (size_t)SCRL * SL + (size_t)((nlines + 1) & ~1));
  }
};

template <int NN>
__global__ void __launch_bounds__(T20_K3_THREADS, 1)
k_xy_bwd_t20(const cplx<float>* __restrict__ pen, const float* __restrict__ vks,
             cplx<float>* __restrict__ pen_out, StateGeom g,
             const cplx<float>* __restrict__ twx_g, const double* __restrict__ occ,
             int nstates) {
  static_assert(NN == 200, "the 20 x 10 two-stage form");
  using S = T20Shape;
  constexpr int N = S::N, LDY = S::LDY, SLOTS = S::SLOTS, R = S::R, LPW = S::LPW, P = 20;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<float>* tw = reinterpret_cast<cplx<float>*>(smem_raw);
  cplx<float>* plane = tw + N;
  const int nplx = g.nplane_x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = lane / R;                 // 0..2 working, 3 idle
  const bool idle = grp >= LPW;
  const int slot = warp * LPW + (idle ? 0 : grp);
  const int wslot = warp * LPW;
  cplx<float>* scr = plane + (size_t)nplx * LDY + (size_t)(warp * (LPW + 1) + grp) * S::SL;
  cplx<float>* stage = plane + (size_t)nplx * LDY + (size_t)S::SCRL * S::SL;
  const long long items = (long long)N * nstates;
  const long long i0 = p16_item_start(items, blockIdx.x, gridDim.x);
  const long long i1 = p16_item_start(items, blockIdx.x + 1, gridDim.x);
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = twx_g[i];
  if (i0 < i1)
    p16_prefetch(pen + ((size_t)(i0 % nstates) * N + (size_t)(i0 / nstates)) * g.nlpad, stage,
                 g.nlines);
  __syncthreads();
  T20Fft<float> F;
  F.init(tw);
  // partner lane of the R2C split (kx -> N - kx): thread (R - t) % R of the group
  const int src = idle ? lane : grp * R + (R - F.t) % R;
  for (long long it = i0; it < i1; ++it) {
    const int z = (int)(it / nstates), s = (int)(it % nstates);
    p16_scatter<N, LDY>(stage, plane, g);
    if (it + 1 < i1)
      p16_prefetch(pen + ((size_t)((it + 1) % nstates) * N + (size_t)((it + 1) / nstates)) *
                             g.nlpad,
                   stage, g.nlines);
    // y pass, forward (FFTW_FORWARD y)
    for (int c0 = 0; c0 < nplx; c0 += SLOTS) {
      if (c0 + wslot >= nplx) break;  // warp-uniform
      const int c = c0 + slot;
      const bool act = !idle && c < nplx;
      cplx<float>* col = plane + (size_t)(act ? c : 0) * LDY;
      cplx<float> v[P];
#pragma unroll
      for (int k = 0; k < P; ++k) v[k] = act ? col[F.t + R * k] : mk<float>(0.f, 0.f);
      F.template s2b<false>(v, scr);
      if (act) {
#pragma unroll
        for (int q = 0; q < P; ++q) col[F.bpos(q)] = v[q];
      }
      __syncwarp();
    }
    __syncthreads();
    const float* vplane = vks + (size_t)z * N * N;
    const float w = (float)occ[s];
    for (int p0 = 0; p0 < N / 2; p0 += SLOTS) {
      if (p0 + wslot >= N / 2) break;  // warp-uniform
      const int pp = p0 + slot;
      const bool act = !idle && pp < N / 2;
      const int ya = act ? 2 * pp : 0;
      // C2R input of rows (ya, ya + 1): Z = conj(Xa) + i conj(Xb), Hermitian-
      // extended to kx > N / 2
      cplx<float> v[P];
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const int x = F.t + R * k;
        cplx<float> zv = mk<float>(0, 0);
        if (act) {
          if (x == 0) {
            zv = mk<float>(plane[ya].x, plane[ya + 1].x);
          } else if (x < nplx) {
            const cplx<float> a = plane[x * LDY + ya], b = plane[x * LDY + ya + 1];
            zv = mk<float>(a.x + b.y, b.x - a.y);
          } else if (N - x < nplx) {
            const int m = N - x;
            const cplx<float> a = plane[m * LDY + ya], b = plane[m * LDY + ya + 1];
            zv = mk<float>(a.x - b.y, a.y + b.x);
          }
        }
        v[k] = zv;
      }
      F.template s2b<true>(v, scr);  // C2R, +i sign
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const int x = F.bpos(q);
        const float va = act ? __ldg(vplane + ya * N + x) : 0.f;
        const float vb = act ? __ldg(vplane + (ya + 1) * N + x) : 0.f;
        v[q].x *= va * w;
        v[q].y *= vb * w;
      }
      F.template b2s<false>(v, scr);  // R2C, -i sign
      // split the two real rows' spectra: partner N - kx in thread (R - t) % R,
      // slot P - 1 - b (thread 0 keeps its own slot (P - b) % P); store kx < nplx
#pragma unroll
      for (int b = 0; b < P; ++b) {
        cplx<float> zm;
        zm.x = __shfl_sync(0xffffffffu, v[P - 1 - b].x, src);
        zm.y = __shfl_sync(0xffffffffu, v[P - 1 - b].y, src);
        if (F.t == 0) zm = v[(P - b) % P];
        const int kx = F.t + R * b;
        if (act && kx < nplx) {
          const cplx<float> zk = v[b];
          plane[kx * LDY + ya] = mk<float>(0.5f * (zk.x + zm.x), 0.5f * (zm.y - zk.y));
          plane[kx * LDY + ya + 1] = mk<float>(0.5f * (zk.y + zm.y), 0.5f * (zk.x - zm.x));
        }
      }
    }
    __syncthreads();
    // y pass, backward (FFTW_BACKWARD y)
    for (int c0 = 0; c0 < nplx; c0 += SLOTS) {
      if (c0 + wslot >= nplx) break;
      const int c = c0 + slot;
      const bool act = !idle && c < nplx;
      cplx<float>* col = plane + (size_t)(act ? c : 0) * LDY;
      cplx<float> v[P];
#pragma unroll
      for (int k = 0; k < P; ++k) v[k] = act ? col[F.t + R * k] : mk<float>(0.f, 0.f);
      F.template s2b<true>(v, scr);
      if (act) {
#pragma unroll
        for (int q = 0; q < P; ++q) col[F.bpos(q)] = v[q];
      }
      __syncwarp();
    }
    __syncthreads();
    cplx<float>* po = pen_out + ((size_t)s * N + z) * g.nlpad;
    for (int l = threadIdx.x; l < g.nlines; l += blockDim.x) {
      const int xy = __ldg(g.line_xy + l);
      po[l] = plane[(xy & 0xffff) * LDY + (xy >> 16)];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// K4: pencils -> backward z-FFT -> pack -> scale.
//   MODE 0: F = scale * wpt * val (then, if occ != null, the kinetic term)
//   MODE 1: plain pack with scale (adjoint transform)
//   MODE 2: EES psi force, F += -wpt conj(mul * val) with the imaginary parts
//           of val and mul dropped at G = 0 (eesPsiForcGspace,
//           cp_ees_nonlocal.C:2000-2064)
template <typename T, int N, int MODE>
__global__ void __launch_bounds__(ZTHREADS)
k_zfft_bwd(const cplx<T>* __restrict__ pen, double2* __restrict__ fout,
           const double2* __restrict__ psi, const double* __restrict__ occ, StateGeom g,
           const cplx<T>* __restrict__ twz, double scale, double ecut,
           double* __restrict__ eke_part, const double2* __restrict__ mul) {
  constexpr int LB = ZShape<N>::LB, LD = ZShape<N>::LD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* buf = tw + N;
  int* soff = reinterpret_cast<int*>(buf + LB * LD);
  int* snneg = soff + LB + 1;
  int* szneg = snneg + LB;
  int* szpos = szneg + LB;
  const int s = blockIdx.y;
  const int l0 = blockIdx.x * LB;
  const int nl = min(LB, g.nlines - l0);
  for (int i = threadIdx.x; i < N; i += ZTHREADS) tw[i] = twz[i];
  for (int i = threadIdx.x; i < nl; i += ZTHREADS) {
    soff[i] = g.line_off[l0 + i];
    snneg[i] = g.line_nneg[l0 + i];
    szneg[i] = g.line_zneg[l0 + i];
    szpos[i] = g.line_zpos[l0 + i];
  }
  if (threadIdx.x == 0) soff[nl] = (l0 + nl < g.nlines) ? g.line_off[l0 + nl] : g.npts;
  const cplx<T>* pi = pen + (size_t)s * N * g.nlpad + l0;
  for (int i = threadIdx.x; i < nl * N; i += ZTHREADS) {
    int z = i / nl, li = i - z * nl;
    buf[li * LD + z] = pi[(size_t)z * g.nlpad + li];
  }
  __syncthreads();
  if constexpr (ShflCfg<N>::ok) {
    ShflFft<T, N> F;
    F.init(tw);
    shfl_columns<T, N, true, true>(buf, LD, nl, F, tw, threadIdx.x / ShflCfg<N>::NL,
                                   ZTHREADS / ShflCfg<N>::NL);  // FFTW_BACKWARD along z
  } else {
    block_lines<T, N, true>(buf, LD, nl, tw);  // FFTW_BACKWARD along z
  }
  __syncthreads();
  const int p0 = soff[0], p1 = soff[nl];
  double e = 0.0;
  const double wocc = (MODE == 0 && occ) ? occ[s] : 0.0;
  for (int p = p0 + threadIdx.x; p < p1; p += ZTHREADS) {
    int li, z;
    locate(p, soff, nl, snneg, szneg, szpos, li, z);
    cplx<T> v = buf[li * LD + (ShflCfg<N>::ok ? shfl_perm<N>(z) : z)];
    if (MODE == 2) {
      double vx = (double)v.x, vy = (double)v.y;
      double2 d = mul[p];
      if (g.g2[p] == 0.0) {
        vy = 0.0;
        d.y = 0.0;
      }
      const double wp = g.wpt[p];
      double2 f = fout[(size_t)s * g.npts + p];
      f.x -= wp * (d.x * vx - d.y * vy);
      f.y += wp * (d.y * vx + d.x * vy);
      fout[(size_t)s * g.npts + p] = f;
      continue;
    }
    double fx = (double)v.x * scale, fy = (double)v.y * scale;
    if (MODE == 0) {
      double wp = g.wpt[p];
      fx *= wp;
      fy *= wp;
      if (occ) {
        double g2 = g.g2[p];
        double2 ps = psi[(size_t)s * g.npts + p];
        if (g2 <= ecut) {
          double wt = wocc * wp * g2;
          fx -= wt * ps.x;
          fy -= wt * ps.y;
          e += wt * (ps.x * ps.x + ps.y * ps.y);
        } else {
          fx = 0.0;
          fy = 0.0;
        }
      }
    }
    fout[(size_t)s * g.npts + p] = make_double2(fx, fy);
  }
  if (MODE == 0 && occ) {
    double t = block_sum(e, red);
    if (threadIdx.x == 0) eke_part[(size_t)s * gridDim.x + blockIdx.x] = 0.5 * t;
  }
}

// ---------------------------------------------------------------------------
// EES non-local plane kernels (N is the NL grid).  The real plane [N][N] lives
// in shared memory and doubles as the row-pair buffers of the x transforms: a
// complex row of N elements occupies exactly the two real rows it produces.

// Per-plane shared memory of the NL kernels: twiddles, the complex plane, the
// real plane.
template <typename T, int N>
struct NlShape {
  static constexpr int LDY = PlaneLd<N>::value;
  static size_t bytes(int nplx) {
    return sizeof(cplx<T>) * ((size_t)N + (size_t)nplx * LDY) + sizeof(T) * (size_t)N * N;
  }
};

// NL G->R (doNlFFTGtoR_Gchare/Rchare, fftCache.C:589-809) of plane z for the
// block's states s0..s1, then for every atom of type ctype with an
// interpolation plane jc on z: zpart[s][atom][jc] = (sum P mn, sum P dmn_x,
// sum P dmn_y, sum P dmn_z) over its 8x8 points (eesZmatRchare :1238-1346 and
// the force sums of eesEnergyAtmForcRchare :1480-1700, before the Z factor).
constexpr int NLTHREADS = 256;  // NL plane kernels: 8 warps, three blocks per SM
template <typename T, int N>
__global__ void __launch_bounds__(NLTHREADS, 3)
k_nl_fwd(const cplx<T>* __restrict__ pen, StateGeom g, const cplx<T>* __restrict__ twx_g,
         NlAtoms A, int ctype, int nstates, int spg, double* __restrict__ zpart) {
  constexpr int LDY = PlaneLd<N>::value;
  constexpr int E = (N + 31) / 32;
  constexpr int NW = NLTHREADS / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* plane = tw + N;
  T* R = reinterpret_cast<T*>(plane + g.nplane_x * LDY);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int z = blockIdx.x;
  const int s0 = blockIdx.y * spg, s1 = min(nstates, s0 + spg);
  for (int i = threadIdx.x; i < N; i += NLTHREADS) tw[i] = twx_g[i];
  const int* pl = A.plist + ((size_t)ctype * (int)A.grid + z) * A.natm;
  const int npl = A.pcount[ctype * (int)A.grid + z];
  const int* tcell = A.tcell + (size_t)z * A.tcap;
  const NlVal* tval = A.tval + (size_t)z * A.tcap;
  // row pairs that some atom's stencil reads (the others are not transformed)
  __shared__ int pairs[N / 2];
  for (int i = threadIdx.x; i < N / 2; i += NLTHREADS) pairs[i] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < npl * kNlInterp; i += NLTHREADS) {
    const int e = i / kNlInterp, jb = i - e * kNlInterp;
    pairs[A.ig[(size_t)(pl[e] & 0xffff) * 3 * kNlInterp + kNlInterp + jb] >> 1] = 1;
  }
  __syncthreads();
  ShflFft<T, N> F;
  if constexpr (ShflCfg<N>::ok) F.init(tw);
  for (int s = s0; s < s1; ++s) {
    scatter_plane<T, N>(pen + ((size_t)s * N + z) * g.nlpad, plane, g);
    if constexpr (ShflCfg<N>::ok) {
      constexpr int NL = ShflCfg<N>::NL, M = ShflCfg<N>::M, NG = NLTHREADS / NL;
      const int grp = threadIdx.x / NL;
      shfl_columns<T, N, false, true>(plane, LDY, g.nplane_x, F, tw, grp, NG);  // FORWARD y
      __syncthreads();
      for (int p0 = 0; p0 < N / 2; p0 += NG) {
        const int pp = p0 + grp;
        const bool act = pp < N / 2 && pairs[pp];
        if (!__any_sync(0xffffffffu, act)) continue;  // warp-uniform: the shuffles need all lanes
        const int ya = act ? 2 * pp : 0;
        cplx<T> v[M];
        shfl_build_row<T, N>(plane, LDY, g.nplane_x, ya, F, v);
        F.template dif<true>(v, tw);  // C2R, +i sign
        if (act) {
#pragma unroll
          for (int k = 0; k < M; ++k) {
            const int x = F.pos(k);
            R[(size_t)ya * N + x] = v[k].x;
            R[(size_t)(ya + 1) * N + x] = v[k].y;
          }
        }
      }
      __syncthreads();
    } else {
    plane_columns<T, N, false>(plane, g.nplane_x, tw);  // FFTW_FORWARD y
    __syncthreads();
    for (int pp = warp; pp < N / 2; pp += NW) {
      if (!pairs[pp]) continue;
      const int ya = 2 * pp;
      cplx<T>* row = reinterpret_cast<cplx<T>*>(R + (size_t)ya * N);
      build_c2r_row<T, N>(plane, row, g.nplane_x, ya);
      fft_line_warp<T, N, true>(row, tw);  // C2R, +i sign
      cplx<T> v[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int x = lane + 32 * e;
        if (x < N) v[e] = row[x];
      }
      __syncwarp();
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int x = lane + 32 * e;
        if (x < N) {
          R[(size_t)ya * N + x] = v[e].x;
          R[(size_t)(ya + 1) * N + x] = v[e].y;
        }
      }
      __syncwarp();
    }
    __syncthreads();
    }
    // atoms on this plane: lane -> point q = lane + 32 h, (jb, ja) = (q / 8, q % 8),
    // cells and Mn products from the plane's stencil table
    for (int e = warp; e < npl; e += NW) {
      const int a = pl[e] & 0xffff, jc = pl[e] >> 16;
      double sz = 0.0, sx = 0.0, sy = 0.0, sw = 0.0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = e * 64 + lane + 32 * h;
        const double pz = (double)R[tcell[i]];
        const NlVal v = tval[i];
        sz += pz * v.mn;
        sx += pz * v.dx;
        sy += pz * v.dy;
        sw += pz * v.dz;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sz += __shfl_xor_sync(0xffffffffu, sz, o);
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sw += __shfl_xor_sync(0xffffffffu, sw, o);
      }
      if (lane == 0) {
        double* o = zpart + (((size_t)s * A.natm + a) * kNlInterp + jc) * 4;
        o[0] = sz; o[1] = sx; o[2] = sy; o[3] = sw;
      }
    }
    __syncthreads();
  }
}

// NL R->G of plane z for the block's states: the plane holds sum_atoms
// zs[s][atom] Mn over the atoms of type ctype (the projPsiRScr scatter of
// eesEnergyAtmForcRchare, formed per touched cell from the plane's gather
// list, atoms in list order, so the sum order is fixed), then x R2C, imag
// flip, y-FFT (doNlFFTRtoG_Rchare, fftCache.C:634-699) into pencils.
template <typename T, int N>
__global__ void __launch_bounds__(NLTHREADS, 3)
k_nl_bwd(cplx<T>* __restrict__ pen_out, StateGeom g, const cplx<T>* __restrict__ twx_g,
         NlAtoms A, int ctype, int nstates, int spg, const double* __restrict__ zs) {
  constexpr int LDY = PlaneLd<N>::value;
  constexpr int E = (N + 31) / 32;
  constexpr int NW = NLTHREADS / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* tw = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* plane = tw + N;
  T* R = reinterpret_cast<T*>(plane + g.nplane_x * LDY);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int z = blockIdx.x;
  const int s0 = blockIdx.y * spg, s1 = min(nstates, s0 + spg);
  for (int i = threadIdx.x; i < N; i += NLTHREADS) tw[i] = twx_g[i];
  const int* pl = A.plist + ((size_t)ctype * (int)A.grid + z) * A.natm;
  const int npl = A.pcount[ctype * (int)A.grid + z];
  // row pairs the scatter writes (the others transform to zero)
  __shared__ int pairs[N / 2];
  for (int i = threadIdx.x; i < N / 2; i += NLTHREADS) pairs[i] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < npl * kNlInterp; i += NLTHREADS) {
    const int e = i / kNlInterp, jb = i - e * kNlInterp;
    pairs[A.ig[(size_t)(pl[e] & 0xffff) * 3 * kNlInterp + kNlInterp + jb] >> 1] = 1;
  }
  __syncthreads();
  ShflFft<T, N> F;
  if constexpr (ShflCfg<N>::ok) F.init(tw);
  const int ncell = A.gcount[z];
  const int* gcell = A.gcell + (size_t)z * A.tcap;
  const int* goff = A.goff + (size_t)z * (A.tcap + 1);
  const int* gent = A.gent + (size_t)z * A.tcap;
  const NlVal* tval = A.tval + (size_t)z * A.tcap;
  // the shuffle row transforms only read R, so the untouched cells stay zero
  // for every state; the shared-memory line FFT works in place in R
  constexpr bool RKEEP = ShflCfg<N>::ok;
  if (RKEEP) {
    for (int i = threadIdx.x; i < N * N; i += NLTHREADS) R[i] = (T)0;
  }
  for (int s = s0; s < s1; ++s) {
    if (!RKEEP) {
      for (int i = threadIdx.x; i < N * N; i += NLTHREADS) R[i] = (T)0;
    }
    for (int i = threadIdx.x; i < g.nplane_x * LDY; i += NLTHREADS) plane[i] = mk<T>(0, 0);
    __syncthreads();
    // each touched cell: sum over its atoms in list order of Z Mn (the order a
    // serial scatter atom after atom would add them)
    const double* zss = zs + (size_t)s * A.natm;
    for (int c = threadIdx.x; c < ncell; c += NLTHREADS) {
      double v = 0.0;
      for (int k = goff[c]; k < goff[c + 1]; ++k) {
        const int i = gent[k];
        v += zss[pl[i >> 6] & 0xffff] * tval[i].mn;
      }
      R[gcell[c]] = (T)v;
    }
    __syncthreads();
    if constexpr (ShflCfg<N>::ok) {
      constexpr int NL = ShflCfg<N>::NL, M = ShflCfg<N>::M, NG = NLTHREADS / NL;
      const int grp = threadIdx.x / NL;
      for (int p0 = 0; p0 < N / 2; p0 += NG) {
        const int pp = p0 + grp;
        const bool act = pp < N / 2 && pairs[pp];
        if (!__any_sync(0xffffffffu, act)) continue;  // warp-uniform: the shuffles need all lanes
        const int ya = act ? 2 * pp : 0;
        cplx<T> v[M];
#pragma unroll
        for (int k = 0; k < M; ++k) {
          const int x = F.pos(k);
          v[k] = mk<T>(R[(size_t)ya * N + x], R[(size_t)(ya + 1) * N + x]);
        }
        F.template dit<false>(v, tw);  // R2C, -i sign
        shfl_extract_row<T, N>(v, plane, LDY, g.nplane_x, ya, F, act);
      }
      __syncthreads();
      shfl_columns<T, N, true, false>(plane, LDY, g.nplane_x, F, tw, grp, NG);  // BACKWARD y
      __syncthreads();
    } else {
    for (int pp = warp; pp < N / 2; pp += NW) {
      if (!pairs[pp]) continue;
      const int ya = 2 * pp;
      cplx<T>* row = reinterpret_cast<cplx<T>*>(R + (size_t)ya * N);
      cplx<T> v[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int x = lane + 32 * e;
        if (x < N) v[e] = mk<T>(R[(size_t)ya * N + x], R[(size_t)(ya + 1) * N + x]);
      }
      __syncwarp();
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int x = lane + 32 * e;
        if (x < N) row[x] = v[e];
      }
      __syncwarp();
      fft_line_warp<T, N, false>(row, tw);  // R2C, -i sign
      extract_r2c_row<T, N>(row, plane, g.nplane_x, ya);
    }
    __syncthreads();
    plane_columns<T, N, true>(plane, g.nplane_x, tw);  // FFTW_BACKWARD along y
    __syncthreads();
    }
    cplx<T>* po = pen_out + ((size_t)s * N + z) * g.nlpad;
    for (int l = threadIdx.x; l < g.nlines; l += NLTHREADS) {
      int xy = __ldg(g.line_xy + l);
      po[l] = plane[(xy & 0xffff) * LDY + (xy >> 16)];
    }
    __syncthreads();
  }
}

// sum rho partials over groups, scale by 1/vol
__global__ void k_rho_reduce(const double* __restrict__ part, int ngroups, size_t nr,
                             double scale, double* __restrict__ rho);
__global__ void k_rowsum(const double* __restrict__ part, int ncol, int nrow,
                         double* __restrict__ out);
__global__ void k_to_float(const double* __restrict__ in, float* __restrict__ out, size_t n);

// ---------------------------------------------------------------------------
// host side

template <typename T>
const Twiddles<T>& tws(const cpstep_ctx* c);
template <>
inline const Twiddles<double>& tws<double>(const cpstep_ctx* c) { return c->tw64; }
template <>
inline const Twiddles<float>& tws<float>(const cpstep_ctx* c) { return c->tw32; }

template <typename K>
int set_smem(K kernel, size_t smem) {
  CPSTEP_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
  return CPSTEP_OK;
}

// resident blocks of a plane-pass kernel on this device (blocks per SM x SMs),
// looked up once per context
template <typename K>
int resident_blocks(const cpstep_ctx* c, K kernel, int threads, size_t smem, int* cache) {
  if (*cache > 0) return CPSTEP_OK;
  int per = 0;
  CPSTEP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
  if (per < 1) {
    cpstep_set_error("state FFT: plane-pass kernel does not fit an SM (%zu bytes shared)", smem);
    return CPSTEP_ERR_CUDA;
  }
  *cache = per * c->num_sms;
  return CPSTEP_OK;
}

// state groups for the plane passes: aim at tune.plane_waves (default 3)
// waves of CTAs
inline int plane_groups(const cpstep_ctx* c, int nstates, int other) {
  int target = c->tune.plane_waves * c->num_sms;
  int per = c->nz * other;
  int g = cdiv(target, per);
  return std::max(1, std::min(nstates, g));
}

template <typename T, int N>
struct StateFft {
  static int zfft_fwd(cpstep_ctx* c, const FftJob& j, const double* psi, int nstates,
                      const cplx<T>* twz = nullptr, const double2* mul = nullptr) {
    dim3 grid(cdiv(j.g.nlines, ZShape<N>::LB), nstates);
    const size_t smem = ZShape<N>::template bytes<T>();
    if (int rc = set_smem(k_zfft_fwd<T, N>, smem)) return rc;
    k_zfft_fwd<T, N><<<grid, ZTHREADS, smem, c->stream>>>(
        reinterpret_cast<const double2*>(psi), reinterpret_cast<cplx<T>*>(j.pen_a), j.g,
        twz ? twz : tws<T>(c).z, mul);
    CPSTEP_LAUNCH_CHECK();
    return CPSTEP_OK;
  }

  static int density(cpstep_ctx* c, const double* psi, const double* occ, double* rho) {
    const FftJob j = c->state_job();
    if (int rc = zfft_fwd(c, j, psi, c->nstates)) return rc;
    if constexpr (P16Cfg<N>::ok && sizeof(T) == 4) {
      if (c->tune.shfl == 2) {
        const size_t smem = P16Shape<N, P16_K2_THREADS>::bytes(j.g.nplane_x, j.g.nlines);
        if (int rc = set_smem(k_xy_fwd_p16<N>, smem)) return rc;
        if (int rc = resident_blocks(c, k_xy_fwd_p16<N>, P16_K2_THREADS, smem, &c->p16_blocks_k2))
          return rc;
        const int nb = c->p16_blocks_k2;
        const long long items = (long long)N * c->nstates;
        const int segs = (int)(((items + nb - 1) / nb + c->nstates - 1) / c->nstates) + 1;
        if ((size_t)nb * segs * N * N > c->rho_part_elems) {
          cpstep_set_error("state FFT: density partials need %zu doubles, %zu allocated",
                           (size_t)nb * segs * N * N, c->rho_part_elems);
          return CPSTEP_ERR_CUDA;
        }
        k_xy_fwd_p16<N><<<nb, P16_K2_THREADS, smem, c->stream>>>(
            reinterpret_cast<const cplx<float>*>(j.pen_a), j.g, tws<float>(c).x, occ,
            c->nstates, segs, c->d_rho_part);
        CPSTEP_LAUNCH_CHECK();
        if ((long long)nb > 62LL * N) {  // more blocks on one plane than the reduction lists
          cpstep_set_error("state FFT: %d density blocks over %d planes", nb, N);
          return CPSTEP_ERR_CUDA;
        }
        k_rho_reduce_items<<<dim3(N, cdiv(4 * c->num_sms, N)), 256, 0, c->stream>>>(
            c->d_rho_part, N, c->nstates, nb, segs, 1.0 / c->vol, rho);
        CPSTEP_LAUNCH_CHECK();
        return CPSTEP_OK;
      }
    }
    if constexpr (ShflCfg<N>::ok) {
      if (c->tune.shfl) {
        const size_t smem = SShape<T, N>::bytes(j.g.nplane_x);
        int ng = std::min(c->ngroups_rho, plane_groups(c, c->nstates, 1));
        int spg = cdiv(c->nstates, ng);
        ng = cdiv(c->nstates, spg);
        if (int rc = set_smem(k_xy_fwd_s<T, N, 0>, smem)) return rc;
        k_xy_fwd_s<T, N, 0><<<dim3(N, ng), PTHREADS, smem, c->stream>>>(
            reinterpret_cast<const cplx<T>*>(j.pen_a), j.g, tws<T>(c).x, occ, c->nstates, spg,
            c->d_rho_part);
        CPSTEP_LAUNCH_CHECK();
        size_t nr = (size_t)N * N * N;
        k_rho_reduce<<<2 * c->num_sms, 256, 0, c->stream>>>(c->d_rho_part, ng, nr, 1.0 / c->vol,
                                                            rho);
        CPSTEP_LAUNCH_CHECK();
        return CPSTEP_OK;
      }
    }
    const size_t smem = PShape<T, N>::bytes(j.g.nplane_x);
    const int rows = PShape<T, N>::ROWS;
    int ysplit = cdiv(N, rows);
    int ng = std::min(c->ngroups_rho, plane_groups(c, c->nstates, ysplit));
    int spg = cdiv(c->nstates, ng);
    ng = cdiv(c->nstates, spg);
    if (int rc = set_smem(k_xy_fwd<T, N, 0>, smem)) return rc;
    k_xy_fwd<T, N, 0><<<dim3(N, ng, ysplit), PTHREADS, smem, c->stream>>>(
        reinterpret_cast<const cplx<T>*>(j.pen_a), j.g, tws<T>(c).x, occ, c->nstates, spg, rows,
        c->d_rho_part);
    CPSTEP_LAUNCH_CHECK();
    size_t nr = (size_t)N * N * N;
    k_rho_reduce<<<2 * c->num_sms, 256, 0, c->stream>>>(c->d_rho_part, ng, nr, 1.0 / c->vol, rho);
    CPSTEP_LAUNCH_CHECK();
    return CPSTEP_OK;
  }

  // packed G -> real r for nstates arrays of the job's geometry
  static int g2r(cpstep_ctx* c, const FftJob& j, const double* packed, double* real, int nstates) {
    if (int rc = zfft_fwd(c, j, packed, nstates)) return rc;
    if constexpr (ShflCfg<N>::ok) {
      const size_t smem = SShape<T, N>::bytes(j.g.nplane_x);
      if (int rc = set_smem(k_xy_fwd_s<T, N, 1>, smem)) return rc;
      k_xy_fwd_s<T, N, 1><<<dim3(N, nstates), PTHREADS, smem, c->stream>>>(
          reinterpret_cast<const cplx<T>*>(j.pen_a), j.g, tws<T>(c).x, nullptr, nstates, 1, real);
      CPSTEP_LAUNCH_CHECK();
      return CPSTEP_OK;
    }
    const size_t smem = PShape<T, N>::bytes(j.g.nplane_x);
    if (smem > PShape<T, N>::LIMIT) return split_g2r(c, j, real, nstates);
    if (int rc = set_smem(k_xy_fwd<T, N, 1>, smem)) return rc;
    k_xy_fwd<T, N, 1><<<dim3(N, nstates, 1), PTHREADS, smem, c->stream>>>(
        reinterpret_cast<const cplx<T>*>(j.pen_a), j.g, tws<T>(c).x, nullptr, nstates, 1, N,
        real);
    CPSTEP_LAUNCH_CHECK();
    return CPSTEP_OK;
  }

  // the split plane passes (k_split_cols / k_split_rows) with their buffer
  static int split_buf(cpstep_ctx* c, const FftJob& j, int nstates, cplx<T>** buf) {
    const size_t need = sizeof(cplx<T>) * (size_t)nstates * N * N * j.g.nplane_x;
    if (int rc = split_reserve(c, need)) return rc;
    *buf = reinterpret_cast<cplx<T>*>(c->d_split);
    return CPSTEP_OK;
  }
  static size_t split_smem() { return sizeof(cplx<T>) * (N + (size_t)SPLIT_CW * PlaneLd<N>::value); }
  static int split_g2r(cpstep_ctx* c, const FftJob& j, double* real, int nstates) {
    cplx<T>* tb;
    if (int rc = split_buf(c, j, nstates, &tb)) return rc;
    const size_t sm = split_smem();
    if (int rc = set_smem(k_split_cols<T, N, true>, sm)) return rc;
    k_split_cols<T, N, true><<<dim3(N, cdiv(j.g.nplane_x, SPLIT_CW), nstates), SPLIT_THREADS, sm,
                               c->stream>>>(reinterpret_cast<const cplx<T>*>(j.pen_a), nullptr,
                                            j.g, tws<T>(c).x, tb);
    CPSTEP_LAUNCH_CHECK();
    if (int rc = set_smem(k_split_rows<T, N, true>, sm)) return rc;
    k_split_rows<T, N, true><<<dim3(N, cdiv(N / 2, SPLIT_THREADS / 32), nstates), SPLIT_THREADS,
                               sm, c->stream>>>(nullptr, real, j.g, tws<T>(c).x, tb);
    CPSTEP_LAUNCH_CHECK();
    return CPSTEP_OK;
  }
  static int split_r2g(cpstep_ctx* c, const FftJob& j, const double* f_r, int nstates) {
    cplx<T>* tb;
    if (int rc = split_buf(c, j, nstates, &tb)) return rc;
    const size_t sm = split_smem();
    if (int rc = set_smem(k_split_rows<T, N, false>, sm)) return rc;
    k_split_rows<T, N, false><<<dim3(N, cdiv(N / 2, SPLIT_THREADS / 32), nstates), SPLIT_THREADS,
                                sm, c->stream>>>(f_r, nullptr, j.g, tws<T>(c).x, tb);
    CPSTEP_LAUNCH_CHECK();
    if (int rc = set_smem(k_split_cols<T, N, false>, sm)) return rc;
    k_split_cols<T, N, false><<<dim3(N, cdiv(j.g.nplane_x, SPLIT_CW), nstates), SPLIT_THREADS,
                                sm, c->stream>>>(nullptr, reinterpret_cast<cplx<T>*>(j.pen_b),
                                                 j.g, tws<T>(c).x, tb);
    CPSTEP_LAUNCH_CHECK();
    return CPSTEP_OK;
  }

  static int zfft_bwd(cpstep_ctx* c, const FftJob& j, double* out, const double* psi,
                      const double* occ, int nstates, double scale, int mode) {
    dim3 grid(cdiv(j.g.nlines, ZShape<N>::LB), nstates);
    const size_t smem = ZShape<N>::template bytes<T>();
    if (mode == 0) {
      if (int rc = set_smem(k_zfft_bwd<T, N, 0>, smem)) return rc;
      k_zfft_bwd<T, N, 0><<<grid, ZTHREADS, smem, c->stream>>>(
          reinterpret_cast<const cplx<T>*>(j.pen_b), reinterpret_cast<double2*>(out),
          reinterpret_cast<const double2*>(psi), occ, j.g, tws<T>(c).z, scale, c->ecut_ry,
          c->d_eke_part, nullptr);
    } else {
      if (int rc = set_smem(k_zfft_bwd<T, N, 1>, smem)) return rc;
      k_zfft_bwd<T, N, 1><<<grid, ZTHREADS, smem, c->stream>>>(
          reinterpret_cast<const cplx<T>*>(j.pen_b), reinterpret_cast<double2*>(out), nullptr,
          nullptr, j.g, tws<T>(c).z, scale, 0.0, nullptr, nullptr);
    }
    CPSTEP_LAUNCH_CHECK();
    return CPSTEP_OK;
  }

  static int vpsi(cpstep_ctx* c, const double* psi, const double* vks, const double* occ,
                  double* force, double* eke, int pencils_ready) {
    const FftJob j = c->state_job();
    size_t nr = (size_t)N * N * N;
    if (!pencils_ready) {
      if (int rc = zfft_fwd(c, j, psi, c->nstates)) return rc;
    }
    const T* vt;
    if (sizeof(T) == sizeof(double)) {
      vt = reinterpret_cast<const T*>(vks);
    } else {
      k_to_float<<<2 * c->num_sms, 256, 0, c->stream>>>(vks, reinterpret_cast<float*>(c->d_vks_t), nr);
      CPSTEP_LAUNCH_CHECK();
      vt = reinterpret_cast<const T*>(c->d_vks_t);
    }
    int ng = plane_groups(c, c->nstates, 1);
    int spg = cdiv(c->nstates, ng);
    ng = cdiv(c->nstates, spg);
    bool shfl_done = false;
    if constexpr (P16Cfg<N>::ok && sizeof(T) == 4) {
      if (c->tune.shfl == 2) {
        const size_t smem = P16Shape<N, P16_K3_THREADS>::bytes(j.g.nplane_x, j.g.nlines);
        if (int rc = set_smem(k_xy_bwd_p16<N>, smem)) return rc;
        if (int rc = resident_blocks(c, k_xy_bwd_p16<N>, P16_K3_THREADS, smem, &c->p16_blocks_k3))
          return rc;
        k_xy_bwd_p16<N><<<c->p16_blocks_k3, P16_K3_THREADS, smem, c->stream>>>(
            reinterpret_cast<const cplx<float>*>(j.pen_a), reinterpret_cast<const float*>(vt),
            reinterpret_cast<cplx<float>*>(j.pen_b), j.g, tws<float>(c).x, occ, c->nstates);
        shfl_done = true;
      }
    }
    if constexpr (N == 200 && sizeof(T) == 4) {
      const size_t smem = T20Shape::bytes(j.g.nplane_x, j.g.nlines);
      if (c->tune.shfl == 2 && smem <= 227 * 1024) {  // else the Stockham form below
        if (int rc = set_smem(k_xy_bwd_t20<N>, smem)) return rc;
        if (int rc = resident_blocks(c, k_xy_bwd_t20<N>, T20_K3_THREADS, smem, &c->p16_blocks_k3))
          return rc;
        k_xy_bwd_t20<N><<<c->p16_blocks_k3, T20_K3_THREADS, smem, c->stream>>>(
            reinterpret_cast<const cplx<float>*>(j.pen_a), reinterpret_cast<const float*>(vt),
            reinterpret_cast<cplx<float>*>(j.pen_b), j.g, tws<float>(c).x, occ, c->nstates);
        shfl_done = true;
      }
    }
    if constexpr (ShflCfg<N>::ok) {
      if (c->tune.shfl && !shfl_done) {
        const size_t smem = SShape<T, N>::bytes(j.g.nplane_x);
        if (int rc = set_smem(k_xy_bwd_s<T, N, 0>, smem)) return rc;
        k_xy_bwd_s<T, N, 0><<<dim3(N, ng), PTHREADS, smem, c->stream>>>(
            reinterpret_cast<const cplx<T>*>(j.pen_a), nullptr, vt,
            reinterpret_cast<cplx<T>*>(j.pen_b), j.g, tws<T>(c).x, occ, c->nstates, spg);
        shfl_done = true;
      }
    }
    if (!shfl_done) {
      const size_t smem = PShape<T, N>::bytes(j.g.nplane_x);
      if (int rc = set_smem(k_xy_bwd<T, N, 0>, smem)) return rc;
      k_xy_bwd<T, N, 0><<<dim3(N, ng), PTHREADS, smem, c->stream>>>(
          reinterpret_cast<const cplx<T>*>(j.pen_a), nullptr, vt,
          reinterpret_cast<cplx<T>*>(j.pen_b), j.g, tws<T>(c).x, occ, c->nstates, spg);
    }
    CPSTEP_LAUNCH_CHECK();
    double scale = -2.0 / ((double)N * N * N);
    if (int rc = zfft_bwd(c, j, force, psi, eke ? occ : nullptr, c->nstates, scale, 0)) return rc;
    if (eke) {
      int nblk = cdiv(j.g.nlines, ZShape<N>::LB);
      k_rowsum<<<cdiv(c->nstates, 128), 128, 0, c->stream>>>(c->d_eke_part, nblk, c->nstates, eke);
      CPSTEP_LAUNCH_CHECK();
    }
    return CPSTEP_OK;
  }

  // real r -> packed G (sum_r f(r) e^{+iG.r}) times scale, for the job's geometry
  static int r2g(cpstep_ctx* c, const FftJob& j, const double* f_r, double* fg, int nstates,
                 double scale) {
    if constexpr (ShflCfg<N>::ok) {
      const size_t smem = SShape<T, N>::bytes(j.g.nplane_x);
      if (int rc = set_smem(k_xy_bwd_s<T, N, 1>, smem)) return rc;
      k_xy_bwd_s<T, N, 1><<<dim3(N, nstates), PTHREADS, smem, c->stream>>>(
          nullptr, f_r, nullptr, reinterpret_cast<cplx<T>*>(j.pen_b), j.g, tws<T>(c).x, nullptr,
          nstates, 1);
    } else {
      const size_t smem = PShape<T, N>::bytes(j.g.nplane_x);
      if (smem > PShape<T, N>::LIMIT) {
        if (int rc = split_r2g(c, j, f_r, nstates)) return rc;
        return zfft_bwd(c, j, fg, nullptr, nullptr, nstates, scale, 1);
      }
      if (int rc = set_smem(k_xy_bwd<T, N, 1>, smem)) return rc;
      k_xy_bwd<T, N, 1><<<dim3(N, nstates), PTHREADS, smem, c->stream>>>(
          nullptr, f_r, nullptr, reinterpret_cast<cplx<T>*>(j.pen_b), j.g, tws<T>(c).x, nullptr,
          nstates, 1);
    }
    CPSTEP_LAUNCH_CHECK();
    return zfft_bwd(c, j, fg, nullptr, nullptr, nstates, scale, 1);
  }

  static int gtor(cpstep_ctx* c, const double* psi, double* psi_r, int nstates) {
    return g2r(c, c->state_job(), psi, psi_r, nstates);
  }
  static int rtog(cpstep_ctx* c, const double* f_r, double* fg, int nstates) {
    return r2g(c, c->state_job(), f_r, fg, nstates, 1.0);
  }

  // NL plane kernels: states per block so that N x groups is about six blocks
  // per SM
  static void nl_groups(const cpstep_ctx* c, int nstates, int& spg, int& ng) {
    ng = std::max(1, std::min(nstates, cdiv(c->tune.nl_blocks * c->num_sms, N)));
    spg = cdiv(nstates, ng);
    ng = cdiv(nstates, spg);
  }

  // EES: K1 with the projector, then the NL plane pass with the atom sums
  static int nl_proj(cpstep_ctx* c, const NlJob& j, const double* psi, const double2* dyp,
                     int nstates, double* zpart) {
    const cplx<T>* tw = reinterpret_cast<const cplx<T>*>(j.tw);
    if (int rc = zfft_fwd(c, j.f, psi, nstates, tw, dyp)) return rc;
    const size_t smem = NlShape<T, N>::bytes(j.f.g.nplane_x);
    int spg, ng;
    nl_groups(c, nstates, spg, ng);
    if (int rc = set_smem(k_nl_fwd<T, N>, smem)) return rc;
    k_nl_fwd<T, N><<<dim3(N, ng), NLTHREADS, smem, c->stream>>>(
        reinterpret_cast<const cplx<T>*>(j.f.pen_a), j.f.g, tw, j.A, j.ctype, nstates, spg, zpart);
    CPSTEP_LAUNCH_CHECK();
    return CPSTEP_OK;
  }

  // EES: scatter of the scaled Z, NL plane pass back, K4 into the psi force
  static int nl_force(cpstep_ctx* c, const NlJob& j, const double* zs, const double2* dyp,
                      int nstates, double* fpsi) {
    const cplx<T>* tw = reinterpret_cast<const cplx<T>*>(j.tw);
    const size_t smem = NlShape<T, N>::bytes(j.f.g.nplane_x);
    int spg, ng;
    nl_groups(c, nstates, spg, ng);
    if (int rc = set_smem(k_nl_bwd<T, N>, smem)) return rc;
    k_nl_bwd<T, N><<<dim3(N, ng), NLTHREADS, smem, c->stream>>>(
        reinterpret_cast<cplx<T>*>(j.f.pen_b), j.f.g, tw, j.A, j.ctype, nstates, spg, zs);
    CPSTEP_LAUNCH_CHECK();
    dim3 grid(cdiv(j.f.g.nlines, ZShape<N>::LB), nstates);
    const size_t zsm = ZShape<N>::template bytes<T>();
    if (int rc = set_smem(k_zfft_bwd<T, N, 2>, zsm)) return rc;
    k_zfft_bwd<T, N, 2><<<grid, ZTHREADS, zsm, c->stream>>>(
        reinterpret_cast<const cplx<T>*>(j.f.pen_b), reinterpret_cast<double2*>(fpsi), nullptr,
        nullptr, j.f.g, tw, 1.0, 0.0, nullptr, dyp);
    CPSTEP_LAUNCH_CHECK();
    return CPSTEP_OK;
  }

  static size_t nl_smem(int nplx) { return NlShape<T, N>::bytes(nplx); }

  static StateFftOps ops() {
    StateFftOps o;
    o.nl_proj = &nl_proj;
    o.nl_force = &nl_force;
    o.nl_smem = &nl_smem;
    o.density = &density;
    o.vpsi = &vpsi;
    o.gtor = &gtor;
    o.rtog = &rtog;
    o.g2r = &g2r;
    o.r2g = &r2g;
    o.lb = ZShape<N>::LB;
    return o;
  }
};

}  // namespace sfft

#define CPSTEP_INSTANTIATE_STATEFFT(N)                                         \
  template <>                                                                  \
  StateFftOps statefft_ops<double, N>() { return sfft::StateFft<double, N>::ops(); } \
  template <>                                                                  \
  StateFftOps statefft_ops<float, N>() { return sfft::StateFft<float, N>::ops(); }
