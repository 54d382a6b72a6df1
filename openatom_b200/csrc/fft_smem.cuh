// Batched mixed-radix Stockham FFT on lines held in shared memory, with the
// line length N a compile-time constant.
//
// Each stage of radix R takes butterfly j of a line from x[j + r*N/R] (r < R),
// twiddles input r by W^(r*(j%Ns)*N/(Ns*R)), runs a length-R DFT and writes
// the results to x[(j/Ns)*Ns*R + j%Ns + r*Ns]; Ns is the product of the radices
// of the earlier stages (Stockham auto-sort, natural order in and out).  The
// stage is done in place: every thread holds its butterflies in registers
// across a __syncthreads between the reads and the writes.  With N, R and Ns
// known at compile time every index is a constant multiply/shift.
//
// Sign conventions follow FFTW-2 as the reference uses it: forward =
// exp(-2 pi i jk/n), backward = exp(+2 pi i jk/n), neither normalised.
#pragma once
#include "common.cuh"

// math constants of the small DFTs (exact values of cos/sin at 2 pi/3, 2 pi/5, 2 pi/8)
#define K_S3 0.86602540378443864676   /* sin(2pi/3) = sqrt(3)/2        */
#define K_C51 0.30901699437494742410  /* cos(2pi/5) = (sqrt5-1)/4      */
#define K_C52 -0.80901699437494742410 /* cos(4pi/5) = -(sqrt5+1)/4     */
#define K_S51 0.95105651629515357212  /* sin(2pi/5)                    */
#define K_S52 0.58778525229247312917  /* sin(4pi/5)                    */
#define K_R2 0.70710678118654752440   /* sqrt(1/2)                     */

// next radix for a remaining length m: 8, 4, 2, then the odd primes
__host__ __device__ constexpr int next_radix(int m) {
  return (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3
         : (m % 5 == 0) ? 5 : (m % 7 == 0) ? 7 : (m % 11 == 0) ? 11 : 0;
}
__host__ __device__ constexpr bool fft_size_ok(int m) {
  return m == 1 ? true : (next_radix(m) == 0 ? false : fft_size_ok(m / next_radix(m)));
}

// In-register DFT of length R.  INV=false: exp(-i...), INV=true: exp(+i...).
template <typename T, int R, bool INV>
struct Dft {
  // generic odd radix via the line's twiddle table: W_R^m = tw[m * N / R]
  template <int N>
  static __device__ __forceinline__ void run(cplx<T>* v, const cplx<T>* tw) {
    cplx<T> o[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      cplx<T> acc = v[0];
#pragma unroll
      for (int j = 1; j < R; ++j) {
        cplx<T> w = tw[((j * k) % R) * (N / R)];
        acc = acc + (INV ? cmulc(v[j], w) : cmul(v[j], w));
      }
      o[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = o[k];
  }
};

template <typename T, bool INV>
struct Dft<T, 2, INV> {
  template <int N>
  static __device__ __forceinline__ void run(cplx<T>* v, const cplx<T>*) {
    cplx<T> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  }
};

template <typename T, bool INV>
struct Dft<T, 3, INV> {
  template <int N>
  static __device__ __forceinline__ void run(cplx<T>* v, const cplx<T>*) {
    cplx<T> t1 = v[1] + v[2];
    cplx<T> t2 = cscale(v[1] - v[2], (T)K_S3);
    cplx<T> m = v[0] + cscale(t1, (T)-0.5);
    v[0] = v[0] + t1;
    // forward: X1 = m - i t2, X2 = m + i t2
    cplx<T> it2 = mul_i(t2, true);
    v[1] = INV ? m + it2 : m - it2;
    v[2] = INV ? m - it2 : m + it2;
  }
};

template <typename T, bool INV>
struct Dft<T, 4, INV> {
  template <int N>
  static __device__ __forceinline__ void run(cplx<T>* v, const cplx<T>*) {
    cplx<T> a = v[0] + v[2], b = v[0] - v[2];
    cplx<T> c = v[1] + v[3], d = v[1] - v[3];
    cplx<T> id = mul_i(d, INV);  // forward: -i d, inverse: +i d
    v[0] = a + c;
    v[2] = a - c;
    v[1] = b + id;
    v[3] = b - id;
  }
};

template <typename T, bool INV>
struct Dft<T, 5, INV> {
  template <int N>
  static __device__ __forceinline__ void run(cplx<T>* v, const cplx<T>*) {
    cplx<T> t1 = v[1] + v[4], t2 = v[2] + v[3];
    cplx<T> t3 = v[1] - v[4], t4 = v[2] - v[3];
    cplx<T> a1 = v[0] + cscale(t1, (T)K_C51) + cscale(t2, (T)K_C52);
    cplx<T> a2 = v[0] + cscale(t1, (T)K_C52) + cscale(t2, (T)K_C51);
    cplx<T> b1 = cscale(t3, (T)K_S51) + cscale(t4, (T)K_S52);
    cplx<T> b2 = cscale(t3, (T)K_S52) - cscale(t4, (T)K_S51);
    cplx<T> ib1 = mul_i(b1, true), ib2 = mul_i(b2, true);
    v[0] = v[0] + t1 + t2;
    if (!INV) {
      v[1] = a1 - ib1; v[4] = a1 + ib1;
      v[2] = a2 - ib2; v[3] = a2 + ib2;
    } else {
      v[1] = a1 + ib1; v[4] = a1 - ib1;
      v[2] = a2 + ib2; v[3] = a2 - ib2;
    }
  }
};

template <typename T, bool INV>
struct Dft<T, 8, INV> {
  template <int N>
  static __device__ __forceinline__ void run(cplx<T>* v, const cplx<T>* tw) {
    cplx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cplx<T> o[4] = {v[1], v[3], v[5], v[7]};
    Dft<T, 4, INV>::template run<N>(e, tw);
    Dft<T, 4, INV>::template run<N>(o, tw);
    // w8^k, forward w8 = (1 - i)/sqrt2
    const T r = (T)K_R2;
    cplx<T> o1 = INV ? mk<T>(r * (o[1].x - o[1].y), r * (o[1].x + o[1].y))
                     : mk<T>(r * (o[1].x + o[1].y), r * (o[1].y - o[1].x));
    cplx<T> o2 = mul_i(o[2], INV);
    cplx<T> o3 = INV ? mk<T>(-r * (o[3].x + o[3].y), r * (o[3].x - o[3].y))
                     : mk<T>(r * (o[3].y - o[3].x), -r * (o[3].x + o[3].y));
    v[0] = e[0] + o[0]; v[4] = e[0] - o[0];
    v[1] = e[1] + o1;   v[5] = e[1] - o1;
    v[2] = e[2] + o2;   v[6] = e[2] - o2;
    v[3] = e[3] + o3;   v[7] = e[3] - o3;
  }
};

// One Stockham stage (radix R, product of earlier radices NS) over `nlines`
// lines of length N (line stride ldl) in smem.  EPT bounds the elements a
// thread holds: nlines*N <= EPT*NT.
template <typename T, int N, int R, int NS, int EPT, int NT, bool INV>
__device__ __forceinline__ void fft_stage(cplx<T>* buf, int ldl, int nlines, const cplx<T>* tw) {
  constexpr int MAXB = (EPT + R - 1) / R;
  constexpr int NBL = N / R;
  constexpr int TSTRIDE = N / (NS * R);
  const int total = nlines * NBL;
  // thread index read through volatile asm: keeps the per-stage index math
  // inside the stage (otherwise it is hoisted out of the callers' loops and
  // stays live in registers across every stage)
  int tid;
  asm volatile("mov.u32 %0, %%tid.x;" : "=r"(tid));
  cplx<T> v[MAXB][R];
  int dsto[MAXB];
#pragma unroll
  for (int b = 0; b < MAXB; ++b) {
    const int idx = tid + b * NT;
    dsto[b] = -1;
    if (idx < total) {
      const int line = idx / NBL;
      const int j = idx - line * NBL;
      const int k = j % NS;
      const cplx<T>* src = buf + line * ldl + j;
      const int ts = k * TSTRIDE;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        cplx<T> a = src[r * NBL];
        if (NS > 1 && r > 0) {
          cplx<T> w = tw[r * ts];
          a = INV ? cmulc(a, w) : cmul(a, w);
        }
        v[b][r] = a;
      }
      Dft<T, R, INV>::template run<N>(v[b], tw);
      dsto[b] = line * ldl + (j - k) * R + k;
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < MAXB; ++b) {
    if (dsto[b] >= 0) {
      cplx<T>* dst = buf + dsto[b];
#pragma unroll
      for (int r = 0; r < R; ++r) dst[r * NS] = v[b][r];
    }
  }
  __syncthreads();
}

template <typename T, int N, int NS, int EPT, int NT, bool INV>
struct FftStages {
  static __device__ __forceinline__ void run(cplx<T>* buf, int ldl, int nlines,
                                             const cplx<T>* tw) {
    constexpr int R = next_radix(N / NS);
    static_assert(R > 0, "FFT length has an unsupported prime factor");
    fft_stage<T, N, R, NS, EPT, NT, INV>(buf, ldl, nlines, tw);
    FftStages<T, N, NS * R, EPT, NT, INV>::run(buf, ldl, nlines, tw);
  }
};
template <typename T, int N, int EPT, int NT, bool INV>
struct FftStages<T, N, N, EPT, NT, INV> {
  static __device__ __forceinline__ void run(cplx<T>*, int, int, const cplx<T>*) {}
};

// ---------------------------------------------------------------------------
// Warp-per-line variant: a warp runs every stage of its own lines with only
// __syncwarp between stages (no block barriers).  Radix 4 first for powers of
// two so that a 128-point stage has 32 butterflies, one per lane.

__host__ __device__ constexpr int next_radix_w(int m) {
  return (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5
         : (m % 7 == 0) ? 7 : (m % 11 == 0) ? 11 : 0;
}

template <typename T, int N, int R, int NS, bool INV>
__device__ __forceinline__ void warp_stage(cplx<T>* line, const cplx<T>* tw, int lane) {
  constexpr int NBL = N / R;
  constexpr int PER = (NBL + 31) / 32;
  constexpr int TSTRIDE = N / (NS * R);
  cplx<T> v[PER][R];
  int dst[PER];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + 32 * b;
    dst[b] = -1;
    if (j < NBL) {
      const int k = j % NS;
      const int ts = k * TSTRIDE;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        cplx<T> a = line[j + r * NBL];
        if (NS > 1 && r > 0) {
          cplx<T> w = tw[r * ts];
          a = INV ? cmulc(a, w) : cmul(a, w);
        }
        v[b][r] = a;
      }
      Dft<T, R, INV>::template run<N>(v[b], tw);
      dst[b] = (j - k) * R + k;
    }
  }
  __syncwarp();
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    if (dst[b] >= 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) line[dst[b] + r * NS] = v[b][r];
    }
  }
  __syncwarp();
}

template <typename T, int N, int NS, bool INV>
struct WarpStages {
  static __device__ __forceinline__ void run(cplx<T>* line, const cplx<T>* tw, int lane) {
    constexpr int R = next_radix_w(N / NS);
    static_assert(R > 0, "FFT length has an unsupported prime factor");
    warp_stage<T, N, R, NS, INV>(line, tw, lane);
    WarpStages<T, N, NS * R, INV>::run(line, tw, lane);
  }
};
template <typename T, int N, bool INV>
struct WarpStages<T, N, N, INV> {
  static __device__ __forceinline__ void run(cplx<T>*, const cplx<T>*, int) {}
};

// One line of length N in smem by the calling warp (all 32 lanes).
template <typename T, int N, bool INV>
__device__ __forceinline__ void fft_line_warp(cplx<T>* line, const cplx<T>* tw) {
  WarpStages<T, N, 1, INV>::run(line, tw, threadIdx.x & 31);
}

// Lines l = warp, warp + nwarps, ... of `nlines` (stride ldl), warp-local only.
template <typename T, int N, bool INV>
__device__ __forceinline__ void fft_lines_warp(cplx<T>* buf, int ldl, int nlines,
                                               const cplx<T>* tw) {
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int l = warp; l < nlines; l += nw) fft_line_warp<T, N, INV>(buf + l * ldl, tw);
}

// Full FFT of `nlines` lines of length N in smem (line stride ldl), in batches
// that respect the EPT register budget.  Called by all NT threads of the block.
template <typename T, int N, int EPT, int NT, bool INV>
__device__ __forceinline__ void fft_lines(cplx<T>* buf, int ldl, int nlines, const cplx<T>* tw) {
  constexpr int CAP = (EPT * NT) / N;
  static_assert(CAP >= 1, "FFT line longer than EPT*NT");
  for (int l0 = 0; l0 < nlines; l0 += CAP) {
    const int nl = min(CAP, nlines - l0);
    FftStages<T, N, 1, EPT, NT, INV>::run(buf + l0 * ldl, ldl, nl, tw);
  }
}
