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

// 16-point DFT as 4 x 4: X[k1 + 4 k2] = sum_n2 W16^(n2 k1) W4^(n2 k2) [DFT4 over n1
// of x[4 n1 + n2]](k1).  W16 constants: cos(pi/8) = sqrt(2 + sqrt2)/2,
// sin(pi/8) = sqrt(2 - sqrt2)/2.
#define K_C8 0.92387953251128675613   /* cos(pi/8) */
#define K_S8 0.38268343236508977173   /* sin(pi/8) */
template <typename T, bool INV>
struct Dft<T, 16, INV> {
  // multiply by W16^e (forward e^{-2 pi i e/16}; INV: conjugate), e in 0..9
  static __device__ __forceinline__ cplx<T> w16(cplx<T> a, int e) {
    const T c = (T)K_C8, s = (T)K_S8, r = (T)K_R2;
    cplx<T> w;
    switch (e) {
      case 1: w = mk<T>(c, -s); break;
      case 2: w = mk<T>(r, -r); break;
      case 3: w = mk<T>(s, -c); break;
      case 4: return mul_i(a, INV);
      case 6: w = mk<T>(-r, -r); break;
      case 9: w = mk<T>(-c, s); break;
      default: return a;
    }
    return INV ? cmulc(a, w) : cmul(a, w);
  }
  template <int N>
  static __device__ __forceinline__ void run(cplx<T>* v, const cplx<T>* tw) {
    // DFT4 over n1 in place: element k1 of column n2 lands in v[4 k1 + n2]
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      cplx<T> a[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
      Dft<T, 4, INV>::template run<N>(a, tw);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) v[4 * k1 + n2] = w16(a[k1], n2 * k1);
    }
    // DFT4 over n2 in place: X[k1 + 4 k2] lands in v[4 k1 + k2]
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) Dft<T, 4, INV>::template run<N>(v + 4 * k1, tw);
    // transpose 4 x 4 (register renaming)
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = i + 1; j < 4; ++j) {
        cplx<T> t = v[4 * i + j];
        v[4 * i + j] = v[4 * j + i];
        v[4 * j + i] = t;
      }
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

// ---------------------------------------------------------------------------
// Two-stage warp FFT for N = 16 * M2: a radix-16 stage, then a radix-M2 stage,
// on up to L = 32 / M2 lines at a time per warp (lines base + i*ld).  The
// stage-1 output goes to the line buffer padded by one element every 16
// (index i -> i + i/16), so ld must be >= N + N/16; with ld = 8 (mod 16)
// complex elements neither stage has shared-memory bank conflicts for the
// FP32 and FP64 access widths.  Input and output are in natural order.
template <int N>
struct Fft16Shape {
  // Not selected by the plane kernels for now: with the density accumulators
  // the 512-thread plane kernels run out of their 128 registers and spill, and
  // the one-line-at-a-time Stockham path measured as fast.
  static constexpr bool ok = false && (N % 16 == 0) && (N / 16 >= 2) && (N / 16 <= 8);
  static constexpr int M2 = ok ? N / 16 : 1;
  static constexpr int L = ok ? 32 / M2 : 1;           // lines per warp pass
  static constexpr int PER2 = ok ? (L * 16 + 31) / 32 : 1;  // stage-2 butterflies per lane
  static constexpr int LD = ((N + N / 16 + 7) / 16) * 16 + 8;  // >= N + N/16, = 8 mod 16
};

template <typename T, int N, bool INV>
__device__ __forceinline__ void fft16_lines(cplx<T>* base, int ld, int nl, const cplx<T>* tw,
                                            int lane) {
  using S = Fft16Shape<N>;
  constexpr int M2 = S::M2;
  // stage 1: radix 16, butterfly j < M2 of line li = lane / M2
  {
    const int li = lane / M2, j = lane - li * M2;
    const bool act = (li < S::L) && (li < nl);
    cplx<T> v[16];
    cplx<T>* line = base + (size_t)li * ld;
    if (act) {
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = line[j + M2 * r];
      Dft<T, 16, INV>::template run<N>(v, tw);
    }
    __syncwarp();
    if (act) {
#pragma unroll
      for (int r = 0; r < 16; ++r) line[j * 17 + r] = v[r];  // padded j*16 + r
    }
    __syncwarp();
  }
  // stage 2: radix M2, butterfly j < 16 (twiddle W_N^(r j)), natural-order output.
  // Butterflies t = 0, 1, .. of a lane lie on different lines (b = lane + 32 t,
  // line b / 16), so each t is read, transformed and written on its own.
#pragma unroll 1
  for (int t = 0; t < S::PER2; ++t) {
    const int b = lane + 32 * t;
    const int li = b >> 4, j = b & 15;
    const bool act = (li < nl) && (li < S::L);
    cplx<T>* line = base + (size_t)li * ld;
    cplx<T> v[M2];
    if (act) {
#pragma unroll
      for (int r = 0; r < M2; ++r) {
        cplx<T> a = line[j + 17 * r];
        if (r > 0) {
          cplx<T> w = tw[r * j];
          a = INV ? cmulc(a, w) : cmul(a, w);
        }
        v[r] = a;
      }
      Dft<T, M2, INV>::template run<N>(v, tw);
    }
    __syncwarp();
    if (act) {
#pragma unroll
      for (int r = 0; r < M2; ++r) line[j + 16 * r] = v[r];
    }
    __syncwarp();
  }
}
