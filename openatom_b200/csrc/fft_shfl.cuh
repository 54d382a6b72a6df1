// Register-resident line FFT for N = M * NL: a group of NL lanes (NL a power
// of two, 16 or 32) holds one line, M elements per lane.
//
//   dif: input in natural order, element x = l + NL k in slot k of lane l;
//        output X[k' + M rev(l)] in slot k' of lane l (rev = bit reversal of
//        the lane index over log2 NL bits).
//   dit: input z[k' + M rev(l)] in slot k' of lane l; output in natural order,
//        Z[l + NL k] in slot k of lane l.
//
// With q = k' + M m and x = l + NL k,
//   X[k' + M m] = sum_l W_NL^{l m} [W_N^{l k'} sum_k x[l + NL k] W_M^{k k'}],
// so dif is an in-lane length-M DFT, a per-lane twiddle, then a radix-2
// decimation-in-frequency FFT of length NL across the lanes (shuffles, stages
// d = NL/2 .. 1, bit-reversed output); dit is the same steps reversed
// (decimation in time across the lanes from bit-reversed input, twiddle,
// in-lane DFT).  No shared memory is touched.  Sign convention: forward =
// exp(-2 pi i jk/N) (the twiddle table tw[m] = W_N^m), INV = conjugate.
#pragma once
#include "fft_smem.cuh"

template <int N>
struct ShflCfg {
  static constexpr int NL = (N == 128 || N == 96 || N == 64) ? 32
                            : (N == 80 || N == 48 || N == 32) ? 16 : 0;
  static constexpr bool ok = NL != 0;
  static constexpr int M = ok ? N / NL : 1;
  static constexpr int LOG = NL == 32 ? 5 : 4;
};

__device__ __forceinline__ int rev_bits(int l, int bits) {
  return (int)(__brev((unsigned)l) >> (32 - bits));
}

template <typename T, int N>
struct ShflFft {
  using C = ShflCfg<N>;
  static constexpr int NL = C::NL, M = C::M, LOG = C::LOG;
  cplx<T> twl[M];    // W_N^{l k'}, k' < M
  // per stage d = 2^s: W_{2d}^{l mod d} = W_N^{(l mod d) N / (2d)} on the upper
  // lane of each pair (l & d), 1 on the lower one; sgn = -1 upper, +1 lower.
  // With them a butterfly is the same straight-line code on both lanes.
  cplx<T> twd[LOG];
  T sgn[LOG];
  int l;             // lane within the group

  __device__ __forceinline__ void init(const cplx<T>* tw) {
    l = threadIdx.x & (NL - 1);
#pragma unroll
    for (int k = 0; k < M; ++k) twl[k] = tw[(l * k) % N];
#pragma unroll
    for (int s = 0; s < LOG; ++s) {
      const int d = 1 << s;
      const bool up = (l & d) != 0;
      twd[s] = up ? tw[(l & (d - 1)) * (N / (2 * d))] : mk<T>((T)1, (T)0);
      sgn[s] = up ? (T)-1 : (T)1;
    }
  }

  template <bool INV>
  __device__ __forceinline__ static cplx<T> mulw(cplx<T> a, cplx<T> w) {
    return INV ? cmulc(a, w) : cmul(a, w);
  }
  __device__ __forceinline__ static cplx<T> shfl(cplx<T> a, int d) {
    return mk<T>(__shfl_xor_sync(0xffffffffu, a.x, d), __shfl_xor_sync(0xffffffffu, a.y, d));
  }

  template <bool INV>
  __device__ __forceinline__ void dif(cplx<T> (&v)[M], const cplx<T>* tw) const {
    Dft<T, M, INV>::template run<N>(v, tw);
#pragma unroll
    for (int k = 1; k < M; ++k) v[k] = mulw<INV>(v[k], twl[k]);
    // lower lane: a + b; upper lane: (a - b) W  (a lower value, b upper value)
#pragma unroll
    for (int s = LOG - 1; s >= 0; --s) {
      const int d = 1 << s;
#pragma unroll
      for (int k = 0; k < M; ++k) {
        const cplx<T> p = shfl(v[k], d);
        const cplx<T> t = mk<T>(p.x + sgn[s] * v[k].x, p.y + sgn[s] * v[k].y);
        v[k] = mulw<INV>(t, twd[s]);
      }
    }
  }

  template <bool INV>
  __device__ __forceinline__ void dit(cplx<T> (&v)[M], const cplx<T>* tw) const {
    // lower lane: a + W b; upper lane: a - W b.  The upper lane applies W to
    // its own value before the exchange.
#pragma unroll
    for (int s = 0; s < LOG; ++s) {
      const int d = 1 << s;
#pragma unroll
      for (int k = 0; k < M; ++k) {
        const cplx<T> u = mulw<INV>(v[k], twd[s]);
        const cplx<T> p = shfl(u, d);
        v[k] = mk<T>(p.x + sgn[s] * u.x, p.y + sgn[s] * u.y);
      }
    }
#pragma unroll
    for (int k = 1; k < M; ++k) v[k] = mulw<INV>(v[k], twl[k]);
    Dft<T, M, INV>::template run<N>(v, tw);
  }

  // position of slot k of this lane in the dif output / dit input order
  __device__ __forceinline__ int pos(int k) const { return k + M * rev_bits(l, LOG); }
};

// Storage position of y in a column written back by dif in place (slot k' of
// lane l goes to l + NL k'): y = k' + M rev(l)  ->  rev(y / M) + NL (y % M).
template <int N>
__device__ __forceinline__ int shfl_perm(int y) {
  using C = ShflCfg<N>;
  return rev_bits(y / C::M, C::LOG) + C::NL * (y % C::M);
}
