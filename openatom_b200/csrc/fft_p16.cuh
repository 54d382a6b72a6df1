// Two-stage line FFT for N = 16 R with R | 16 (N = 32, 64, 128): R threads
// hold one line, 16 elements each, and exchange once through a per-line
// shared-memory scratch of N + N/16 elements.
//
//   stride layout: slot k of thread t is element t + R k          (k < 16)
//   block layout:  slot h R + m of thread t is element (H t + h) + 16 m
//                  (H = 16 / R, h < H, m < R)
//
// s2b (stride in, block out), with n = t + R k and q = k' + 16 m:
//   X[k' + 16 m] = sum_t W_R^{t m} [W_N^{t k'} sum_k x[t + R k] W_16^{k k'}]
//   a length-16 DFT in registers, a per-thread twiddle, the exchange, H
//   length-R DFTs.
// b2s (block in, stride out), with j = k' + 16 m and q = a + R b:
//   Z[a + R b] = sum_k' W_16^{k' b} [W_N^{k' a} sum_m y[k' + 16 m] W_R^{m a}]
//   H length-R DFTs, a twiddle, the exchange, a length-16 DFT.
// A transform whose output feeds the other therefore needs no reordering:
// the C2R of a row pair runs s2b, the product with V_KS is formed in block
// layout, the R2C runs b2s and leaves the spectrum in stride layout.
//
// Scratch index i is stored at i + i / 16: the exchanges then touch 8-byte
// words in at most two wavefronts per warp access (writes are consecutive in
// the lane index, reads have a stride of 17 words).  Sign: INV = false is
// exp(-2 pi i jk/N) (the tables hold W_N^m = exp(-2 pi i m/N)), INV = true its
// conjugate.
#pragma once
#include "fft_smem.cuh"

template <int N>
struct P16Cfg {
  static constexpr int R = N / 16;
  static constexpr bool ok = (N % 16 == 0) && R >= 2 && R <= 16 && (16 % R == 0);
  static constexpr int H = ok ? 16 / R : 1;
  static constexpr int LPW = ok ? 32 / R : 1;   // lines per warp
  static constexpr int SCR = N + N / 16;        // scratch elements per line
};

__device__ __forceinline__ int p16_pad(int i) { return i + (i >> 4); }

// Twiddles: s2b multiplies by W_N^{t k} and b2s by W_N^{(H t + h) a}.  The
// b2s ones are kept factored, W_N^{H t a} in registers times W_N^{h a} read
// from the shared table (the same word for every lane: a broadcast).  LEAN =
// true factors the s2b ones too, W_N^{t (k % 4)} W_N^{4 t (k / 4)} (12
// registers instead of 30, one more complex multiply per element), for
// kernels that need their registers for accumulators.
template <typename T, int N, bool LEAN = false>
struct P16Fft {
  using C = P16Cfg<N>;
  static constexpr int R = C::R, H = C::H;
  static constexpr int NW1 = LEAN ? 1 : 16;
  cplx<T> w1[NW1];       // W_N^{t k'}   (s2b twiddles of this thread)
  cplx<T> wa[4], wb[4];  // LEAN: W_N^{t j}, W_N^{4 t j}
  cplx<T> w2[R];         // W_N^{H t a}  (b2s twiddles of this thread, before W_N^{h a})
  const cplx<T>* tws;    // the shared W_N^m table
  int t;                 // thread within the line group

  __device__ __forceinline__ void init(const cplx<T>* tw) {
    t = (threadIdx.x & 31) % R;
    tws = tw;
    if (LEAN) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        wa[j] = tw[(t * j) % N];
        wb[j] = tw[(4 * t * j) % N];
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) w1[k] = tw[(t * k) % N];
    }
#pragma unroll
    for (int a = 0; a < R; ++a) w2[a] = tw[(H * t * a) % N];
  }

  __device__ __forceinline__ cplx<T> tw1(int k) const {
    if (LEAN) return (k & 3) ? ((k >> 2) ? cmul(wa[k & 3], wb[k >> 2]) : wa[k & 3]) : wb[k >> 2];
    return w1[k];
  }

  template <bool INV>
  __device__ __forceinline__ static cplx<T> mulw(cplx<T> a, cplx<T> w) {
    return INV ? cmulc(a, w) : cmul(a, w);
  }

  // position (element index) of block-layout slot s of this thread
  __device__ __forceinline__ int bpos(int s) const { return H * t + s / R + 16 * (s % R); }

  template <bool INV>
  __device__ __forceinline__ void s2b(cplx<T> (&v)[16], cplx<T>* scr) const {
    Dft<T, 16, INV>::template run<N>(v, nullptr);
#pragma unroll
    for (int k = 1; k < 16; ++k) v[k] = mulw<INV>(v[k], tw1(k));
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 16; ++k) scr[p16_pad(k * R + t)] = v[k];
    __syncwarp();
#pragma unroll
    for (int h = 0; h < H; ++h) {
      cplx<T> u[R];
#pragma unroll
      for (int s = 0; s < R; ++s) u[s] = scr[p16_pad((H * t + h) * R + s)];
      Dft<T, R, INV>::template run<N>(u, nullptr);
#pragma unroll
      for (int m = 0; m < R; ++m) v[h * R + m] = u[m];
    }
  }

  template <bool INV>
  __device__ __forceinline__ void b2s(cplx<T> (&v)[16], cplx<T>* scr) const {
#pragma unroll
    for (int h = 0; h < H; ++h) {
      cplx<T> u[R];
#pragma unroll
      for (int m = 0; m < R; ++m) u[m] = v[h * R + m];
      Dft<T, R, INV>::template run<N>(u, nullptr);
#pragma unroll
      for (int a = 0; a < R; ++a)
        v[h * R + a] = a ? mulw<INV>(u[a], h ? cmul(w2[a], tws[(h * a) % N]) : w2[a]) : u[a];
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < H; ++h)
#pragma unroll
      for (int a = 0; a < R; ++a) scr[p16_pad((H * t + h) * R + a)] = v[h * R + a];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = scr[p16_pad(k * R + t)];
    Dft<T, 16, INV>::template run<N>(v, nullptr);
  }
};
