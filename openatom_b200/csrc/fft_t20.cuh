// Two-stage line FFT for N = 200 = 20 x 10: R = 10 threads hold one line, 20
// elements each, and exchange once through a per-line shared-memory scratch
// (the N = 200 counterpart of fft_p16.cuh; three line groups per warp, lanes
// 30 and 31 idle).
//
//   stride layout: slot k of thread t is element t + R k          (k < 20)
//   block layout:  slot h R + m of thread t is element (H t + h) + 20 m
//                  (H = 2, h < H, m < R)
//
// s2b: X[k' + 20 m] = sum_t W_R^{t m} [W_N^{t k'} sum_k x[t + R k] W_20^{k k'}]
//   a length-20 DFT in registers, a per-thread twiddle, the exchange, H
//   length-10 DFTs.
// b2s: Z[a + R b] = sum_k' W_20^{k' b} [W_N^{k' a} sum_m y[k' + 20 m] W_R^{m a}]
//   H length-10 DFTs, a twiddle, the exchange, a length-20 DFT.
// Scratch index i is stored at i + i / 20 (reads at a stride of 21 elements
// fall on distinct bank pairs).  Sign: INV = false is exp(-2 pi i jk/N).
#pragma once
#include "fft_smem.cuh"

// cos and sin of 18 m degrees: the W_20 twiddles (W_20^m = c - i s)
#define K_C18 0.95105651629515357212 /* cos 18 = sin 72 */
#define K_S18 0.30901699437494742410 /* sin 18 = cos 72 */
#define K_C36 0.80901699437494742410 /* cos 36          */
#define K_S36 0.58778525229247312917 /* sin 36          */

template <typename T, bool INV>
__device__ __forceinline__ cplx<T> w20(cplx<T> a, int m) {
  cplx<T> w;
  switch (m) {  // m = n2 k1 of the 4 x 5 split: 1..4, 6, 8, 9, 12
    case 1: w = mk<T>((T)K_C18, (T)-K_S18); break;
    case 2: w = mk<T>((T)K_C36, (T)-K_S36); break;
    case 3: w = mk<T>((T)K_S36, (T)-K_C36); break;
    case 4: w = mk<T>((T)K_S18, (T)-K_C18); break;
    case 6: w = mk<T>((T)-K_S18, (T)-K_C18); break;
    case 8: w = mk<T>((T)-K_C36, (T)-K_S36); break;
    case 9: w = mk<T>((T)-K_C18, (T)-K_S18); break;
    case 12: w = mk<T>((T)-K_C36, (T)K_S36); break;
    default: return a;
  }
  return INV ? cmulc(a, w) : cmul(a, w);
}

// 20-point DFT as 4 x 5: with n = 4 n1 + n2 and k = k1 + 5 k2,
//   X[k1 + 5 k2] = sum_n2 W_4^{n2 k2} [W_20^{n2 k1} DFT5_n1(x[4 n1 + n2])(k1)]
template <typename T, bool INV>
__device__ __forceinline__ void dft20(cplx<T> (&v)[20]) {
  cplx<T> a[4][5];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
#pragma unroll
    for (int n1 = 0; n1 < 5; ++n1) a[n2][n1] = v[4 * n1 + n2];
    Dft<T, 5, INV>::template run<20>(a[n2], nullptr);
#pragma unroll
    for (int k1 = 1; k1 < 5; ++k1)
      if (n2) a[n2][k1] = w20<T, INV>(a[n2][k1], n2 * k1);
  }
#pragma unroll
  for (int k1 = 0; k1 < 5; ++k1) {
    cplx<T> b[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    Dft<T, 4, INV>::template run<20>(b, nullptr);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 5 * k2] = b[k2];
  }
}

// 10-point DFT as 2 x 5: X[k1 + 5 k2] = sum_n2 (-1)^{n2 k2} [W_10^{n2 k1} DFT5_n1(x[2 n1 + n2])(k1)]
template <typename T, bool INV>
__device__ __forceinline__ void dft10(cplx<T> (&v)[10]) {
  cplx<T> a[2][5];
#pragma unroll
  for (int n2 = 0; n2 < 2; ++n2) {
#pragma unroll
    for (int n1 = 0; n1 < 5; ++n1) a[n2][n1] = v[2 * n1 + n2];
    Dft<T, 5, INV>::template run<10>(a[n2], nullptr);
  }
#pragma unroll
  for (int k1 = 1; k1 < 5; ++k1) a[1][k1] = w20<T, INV>(a[1][k1], 2 * k1);  // W_10^k1
#pragma unroll
  for (int k1 = 0; k1 < 5; ++k1) {
    v[k1] = a[0][k1] + a[1][k1];
    v[k1 + 5] = a[0][k1] - a[1][k1];
  }
}

struct T20Cfg {
  static constexpr int N = 200, P = 20, R = 10, H = 2;
  static constexpr int LPW = 3;             // line groups per warp (lanes 30, 31 idle)
  static constexpr int SCR = N + N / P;     // scratch elements per line
};

__device__ __forceinline__ int t20_pad(int i) { return i + i / 20; }

// The two-stage transform of one line group's thread; the s2b twiddles kept
// factored (W_N^{t k} = W_N^{t (k % 4)} W_N^{4 t (k / 4)}), the b2s ones as
// W_N^{H t a} times W_N^{h a} from the shared table.
template <typename T>
struct T20Fft {
  using C = T20Cfg;
  static constexpr int N = C::N, P = C::P, R = C::R, H = C::H;
  cplx<T> wa[4], wb[5];  // W_N^{t j} (j < 4), W_N^{4 t j} (j < 5)
  cplx<T> w2[R];         // W_N^{H t a}
  const cplx<T>* tws;    // the shared W_N^m table
  int t;                 // thread within the line group

  __device__ __forceinline__ void init(const cplx<T>* tw) {
    const int lane = threadIdx.x & 31;
    t = lane < C::LPW * R ? lane % R : lane - C::LPW * R;
    tws = tw;
#pragma unroll
    for (int j = 0; j < 4; ++j) wa[j] = tw[(t * j) % N];
#pragma unroll
    for (int j = 0; j < 5; ++j) wb[j] = tw[(4 * t * j) % N];
#pragma unroll
    for (int a = 0; a < R; ++a) w2[a] = tw[(H * t * a) % N];
  }

  __device__ __forceinline__ cplx<T> tw1(int k) const {
    return (k & 3) ? ((k >> 2) ? cmul(wa[k & 3], wb[k >> 2]) : wa[k & 3]) : wb[k >> 2];
  }

  template <bool INV>
  __device__ __forceinline__ static cplx<T> mulw(cplx<T> a, cplx<T> w) {
    return INV ? cmulc(a, w) : cmul(a, w);
  }

  // position (element index) of block-layout slot s of this thread
  __device__ __forceinline__ int bpos(int s) const { return H * t + s / R + P * (s % R); }

  template <bool INV>
  __device__ __forceinline__ void s2b(cplx<T> (&v)[P], cplx<T>* scr) const {
    dft20<T, INV>(v);
#pragma unroll
    for (int k = 1; k < P; ++k) v[k] = mulw<INV>(v[k], tw1(k));
    __syncwarp();
#pragma unroll
    for (int k = 0; k < P; ++k) scr[t20_pad(k * R + t)] = v[k];
    __syncwarp();
#pragma unroll
    for (int h = 0; h < H; ++h) {
      cplx<T> u[R];
#pragma unroll
      for (int s = 0; s < R; ++s) u[s] = scr[t20_pad((H * t + h) * R + s)];
      dft10<T, INV>(u);
#pragma unroll
      for (int m = 0; m < R; ++m) v[h * R + m] = u[m];
    }
  }

  template <bool INV>
  __device__ __forceinline__ void b2s(cplx<T> (&v)[P], cplx<T>* scr) const {
#pragma unroll
    for (int h = 0; h < H; ++h) {
      cplx<T> u[R];
#pragma unroll
      for (int m = 0; m < R; ++m) u[m] = v[h * R + m];
      dft10<T, INV>(u);
#pragma unroll
      for (int a = 0; a < R; ++a)
        v[h * R + a] = a ? mulw<INV>(u[a], h ? cmul(w2[a], tws[(h * a) % N]) : w2[a]) : u[a];
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < H; ++h)
#pragma unroll
      for (int a = 0; a < R; ++a) scr[t20_pad((H * t + h) * R + a)] = v[h * R + a];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < P; ++k) v[k] = scr[t20_pad(k * R + t)];
    dft20<T, INV>(v);
  }
};
