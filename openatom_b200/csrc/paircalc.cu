// PairCalculator products (FP64 SIMT path; the mixed-precision context sends
// them to the tensor-core kernels of paircalc_tc.cu where those apply).
//
//   overlap:      C(i,j) = alpha * sum_p wpt_p Re(conj a_i(p) b_j(p)) (+ beta C)
//                 = the reference's 2 * psi_r^T psi_r with Gx=0 rows scaled by
//                 1/sqrt(2) (ckPairCalculator.C:682-751, multiplyForward 'T','N'
//                 with alpha = 2 for double pack; scaling CP_State_GSpacePlane.C:
//                 1933-1954, :3120-3123).  C is column-major (ld = ldc).
//   backmultiply: out_i(p) = alpha * sum_j M(j,i) in_j(p) + beta * out_i(p),
//                 M column-major: psi.T ('N','N', ckPairCalculator.C:1314) and
//                 the gamma / lambda products (:1358, :1408, :1497).
//   dgemm:        column-major BLAS semantics, the myGEMM wrapper
//                 (ckPairCalculator.C:57-66).
//
// All three run on FP64 SIMT tiles; the overlap is split over K (the
// reference's numChunks K-split, pcCommManager.C:165-172) with a fixed-order
// reduction of the partial tiles, so results are deterministic.
#include <algorithm>
#include <mutex>
#include <cuda.h>
#include "ctx.cuh"

namespace pcalc {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

// C_part[ks] (BM x BN tiles, column-major, ld = M) for the K-slab of split ks.
// A: [M][K] row-major (lda), B: [N][K] row-major (ldb), K counted in reals;
// w (per complex point) multiplies column k by w[k/2] when non-null.
__global__ void __launch_bounds__(NT)
k_overlap_part(const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb,
               const double* __restrict__ w, int M, int N, int K, int kslab,
               double* __restrict__ part) {
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN + 1];
  const int i0 = blockIdx.x * BM, j0 = blockIdx.y * BN, ks = blockIdx.z;
  const int kbeg = ks * kslab, kend = min(K, kbeg + kslab);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4] = {};
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    for (int e = threadIdx.x; e < BM * BK; e += NT) {
      int r = e / BK, c = e % BK;
      int k = k0 + c;
      double av = 0.0, bv = 0.0;
      if (k < kend) {
        if (i0 + r < M) {
          av = A[(size_t)(i0 + r) * lda + k];
          if (w) av *= w[k >> 1];
        }
        if (j0 + r < N) bv = B[(size_t)(j0 + r) * ldb + k];
      }
      As[c][r] = av;
      Bs[c][r] = bv;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[kk][ty + 16 * q];
        b[q] = Bs[kk][tx + 16 * q];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r] += a[q] * b[r];
    }
    __syncthreads();
  }
  double* P = part + (size_t)ks * M * N;
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      int i = i0 + ty + 16 * q, j = j0 + tx + 16 * r;
      if (i < M && j < N) P[(size_t)j * M + i] = acc[q][r];
    }
}

// sym (M == N): C = alpha (P + P^T) / 2 + beta C, summed in the same order for
// (i,j) and (j,i) so the result is exactly symmetric.
__global__ void k_splitk_reduce(const double* __restrict__ part, int nsplit, int M, int N,
                                double alpha, double beta, double* __restrict__ C, int ldc,
                                int sym, const double* __restrict__ diag) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M * N) return;
  int j = e / M, i = e - j * M;
  double s = 0.0;
  if (diag && i == j) {  // the diagonal summed in FP64 elsewhere
    s = diag[i];
  } else if (sym) {
    const size_t e1 = (size_t)min(i, j) * M + max(i, j), e2 = (size_t)max(i, j) * M + min(i, j);
    double s1 = 0.0, s2 = 0.0;
    for (int k = 0; k < nsplit; ++k) {
      s1 += part[(size_t)k * M * N + e1];
      s2 += part[(size_t)k * M * N + e2];
    }
    s = 0.5 * (s1 + s2);
  } else {
    for (int k = 0; k < nsplit; ++k) s += part[(size_t)k * M * N + e];
  }
  double* c = C + (size_t)j * ldc + i;
  *c = alpha * s + (beta == 0.0 ? 0.0 : beta * (*c));
}

// First pass of a long split-K reduction (many partial tiles): group g of
// the nsplit partials summed in order, part2[g][e] (G groups).  The second
// pass is k_splitk_reduce over the G group sums; both orders are fixed.
__global__ void k_splitk_group(const double* __restrict__ part, int nsplit, int G, size_t mn,
                               double* __restrict__ part2) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= mn) return;
  const int g = blockIdx.y;
  const int k0 = (int)((long long)nsplit * g / G), k1 = (int)((long long)nsplit * (g + 1) / G);
  double s = 0.0;
#pragma unroll 8
  for (int k = k0; k < k1; ++k) s += part[(size_t)k * mn + e];
  part2[(size_t)g * mn + e] = s;
}

// column-major C = alpha op(A) op(B) + beta C (reference DGEMM semantics)
__global__ void __launch_bounds__(NT)
k_dgemm(int ta, int tb, int m, int n, int k, double alpha, const double* __restrict__ A, int lda,
        const double* __restrict__ B, int ldb, double beta, double* __restrict__ C, int ldc) {
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN + 1];
  const int i0 = blockIdx.x * BM, j0 = blockIdx.y * BN;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4] = {};
  for (int l0 = 0; l0 < k; l0 += BK) {
    for (int e = threadIdx.x; e < BM * BK; e += NT) {
      int r, c;
      if (ta) { r = e / BK; c = e % BK; } else { c = e / BM; r = e % BM; }
      int i = i0 + r, l = l0 + c;
      double v = 0.0;
      if (i < m && l < k) v = ta ? A[(size_t)i * lda + l] : A[(size_t)l * lda + i];
      As[c][r] = v;
    }
    for (int e = threadIdx.x; e < BN * BK; e += NT) {
      int r, c;
      if (tb) { c = e / BN; r = e % BN; } else { r = e / BK; c = e % BK; }
      int j = j0 + r, l = l0 + c;
      double v = 0.0;
      if (j < n && l < k) v = tb ? B[(size_t)l * ldb + j] : B[(size_t)j * ldb + l];
      Bs[c][r] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[kk][ty + 16 * q];
        b[q] = Bs[kk][tx + 16 * q];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r] += a[q] * b[r];
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      int i = i0 + ty + 16 * q, j = j0 + tx + 16 * r;
      if (i < m && j < n) {
        double* c = C + (size_t)j * ldc + i;
        *c = alpha * acc[q][r] + (beta == 0.0 ? 0.0 : beta * (*c));
      }
    }
}

// ---------------------------------------------------------------------------
// 128 x 128 block tiles: 256 threads, 8 x 8 outputs each (rows ty + 16 i,
// columns tx + 16 j), K chunks of 16 staged through registers into two
// shared buffers so the global loads of chunk k+1 overlap the FMAs of chunk k.
constexpr int TB = 128, TK = 16, TLD = TB + 1;
constexpr size_t T128_SMEM = sizeof(double) * 4 * TK * TLD;  // two operands, two buffers

// C_part[ks] = A[i0:i0+128, kslab] B[j0:j0+128, kslab]^T (A, B row-major [rows][K],
// K in reals; w per complex point scales A).  Column-major partial tiles, ld = M.
__global__ void __launch_bounds__(256, 1)
k_overlap_t128(const double* __restrict__ A, int lda, const double* __restrict__ B, int ldb,
               const double* __restrict__ w, int M, int N, int K, int kslab,
               double* __restrict__ part) {
  extern __shared__ __align__(16) double t128_smem[];
  double (*As)[TK][TLD] = reinterpret_cast<double (*)[TK][TLD]>(t128_smem);
  double (*Bs)[TK][TLD] = reinterpret_cast<double (*)[TK][TLD]>(t128_smem + 2 * TK * TLD);
  const int i0 = blockIdx.x * TB, j0 = blockIdx.y * TB, ks = blockIdx.z;
  const int kbeg = ks * kslab, kend = min(K, kbeg + kslab);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  // loader: 4 double2 of A and of B per thread (row = idx / 8, k pair = idx % 8)
  double2 ra[4], rb[4];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = threadIdx.x + 256 * q;
      const int row = idx >> 3, kp = idx & 7;
      const int k = k0 + 2 * kp;
      double2 va = make_double2(0.0, 0.0), vb = make_double2(0.0, 0.0);
      if (k < kend) {  // kend and k are even: the pair is inside
        if (i0 + row < M) {
          va = *reinterpret_cast<const double2*>(A + (size_t)(i0 + row) * lda + k);
          if (w) {
            const double sw = w[k >> 1];
            va.x *= sw;
            va.y *= sw;
          }
        }
        if (j0 + row < N) vb = *reinterpret_cast<const double2*>(B + (size_t)(j0 + row) * ldb + k);
      }
      ra[q] = va;
      rb[q] = vb;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = threadIdx.x + 256 * q;
      const int row = idx >> 3, kp = idx & 7;
      As[buf][2 * kp][row] = ra[q].x;
      As[buf][2 * kp + 1][row] = ra[q].y;
      Bs[buf][2 * kp][row] = rb[q].x;
      Bs[buf][2 * kp + 1][row] = rb[q].y;
    }
  };
  int buf = 0;
  if (kbeg < kend) {
    load(kbeg);
    store(0);
  }
  __syncthreads();
  for (int k0 = kbeg; k0 < kend; k0 += TK) {
    const bool more = k0 + TK < kend;
    if (more) load(k0 + TK);
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      double a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = As[buf][kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = Bs[buf][kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (more) store(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
  double* P = part + (size_t)ks * M * N;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int r = i0 + ty + 16 * i, c = j0 + tx + 16 * j;
      if (r < M && c < N) P[(size_t)c * M + r] = acc[i][j];
    }
}

// out[i][p] = alpha w[p/2] sum_j Mcm[j + i ldm] in[j][p] + beta out[i][p] on
// 128 (i) x 128 (p) tiles; the inner dimension j runs in chunks of 16.
__global__ void __launch_bounds__(256, 1)
k_backmul_t128(const double* __restrict__ Mcm, int ldm, const double* __restrict__ in, int ldi,
               double* __restrict__ out, int ldo, int nout, int nin, int K, double alpha,
               double beta, const double* __restrict__ w) {
  extern __shared__ __align__(16) double t128_smem[];
  double (*Ms)[TK][TLD] = reinterpret_cast<double (*)[TK][TLD]>(t128_smem);  // [j][i]
  double (*Is)[TK][TLD] = reinterpret_cast<double (*)[TK][TLD]>(t128_smem + 2 * TK * TLD);
  const int p0 = blockIdx.x * TB, i0 = blockIdx.y * TB;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  double2 rm[4], ri[4];
  // M tile: row i (128) x 16 j: idx -> i = idx / 8, j pair = idx % 8 (contiguous j)
  // in tile: 16 j x 128 p: idx -> j = idx / 64, p pair = idx % 64
  auto load = [&](int j0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = threadIdx.x + 256 * q;
      const int i = idx >> 3, jp = idx & 7;
      const int j = j0 + 2 * jp;
      double2 vm = make_double2(0.0, 0.0);
      if (i0 + i < nout) {
        const double* mrow = Mcm + (size_t)(i0 + i) * ldm;
        if (j + 1 < nin) vm = make_double2(mrow[j], mrow[j + 1]);
        else if (j < nin) vm.x = mrow[j];
      }
      rm[q] = vm;
      const int jj = idx >> 6, pp = idx & 63;
      const int jr = j0 + jj, p = p0 + 2 * pp;
      double2 vi = make_double2(0.0, 0.0);
      if (jr < nin && p < K)  // K even, p even: the pair is inside
        vi = *reinterpret_cast<const double2*>(in + (size_t)jr * ldi + p);
      ri[q] = vi;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = threadIdx.x + 256 * q;
      const int i = idx >> 3, jp = idx & 7;
      Ms[buf][2 * jp][i] = rm[q].x;
      Ms[buf][2 * jp + 1][i] = rm[q].y;
      const int jj = idx >> 6, pp = idx & 63;
      Is[buf][jj][2 * pp] = ri[q].x;
      Is[buf][jj][2 * pp + 1] = ri[q].y;
    }
  };
  int buf = 0;
  load(0);
  store(0);
  __syncthreads();
  for (int j0 = 0; j0 < nin; j0 += TK) {
    const bool more = j0 + TK < nin;
    if (more) load(j0 + TK);
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      double a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = Ms[buf][kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = Is[buf][kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (more) store(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int r = i0 + ty + 16 * i, p = p0 + tx + 16 * j;
      if (r < nout && p < K) {
        double* o = out + (size_t)r * ldo + p;
        const double a = w ? alpha * w[p >> 1] : alpha;
        *o = a * acc[i][j] + (beta == 0.0 ? 0.0 : beta * (*o));
      }
    }
}

}  // namespace pcalc

// ---------------------------------------------------------------------------
// host side

static int t128_attr() {
  static unsigned long long done = 0;  // one bit per device (the attribute is per device)
  int dev = 0;
  CPSTEP_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(__atomic_load_n(&done, __ATOMIC_ACQUIRE) & bit)) {
    CPSTEP_CUDA_TRY(cudaFuncSetAttribute(pcalc::k_overlap_t128,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pcalc::T128_SMEM));
    CPSTEP_CUDA_TRY(cudaFuncSetAttribute(pcalc::k_backmul_t128,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pcalc::T128_SMEM));
    __atomic_or_fetch(&done, bit, __ATOMIC_RELEASE);
  }
  return CPSTEP_OK;
}

int pc_part_reserve(cpstep_ctx* c, size_t need) {
  if (need > c->pc_part_elems) {
    graph_drop(c);  // a captured step may hold the old buffer
    cudaFree(c->d_pc_part);
    c->d_pc_part = nullptr;
    c->pc_part_elems = 0;
    CPSTEP_CUDA_TRY(cudaMalloc(&c->d_pc_part, need * sizeof(double)));
    c->pc_part_elems = need;
  }
  return CPSTEP_OK;
}

int lv_reserve(cpstep_ctx* c, size_t bytes) {
  if (bytes > c->lv_bytes) {
    graph_drop(c);  // a captured step may hold the old buffer
    cudaFree(c->d_lv);
    c->d_lv = nullptr;
    c->lv_bytes = 0;
    CPSTEP_CUDA_TRY(cudaMalloc(&c->d_lv, bytes));
    c->lv_bytes = bytes;
  }
  return CPSTEP_OK;
}

int split_reserve(cpstep_ctx* c, size_t bytes) {
  if (bytes > c->split_bytes) {
    graph_drop(c);  // a captured step may hold the old buffer
    cudaFree(c->d_split);
    c->d_split = nullptr;
    c->split_bytes = 0;
    CPSTEP_CUDA_TRY(cudaMalloc(&c->d_split, bytes));
    c->split_bytes = bytes;
  }
  return CPSTEP_OK;
}

// Partials beyond 32 are first summed in 16 groups (k_splitk_group) into the
// tail of the partial buffer: one thread per element over ~150 partials is
// bound by the latency of its loads.
static int splitk_groups(int nsplit) { return nsplit > 32 ? 16 : 0; }

size_t pc_part_need(int nsplit, size_t mn) {
  return (size_t)(nsplit + splitk_groups(nsplit)) * mn;
}

int pc_splitk_reduce_launch(cpstep_ctx* c, int nsplit, int M, int N, double alpha, double beta,
                            double* C, int ldc, int sym, const double* diag) {
  const size_t mn = (size_t)M * N;
  const int G = splitk_groups(nsplit);
  const double* part = c->d_pc_part;
  if (G) {
    if (c->pc_part_elems < pc_part_need(nsplit, mn)) {
      cpstep_set_error("split-K reduction: partial buffer reserved without its group sums");
      return CPSTEP_ERR_STATE;
    }
    double* part2 = c->d_pc_part + (size_t)nsplit * mn;
    pcalc::k_splitk_group<<<dim3((unsigned)((mn + 255) / 256), G), 256, 0, c->stream>>>(
        c->d_pc_part, nsplit, G, mn, part2);
    CPSTEP_LAUNCH_CHECK();
    part = part2;
    nsplit = G;
  }
  pcalc::k_splitk_reduce<<<cdiv(M * N, 256), 256, 0, c->stream>>>(part, nsplit, M, N, alpha,
                                                                   beta, C, ldc, sym, diag);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

int pc_overlap_launch(cpstep_ctx* c, const double* a, const double* b, int M, int N, int K,
                      const double* w, double alpha, double beta, double* C, int ldc) {
  using namespace pcalc;
  bool used = false;
  if (int rc = pc_overlap_tc_launch(c, a, b, M, N, K, w, alpha, beta, C, ldc, &used)) return rc;
  if (used) return CPSTEP_OK;
  if (int rc = t128_attr()) return rc;
  int tm = cdiv(M, TB), tn = cdiv(N, TB);
  int want = std::max(1, c->tune.pc_split * c->num_sms / (tm * tn));
  int kslab = cdiv(cdiv(K, want), TK) * TK;
  int nsplit = cdiv(K, kslab);
  if (int rc = pc_part_reserve(c, pc_part_need(nsplit, (size_t)M * N))) return rc;
  k_overlap_t128<<<dim3(tm, tn, nsplit), 256, T128_SMEM, c->stream>>>(a, K, b, K, w, M, N, K,
                                                                     kslab, c->d_pc_part);
  CPSTEP_LAUNCH_CHECK();
  return pc_splitk_reduce_launch(c, nsplit, M, N, alpha, beta, C, ldc, 0);
}

int pc_backmul_launch(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                      double* out, int ldo, int nout, int nin, int K, double alpha, double beta) {
  using namespace pcalc;
  bool used = false;
  if (int rc = pc_backmul_tc_launch(c, Mcm, ldm, in, ldi, out, ldo, nout, nin, K, alpha, beta,
                                    nullptr, &used))
    return rc;
  if (used) return CPSTEP_OK;
  if (int rc = t128_attr()) return rc;
  dim3 grid(cdiv(K, TB), cdiv(nout, TB));
  k_backmul_t128<<<grid, 256, T128_SMEM, c->stream>>>(Mcm, ldm, in, ldi, out, ldo, nout, nin, K,
                                                      alpha, beta, nullptr);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

int pc_backmul_w_launch(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                        double* out, int ldo, int nout, int nin, int K, double alpha, double beta,
                        const double* w) {
  using namespace pcalc;
  bool used = false;
  if (int rc = pc_backmul_tc_launch(c, Mcm, ldm, in, ldi, out, ldo, nout, nin, K, alpha, beta, w,
                                    &used))
    return rc;
  if (used) return CPSTEP_OK;
  if (int rc = t128_attr()) return rc;
  dim3 grid(cdiv(K, TB), cdiv(nout, TB));
  k_backmul_t128<<<grid, 256, T128_SMEM, c->stream>>>(Mcm, ldm, in, ldi, out, ldo, nout, nin, K,
                                                      alpha, beta, w);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

int dgemm_launch(cudaStream_t s, int ta, int tb, int m, int n, int k, double alpha,
                 const double* A, int lda, const double* B, int ldb, double beta, double* C,
                 int ldc) {
  using namespace pcalc;
  dim3 grid(cdiv(m, BM), cdiv(n, BN));
  k_dgemm<<<grid, NT, 0, s>>>(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the overlap product (cpstep_pc_overlap_noalloc).
//
// For callers that cannot allocate device memory: the split-K partial tiles go
// to a fixed array compiled into the library instead of context scratch.  The
// array exists on every GPU that loads the library, for the life of the
// process.  In host code `g_noalloc_part` names a host-side shadow, not device
// memory, so the kernels get the device address looked up below.

#define CPSTEP_NOALLOC_PART_DOUBLES (1 << 20)  // 8 MiB of partial tiles
static __device__ __align__(256) double g_noalloc_part[CPSTEP_NOALLOC_PART_DOUBLES];

namespace {
std::mutex g_noalloc_mu;
double* g_noalloc_addr[64] = {};            // device address of the array, per device
unsigned long long g_noalloc_ctx[64] = {};  // unique ID of the context it was looked up in
int g_noalloc_sms[64] = {};

// Unique ID of the calling thread's current context (cuCtxGetId: never reused
// within a process), 0 when none is current.  The driver entry points come
// through the runtime, so the library does not link the driver library.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);
unsigned long long current_ctx_id() {
  static PfnCtxGetCurrent get_cur = nullptr;
  static PfnCtxGetId get_id = nullptr;
  if (!get_cur || !get_id) {
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", reinterpret_cast<void**>(&get_cur),
                                cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", reinterpret_cast<void**>(&get_id),
                                cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      get_cur = nullptr;
      get_id = nullptr;
      return 0;
    }
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_cur(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}
}  // namespace

extern "C" int cpstep_pc_overlap_noalloc(const double* d_a, const double* d_b, int na, int nb,
                                         int npts, const double* d_w, double alpha,
                                         double beta, double* d_c, int ldc, void* stream) {
  using namespace pcalc;
  if (!d_a || !d_b || !d_c || na <= 0 || nb <= 0 || npts <= 0 || ldc < na) {
    cpstep_set_error("pc_overlap_noalloc: bad argument");
    return CPSTEP_ERR_ARG;
  }
  if ((size_t)na * nb > CPSTEP_NOALLOC_PART_DOUBLES) {
    cpstep_set_error("pc_overlap_noalloc: na*nb = %zu exceeds the fixed scratch of %d doubles "
                     "(at most %d x %d); use cpstep_pc_overlap",
                     (size_t)na * nb, CPSTEP_NOALLOC_PART_DOUBLES, 1024, 1024);
    return CPSTEP_ERR_ARG;
  }
  int dev = 0;
  CPSTEP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    cpstep_set_error("pc_overlap_noalloc: device index %d out of range", dev);
    return CPSTEP_ERR_ARG;
  }
  double* part = nullptr;
  int nsm = 0;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    const unsigned long long id = current_ctx_id();
    if (!g_noalloc_addr[dev] || id == 0 || id != g_noalloc_ctx[dev]) {
      // once per device and context, with that device current: the address
      // is the array's copy in the current context (a reset of the device's
      // primary context, cudaDeviceReset, makes a new one)
      void* addr = nullptr;
      CPSTEP_CUDA_TRY(cudaGetSymbolAddress(&addr, g_noalloc_part));
      int sms = 0;
      CPSTEP_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      g_noalloc_addr[dev] = static_cast<double*>(addr);
      g_noalloc_ctx[dev] = current_ctx_id();
      g_noalloc_sms[dev] = sms > 0 ? sms : 148;
    }
    part = g_noalloc_addr[dev];
    nsm = g_noalloc_sms[dev];
  }
  const int M = na, N = nb, K = 2 * npts;
  const int tm = cdiv(M, BM), tn = cdiv(N, BN);
  int want = std::max(1, (2 * nsm) / (tm * tn));
  const int fit = (int)std::max<size_t>(1, CPSTEP_NOALLOC_PART_DOUBLES / ((size_t)M * N));
  want = std::min(want, fit);
  int kslab = cdiv(cdiv(K, want), BK) * BK;
  int nsplit = cdiv(K, kslab);
  while ((size_t)nsplit * M * N > CPSTEP_NOALLOC_PART_DOUBLES) {  // rounding of kslab
    kslab += BK;
    nsplit = cdiv(K, kslab);
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // every partial the reduction reads is written by this call: nothing to clear
  k_overlap_part<<<dim3(tm, tn, nsplit), NT, 0, s>>>(d_a, K, d_b, K, d_w, M, N, K, kslab, part);
  CPSTEP_LAUNCH_CHECK();
  k_splitk_reduce<<<cdiv(M * N, 256), 256, 0, s>>>(part, nsplit, M, N, alpha, beta, d_c, ldc, 0,
                                                    nullptr);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}
