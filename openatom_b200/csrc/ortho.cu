// Ortho: T = (S/2)^(-1/2) by the reference's coupled Schulz iteration, as one
// cooperative kernel (grid-wide barriers between the GEMM phases, so the whole
// iteration is a single launch and the host never synchronises in between).
//
//   CPORTHOG::get_iter_Tmat  src_piny_physics_v1.0/abinito_physics/cp_orthog/cp_lowdin.C:180-265
//   Ortho::start_calc / do_iteration / step_2 / step_3 / tolerance_check /
//   collect_error            src_charm_driver/orthog_ctrl/ortho.C:153-269, :862-985, :109-145
//   A = I, B = S/2;  C = 3I - A B^T;  B <- B C^T / 2;  A <- C A^T / 2;
//   stop when rms(A_old - A_new) <= tol (1e-15) or after max_iter (10) iterations;
//   the reference aborts on failure (cp_lowdin.C:243-250), here a status code.
//
// Mixed precision: the iteration runs in FP32 to a looser tolerance, then an
// FP64 correction against the FP64 S restores T^T (S/2) T = I (k_correct64).
// Optional spectral scaling (mixed path only): B = S/sigma with sigma an upper
// bound of the spectrum (Gershgorin), T = A (sigma/2)^(-1/2); it extends the
// convergence region beyond the reference's eig(S/2) < 2 condition.
//
// Every loop in the kernel has a fixed iteration bound; the only waits are the
// cooperative-groups grid barriers of a cooperative launch.
#include <cooperative_groups.h>
#include <algorithm>
#include <cmath>
#include "ctx.cuh"

namespace cg = cooperative_groups;

namespace orth {

constexpr int TS = 32;   // output tile
constexpr int NT = 256;  // threads: 4 outputs each

// C[i][j] = alpha * sum_k X[i][k] Y[j][k] + (diag ? dval * delta_ij : 0) + (Z ? zs*Z[i][j] : 0)
template <typename T>
__device__ void tile_abt(const T* __restrict__ X, const T* __restrict__ Y, T* __restrict__ C,
                         int n, T alpha, T dval, const T* __restrict__ Z, T zs, int tile,
                         T (*Xs)[TS + 1], T (*Ys)[TS + 1]) {
  const int nt = (n + TS - 1) / TS;
  const int ti = tile / nt, tj = tile % nt;
  const int i0 = ti * TS, j0 = tj * TS;
  const int tx = threadIdx.x % TS, ty = threadIdx.x / TS;  // ty in [0, 8)
  T acc[4] = {0, 0, 0, 0};
  for (int k0 = 0; k0 < n; k0 += TS) {
    for (int e = threadIdx.x; e < TS * TS; e += NT) {
      int r = e / TS, c = e % TS;
      int k = k0 + c;
      Xs[r][c] = (i0 + r < n && k < n) ? X[(size_t)(i0 + r) * n + k] : (T)0;
      Ys[r][c] = (j0 + r < n && k < n) ? Y[(size_t)(j0 + r) * n + k] : (T)0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < TS; ++kk) {
      T yv = Ys[tx][kk];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] += Xs[ty + 8 * q][kk] * yv;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int i = i0 + ty + 8 * q, j = j0 + tx;
    if (i < n && j < n) {
      T v = alpha * acc[q];
      if (i == j) v += dval;
      if (Z) v += zs * Z[(size_t)i * n + j];
      C[(size_t)i * n + j] = v;
    }
  }
}

struct Work {
  int n, max_iter;
  double tol;
  const double* S;  // [n][n] FP64 (symmetric)
  void *A, *B, *C, *A2, *B2;  // working precision
  double *X, *Y, *E;          // FP64 correction buffers (mixed) / output staging
  double* partial;            // [gridDim.x]
  double* T;                  // output [n][n] FP64
  int* status;                // [0] iterations, [1] converged flag
  double* rms;                // final rms
  double sigma;               // spectral scale (2 = reference)
  int newton;                 // FP64 Newton correction after the iteration
};

template <typename T>
__global__ void __launch_bounds__(NT) k_schulz(Work w) {
  cg::grid_group grid = cg::this_grid();
  __shared__ T Xs[TS][TS + 1];
  __shared__ T Ys[TS][TS + 1];
  __shared__ double red[32];
  const int n = w.n, nn = n * n;
  const int ntiles = ((n + TS - 1) / TS) * ((n + TS - 1) / TS);
  T* A = (T*)w.A;
  T* B = (T*)w.B;
  T* C = (T*)w.C;
  T* A2 = (T*)w.A2;
  T* B2 = (T*)w.B2;
  const size_t gtid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t gstride = (size_t)gridDim.x * blockDim.x;
  const double inv_sigma = 1.0 / w.sigma;
  for (size_t e = gtid; e < (size_t)nn; e += gstride) {
    int i = e / n, j = e % n;
    A[e] = (i == j) ? (T)1 : (T)0;
    B[e] = (T)(w.S[e] * inv_sigma);
  }
  grid.sync();
  int it = 0;
  double tol_now = 1.0, prev = 1e300;
  while (tol_now > w.tol && it < w.max_iter) {
    ++it;
    // C = 3I - A B^T
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
      tile_abt<T>(A, B, C, n, (T)-1, (T)3, nullptr, (T)0, t, Xs, Ys);
    grid.sync();
    // B2 = B C^T / 2 ;  A2 = C A^T / 2
    for (int t = blockIdx.x; t < 2 * ntiles; t += gridDim.x) {
      if (t < ntiles) tile_abt<T>(B, C, B2, n, (T)0.5, (T)0, nullptr, (T)0, t, Xs, Ys);
      else tile_abt<T>(C, A, A2, n, (T)0.5, (T)0, nullptr, (T)0, t - ntiles, Xs, Ys);
    }
    grid.sync();
    double loc = 0.0;
    for (size_t e = gtid; e < (size_t)nn; e += gstride) {
      double d = (double)A[e] - (double)A2[e];
      loc += d * d;
    }
    double bs = block_sum(loc, red);
    if (threadIdx.x == 0) w.partial[blockIdx.x] = bs;
    grid.sync();
    double tot = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) tot += w.partial[b];  // same order everywhere
    const double r = sqrt(tot / (double)nn);
    // FP32 iteration (mixed path): the coupled iteration loses stability once it
    // has converged to working precision on an ill-conditioned S; stop at the
    // first rise of the update and keep the previous iterate (the FP64
    // correction polishes it).  The FP64 path keeps the reference's rule.
    if (w.newton && prev < 1e-3 && !(r < prev)) {
      grid.sync();
      break;
    }
    prev = r;
    tol_now = r;
    T* t1 = A; A = A2; A2 = t1;
    T* t2 = B; B = B2; B2 = t2;
    grid.sync();  // partials are rewritten next iteration
  }
  // T = A * (sigma/2)^(-1/2); before the FP64 correction the FP32 result is
  // symmetrised, so that W = X (S/2) X below is the matrix T^T (S/2) T tests
  const double post = sqrt(2.0 / w.sigma);
  double* X = w.newton ? w.X : w.T;
  for (size_t e = gtid; e < (size_t)nn; e += gstride) {
    if (w.newton) {
      int i = e / n, j = e % n;
      X[e] = 0.5 * ((double)A[e] + (double)A[(size_t)j * n + i]) * post;
    } else {
      X[e] = (double)A[e] * post;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.status[0] = it;
    // mixed: converged once the FP32 iteration has stagnated below 1e-3 (the
    // FP64 correction takes it from there)
    w.status[1] = (tol_now <= w.tol || (w.newton && tol_now < 1e-3)) ? 1 : 0;
    *w.rms = tol_now;
  }
}

// FP64 correction after an FP32 iteration (cooperative launch): with X the
// FP32 result, W = X (S/2) X is within FP32 rounding of I, and
// T = X W^(-1/2), W^(-1/2) = I - R/2 + 3R^2/8 + O(R^3), R = W - I, satisfies
// T^T (S/2) T = I to FP64 rounding.  T differs from the exact Loewdin
// (S/2)^(-1/2) only by the FP32 error of X (an orbital rotation that leaves
// the density and the energies unchanged).
__global__ void __launch_bounds__(NT) k_correct64(Work w) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double Xs[TS][TS + 1];
  __shared__ double Ys[TS][TS + 1];
  const int n = w.n, nn = n * n;
  const int ntiles = ((n + TS - 1) / TS) * ((n + TS - 1) / TS);
  double* P = w.E + (size_t)nn;  // second FP64 scratch matrix
  // Y = X (S/2)
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    tile_abt<double>(w.X, w.S, w.Y, n, 0.5, 0.0, nullptr, 0.0, t, Xs, Ys);
  grid.sync();
  // E = Y X^T - I = W - I
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    tile_abt<double>(w.Y, w.X, w.E, n, 1.0, -1.0, nullptr, 0.0, t, Xs, Ys);
  grid.sync();
  // P = I - E/2 + 3/8 E E^T
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    tile_abt<double>(w.E, w.E, P, n, 0.375, 1.0, w.E, -0.5, t, Xs, Ys);
  grid.sync();
  // T = X P^T
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    tile_abt<double>(w.X, P, w.T, n, 1.0, 0.0, nullptr, 0.0, t, Xs, Ys);
}

// Gershgorin bound of the spectrum: sigma = max_i sum_j |S_ij|
__global__ void k_gershgorin(const double* __restrict__ S, int n, double* __restrict__ out) {
  __shared__ double red[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += fabs(S[(size_t)i * n + j]);
    m = fmax(m, s);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, red[w]);
    *out = r;
  }
}

}  // namespace orth

// ---------------------------------------------------------------------------

static int ensure(cpstep_ctx* c, double** p, size_t* have, size_t need) {
  if (*have >= need) return CPSTEP_OK;
  graph_drop(c);  // a captured step may hold the old buffer
  cudaFree(*p);
  *p = nullptr;
  CPSTEP_CUDA_TRY(cudaMalloc(p, need * sizeof(double)));
  *have = need;
  return CPSTEP_OK;
}

// T = (S/2)^(-1/2); S, T device [n][n] FP64 (symmetric, so row/column-major agree).
// mixed: FP32 iteration + FP64 Newton step; scale: Gershgorin spectral scaling.
int ortho_tmat(cpstep_ctx* c, const double* S, double* T, int n, int mixed, int scale,
               double tol, int max_iter, int* iters_out, double* rms_out, int check_host) {
  using namespace orth;
  size_t nn = (size_t)n * n;
  // workspace: 5 working matrices (as doubles: enough for either precision), 3 FP64, misc
  size_t need = 9 * nn + 4096 + 8;
  if (int rc = ensure(c, &c->d_ortho_ws, &c->ortho_ws_elems, need)) return rc;
  double* ws = c->d_ortho_ws;
  Work w;
  w.n = n;
  w.max_iter = max_iter;
  w.tol = tol;
  w.S = S;
  w.A = ws;
  w.B = ws + nn;
  w.C = ws + 2 * nn;
  w.A2 = ws + 3 * nn;
  w.B2 = ws + 4 * nn;
  w.X = ws + 5 * nn;
  w.Y = ws + 6 * nn;
  w.E = ws + 7 * nn;
  w.partial = ws + 9 * nn;
  w.T = T;
  w.status = reinterpret_cast<int*>(ws + 9 * nn + 4096);
  w.rms = ws + 9 * nn + 4096 + 2;
  w.newton = mixed ? 1 : 0;
  w.sigma = 2.0;
  double* d_sigma = ws + 9 * nn + 4096 + 4;
  if (scale) {
    orth::k_gershgorin<<<1, 1024, 0, c->stream>>>(S, n, d_sigma);
    CPSTEP_LAUNCH_CHECK();
    double sg = 0.0;
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(&sg, d_sigma, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    w.sigma = std::max(2.0, sg * 1.0001);
  }
  int ntiles = cdiv(n, TS) * cdiv(n, TS);
  int per_sm = 0;
  void* args[] = {&w};
  if (c->ortho_wait) CPSTEP_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ortho_wait, 0));
  if (mixed) {
    CPSTEP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_schulz<float>, NT, 0));
    int nb = std::max(1, std::min(2 * ntiles, per_sm * c->num_sms));
    CPSTEP_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_schulz<float>, nb, NT, args, 0, c->stream));
    int pn = 0;
    CPSTEP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pn, k_correct64, NT, 0));
    int nb2 = std::max(1, std::min(ntiles, pn * c->num_sms));
    CPSTEP_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_correct64, nb2, NT, args, 0, c->stream));
  } else {
    CPSTEP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_schulz<double>, NT, 0));
    int nb = std::max(1, std::min(2 * ntiles, per_sm * c->num_sms));
    CPSTEP_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_schulz<double>, nb, NT, args, 0, c->stream));
  }
  if (c->ortho_signal) CPSTEP_CUDA_TRY(cudaEventRecord(c->ortho_signal, c->stream));
  c->d_ortho_status = w.status;
  if (check_host) {
    int st[2] = {0, 0};
    double r = 0.0;
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(st, w.status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(&r, w.rms, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (iters_out) *iters_out = st[0];
    if (rms_out) *rms_out = r;
    if (!st[1]) {
      cpstep_set_error("Ortho: S^-1/2 iteration not converged in %d iterations (rms %g > %g)",
                       st[0], r, tol);
      return CPSTEP_ERR_NOCONV;
    }
  }
  return CPSTEP_OK;
}
