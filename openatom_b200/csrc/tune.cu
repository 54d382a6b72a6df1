// Autotuner of a context's launch choices (no reference counterpart: FFTW's
// plan search, FFTW_MEASURE in fftCache.C:252-255, is the nearest relative).
//
// Each knob of cpstep_ctx::Tune is set to each of its candidates in turn, the
// phase it affects is run on the caller's data (one untimed run, then the
// fastest of TUNE_REPS runs timed with CUDA events on the context's stream),
// and the fastest candidate is kept.  Knobs are tuned one after the other in
// the order below, each with the earlier ones already chosen.  Results can
// differ from the default launch choices in rounding only (another FFT form or
// another grouping of the same sums); cpstep_tune_get / cpstep_tune_set let a
// caller record a choice and reuse it, so runs stay reproducible.
#include <vector>

#include "ctx.cuh"

int statefft_density(cpstep_ctx* c, const double* psi, const double* occ, double* rho);
int statefft_vpsi(cpstep_ctx* c, const double* psi, const double* vks, const double* occ,
                  double* force, double* eke, int pencils_ready);

namespace {

constexpr int TUNE_REPS = 3;

template <typename F>
int time_ms(cpstep_ctx* c, F&& run, float* best) {
  cudaEvent_t a, b;
  CPSTEP_CUDA_TRY(cudaEventCreate(&a));
  CPSTEP_CUDA_TRY(cudaEventCreate(&b));
  int rc = run();  // untimed: sets attributes, warms caches
  *best = 1e30f;
  for (int r = 0; r < TUNE_REPS && !rc; ++r) {
    cudaEventRecord(a, c->stream);
    rc = run();
    cudaEventRecord(b, c->stream);
    if (!rc && cudaEventSynchronize(b) == cudaSuccess) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (ms < *best) *best = ms;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (!rc && cudaGetLastError() != cudaSuccess) rc = CPSTEP_ERR_CUDA;
  return rc;
}

// knob <- the fastest of cands for run(); restores the previous value on error
template <typename F>
int pick(cpstep_ctx* c, int* knob, const std::vector<int>& cands, F&& run, float* out_ms) {
  const int keep = *knob;
  int best = keep;
  float best_ms = 1e30f;
  for (int v : cands) {
    *knob = v;
    float ms;
    if (int rc = time_ms(c, run, &ms)) {
      *knob = keep;
      return rc;
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  *knob = best;
  if (out_ms) *out_ms = best_ms;
  return CPSTEP_OK;
}

}  // namespace

extern "C" {

int cpstep_tune_get(const cpstep_ctx* c, int* vals, int n) {
  if (!c || !vals || n < CPSTEP_NTUNE) return CPSTEP_ERR_ARG;
  vals[0] = c->tune.shfl;
  vals[1] = c->tune.plane_waves;
  vals[2] = c->tune.nl_blocks;
  vals[3] = c->tune.pc_split;
  // tensor cores: whether the products use them (only a mixed context does)
  vals[4] = c->precision == CPSTEP_PREC_MIXED ? c->tc_ok : 0;
  vals[5] = c->tune.ees_gspace;
  return CPSTEP_OK;
}

int cpstep_tune_set(cpstep_ctx* c, const int* vals, int n) {
  if (!c || !vals || n < CPSTEP_NTUNE) return CPSTEP_ERR_ARG;
  if ((vals[0] < 0 || vals[0] > 2) || vals[1] < 1 || vals[1] > 64 || vals[2] < 1 ||
      vals[2] > 64 || vals[3] < 1 || vals[3] > 16 || (vals[4] != 0 && vals[4] != 1) ||
      (vals[5] != 0 && vals[5] != 1))
    return CPSTEP_ERR_ARG;
  if (vals[4] && !c->tc_ok) {
    if (int rc = cpstep_set_gemm_path(c, 1)) return rc;
  }
  graph_drop(c);
  c->tune.shfl = vals[0];
  c->tune.plane_waves = vals[1];
  c->tune.nl_blocks = vals[2];
  c->tune.pc_split = vals[3];
  c->tc_ok = vals[4];
  c->tune.ees_gspace = vals[5];
  return CPSTEP_OK;
}

int cpstep_autotune(cpstep_ctx* c, const double* d_psi, const double* d_occ, double* ms_out) {
  if (!c || !d_psi || !d_occ) return CPSTEP_ERR_ARG;
  graph_drop(c);
  const int S = c->nstates;
  const size_t nr = (size_t)c->nx * c->ny * c->nz;
  const size_t ncoef = (size_t)S * c->npts;
  double *rho = nullptr, *force = nullptr, *eke = nullptr, *smat = nullptr, *en = nullptr;
  int rc = CPSTEP_OK;
  auto al = [&](double** p, size_t n) {
    if (!rc && cudaMalloc(p, n * sizeof(double)) != cudaSuccess) rc = CPSTEP_ERR_CUDA;
  };
  al(&rho, nr);
  al(&force, 2 * ncoef);
  al(&eke, S);
  al(&smat, (size_t)S * S);
  al(&en, CPSTEP_NENERGY);
  float ms[CPSTEP_NTUNE] = {0, 0, 0, 0, 0, 0};
  // 1, 2: the state plane passes (density, then V.psi with rho standing in for V)
  auto planes = [&]() -> int {
    if (int r = statefft_density(c, d_psi, d_occ, rho)) return r;
    return statefft_vpsi(c, d_psi, rho, d_occ, force, eke, 1);
  };
  // plane-pass form: 1 register shuffles, 0 shared-memory Stockham, 2 the
  // two-stage form (FP32, N = 32, 64, 128; elsewhere it runs as 1)
  if (!rc) {
    std::vector<int> forms = {1, 0};
    if (c->precision == CPSTEP_PREC_MIXED) forms.push_back(2);
    rc = pick(c, &c->tune.shfl, forms, planes, &ms[0]);
  }
  if (!rc) rc = pick(c, &c->tune.plane_waves, {1, 2, 3, 6}, planes, &ms[1]);
  // 4, 5: the overlap product S (split-K width; tensor cores or FP64 in a mixed context)
  auto ovl = [&]() -> int {
    return pc_overlap_launch(c, d_psi, d_psi, S, S, 2 * c->npts, c->d_wpt, 1.0, 0.0, smat, S);
  };
  if (!rc) rc = pick(c, &c->tune.pc_split, {1, 2}, ovl, &ms[3]);
  if (!rc && c->precision == CPSTEP_PREC_MIXED && c->tc_ok) rc = pick(c, &c->tc_ok, {1, 0}, ovl, &ms[4]);
  // 6, 3: the EES pass: G space or NL-grid FFTs (mixed on the tensor cores), then
  // the FFT path's blocks per SM if it runs
  if (!rc && c->nl.on) {
    auto ees = [&]() -> int {
      CPSTEP_CUDA_TRY(cudaMemsetAsync(force, 0, sizeof(double) * 2 * ncoef, c->stream));
      return nl_run(c, d_psi, d_occ, force, en, nullptr);
    };
    const bool gs = c->nl.gspace_ok && c->precision == CPSTEP_PREC_MIXED && c->tc_ok;
    if (gs) rc = pick(c, &c->tune.ees_gspace, {1, 0}, ees, &ms[5]);
    if (!rc && !(gs && c->tune.ees_gspace)) rc = pick(c, &c->tune.nl_blocks, {3, 6, 12}, ees, &ms[2]);
  }
  if (!rc) rc = cudaStreamSynchronize(c->stream) == cudaSuccess ? CPSTEP_OK : CPSTEP_ERR_CUDA;
  cudaFree(rho);
  cudaFree(force);
  cudaFree(eke);
  cudaFree(smat);
  cudaFree(en);
  graph_drop(c);
  if (ms_out)
    for (int k = 0; k < CPSTEP_NTUNE; ++k) ms_out[k] = ms[k];
  return rc;
}

}  // extern "C"
