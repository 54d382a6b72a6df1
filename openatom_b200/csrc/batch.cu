// Many independent systems stepped by one CUDA graph launch.
//
// The reference runs independent instances side by side as separate Charm++
// object arrays (its multi-instance "uber" indices, main/cpaimd.C and
// uber/Uber.h); here each system is its own context, and a batch captures one
// electronic step of every context into a single graph: a fork event on the
// batch's stream, each context's step on its own stream (a branch of the
// graph), a join back.  The branches share nothing, so the GPU overlaps the
// small systems' kernels, except the contexts' Ortho launches (cooperative,
// with grid-wide barriers), which are chained by events so that no two of
// them are resident at once.  As for the single-context graph: iteration 1 and
// a new argument set run directly (one warm-up step), the next call captures,
// later calls replay while the arguments stay the same; if capture fails the
// batch falls back to direct steps.
#include <vector>

#include "ctx.cuh"

struct cpstep_batch {
  std::vector<cpstep_ctx*> ctx;
  std::vector<cudaStream_t> br;      // one branch stream per context
  std::vector<cudaEvent_t> join;
  std::vector<cudaEvent_t> orth;     // Ortho of context i done (chains the Ortho launches)
  cudaEvent_t fork = nullptr;
  cudaStream_t cap = nullptr;        // capture stream (not the legacy default stream)
  cudaStream_t stream = nullptr;     // where the graph is launched
  std::vector<cpstep_ctx::StepKey> key;
  std::vector<unsigned> gen;         // each context's graph generation at capture
  int warm = 0;
  int use_graph = 1;
  cudaGraphExec_t exec = nullptr;
  unsigned long long kernels = 0;
};

static void batch_drop(cpstep_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->warm = 0;
}

extern "C" {

int cpstep_batch_create(cpstep_batch** out, int n, cpstep_ctx* const* ctxs) {
  if (!out || n <= 0 || !ctxs) return CPSTEP_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (!ctxs[i]) return CPSTEP_ERR_ARG;
  cpstep_batch* b = new cpstep_batch();
  b->ctx.assign(ctxs, ctxs + n);
  b->br.assign(n, nullptr);
  b->join.assign(n, nullptr);
  b->orth.assign(n, nullptr);
  b->key.assign(n, cpstep_ctx::StepKey{});
  b->gen.assign(n, 0u);
  cudaError_t e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    e = cudaStreamCreateWithFlags(&b->br[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->orth[i], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    cpstep_batch_destroy(b);
    cpstep_set_error("batch_create: %s", cudaGetErrorString(e));
    return CPSTEP_ERR_CUDA;
  }
  *out = b;
  return CPSTEP_OK;
}

int cpstep_batch_destroy(cpstep_batch* b) {
  if (!b) return CPSTEP_OK;
  batch_drop(b);
  for (auto s : b->br)
    if (s) cudaStreamDestroy(s);
  for (auto ev : b->join)
    if (ev) cudaEventDestroy(ev);
  for (auto ev : b->orth)
    if (ev) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
  return CPSTEP_OK;
}

int cpstep_batch_set_stream(cpstep_batch* b, void* stream) {
  if (!b) return CPSTEP_ERR_ARG;
  b->stream = reinterpret_cast<cudaStream_t>(stream);
  return CPSTEP_OK;
}

int cpstep_batch_set_graph(cpstep_batch* b, int enable) {
  if (!b || (enable != 0 && enable != 1)) return CPSTEP_ERR_ARG;
  batch_drop(b);
  b->use_graph = enable;
  return CPSTEP_OK;
}

int cpstep_batch_status(cpstep_batch* b, int* enabled, int* captured,
                        unsigned long long* kernels) {
  if (!b) return CPSTEP_ERR_ARG;
  if (enabled) *enabled = b->use_graph;
  if (captured) *captured = b->exec != nullptr;
  if (kernels) *kernels = b->kernels;
  return CPSTEP_OK;
}

int cpstep_batch_step(cpstep_batch* b, double* const* psi, double* const* vpsi,
                      const double* const* occ, double dt, int iteration,
                      double* const* energies, double* const* atom_force) {
  if (!b || !psi || !vpsi || !occ || !energies || iteration < 1) return CPSTEP_ERR_ARG;
  const int n = (int)b->ctx.size();
  for (int i = 0; i < n; ++i) {
    cpstep_ctx* c = b->ctx[i];
    if (!psi[i] || !vpsi[i] || !occ[i] || !energies[i]) return CPSTEP_ERR_ARG;
    if (c->atoms.natm <= 0 || !c->d_cmass) {
      cpstep_set_error("batch_step: atoms and CP masses must be set on context %d", i);
      return CPSTEP_ERR_STATE;
    }
  }
  auto direct = [&]() -> int {  // each context on its own stream, ordered after b->stream
    CPSTEP_CUDA_TRY(cudaEventRecord(b->fork, b->stream));
    for (int i = 0; i < n; ++i) {
      cpstep_ctx* c = b->ctx[i];
      const cudaStream_t user = c->stream;
      CPSTEP_CUDA_TRY(cudaStreamWaitEvent(b->br[i], b->fork, 0));
      c->stream = b->br[i];
      c->ortho_wait = i > 0 ? b->orth[i - 1] : nullptr;
      c->ortho_signal = b->orth[i];
      const int rc = step_run(c, psi[i], vpsi[i], occ[i], dt, iteration, energies[i],
                              atom_force ? atom_force[i] : nullptr, 0);
      c->ortho_wait = c->ortho_signal = nullptr;
      c->stream = user;
      if (rc) return rc;
      CPSTEP_CUDA_TRY(cudaEventRecord(b->join[i], b->br[i]));
      CPSTEP_CUDA_TRY(cudaStreamWaitEvent(b->stream, b->join[i], 0));
    }
    return CPSTEP_OK;
  };
  bool prof = false;
  for (int i = 0; i < n; ++i) prof = prof || b->ctx[i]->profile;
  if (!b->use_graph || iteration <= 1 || prof) return direct();
  std::vector<cpstep_ctx::StepKey> key(n);
  for (int i = 0; i < n; ++i)
    key[i] = cpstep_ctx::StepKey{psi[i], vpsi[i], occ[i], dt, energies[i],
                                 atom_force ? atom_force[i] : nullptr};
  // same arguments, and no context changed what a captured step holds
  bool same = true;
  for (int i = 0; i < n; ++i) same = same && key[i] == b->key[i] && b->ctx[i]->gen == b->gen[i];
  if (b->exec && same) {
    CPSTEP_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    __atomic_add_fetch(&g_cpstep_launches, b->kernels, __ATOMIC_RELAXED);
    return CPSTEP_OK;
  }
  if (!b->warm || !same) {
    batch_drop(b);
    const int rc = direct();
    if (!rc) {
      b->warm = 1;
      b->key = key;
      for (int i = 0; i < n; ++i) b->gen[i] = b->ctx[i]->gen;
    }
    return rc;
  }
  // capture: fork from the capture stream into every branch, join back
  const unsigned long long n0 = cpstep_launch_count();
  int rc = CPSTEP_OK;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) e = cudaEventRecord(b->fork, b->cap);
  for (int i = 0; i < n && e == cudaSuccess && !rc; ++i) {
    cpstep_ctx* c = b->ctx[i];
    const cudaStream_t user = c->stream;
    e = cudaStreamWaitEvent(b->br[i], b->fork, 0);
    if (e != cudaSuccess) break;
    c->stream = b->br[i];
    c->ortho_wait = i > 0 ? b->orth[i - 1] : nullptr;
    c->ortho_signal = b->orth[i];
    rc = step_run(c, psi[i], vpsi[i], occ[i], dt, iteration, energies[i],
                  atom_force ? atom_force[i] : nullptr, 0);
    c->ortho_wait = c->ortho_signal = nullptr;
    c->stream = user;
    if (!rc) e = cudaEventRecord(b->join[i], b->br[i]);
    if (!rc && e == cudaSuccess) e = cudaStreamWaitEvent(b->cap, b->join[i], 0);
  }
  const cudaError_t e2 = cudaStreamEndCapture(b->cap, &g);
  if (e == cudaSuccess) e = e2;
  const unsigned long long nk = cpstep_launch_count() - n0;
  __atomic_sub_fetch(&g_cpstep_launches, nk, __ATOMIC_RELAXED);  // captured, not run
  cudaGraphExec_t x = nullptr;
  if (!rc && e == cudaSuccess && g) e = cudaGraphInstantiate(&x, g, 0);
  if (g) cudaGraphDestroy(g);
  if (rc || e != cudaSuccess || !x) {
    cudaGetLastError();
    if (x) cudaGraphExecDestroy(x);
    b->use_graph = 0;
    return direct();
  }
  b->exec = x;
  b->kernels = nk;
  for (int i = 0; i < n; ++i) b->gen[i] = b->ctx[i]->gen;
  CPSTEP_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
  __atomic_add_fetch(&g_cpstep_launches, b->kernels, __ATOMIC_RELAXED);
  return CPSTEP_OK;
}

}  // extern "C"
