// C ABI: context management, layout tables, G-space expand/pack and kinetic
// energy entry points.  See include/cpstep.h for the reference routine each
// entry replaces.
#include <stdarg.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "ctx.cuh"

static thread_local char g_err[1024] = {0};
unsigned long long g_cpstep_launches = 0;

void cpstep_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}


namespace {

template <typename T>
int upload(T** dst, const T* src, size_t n) {
  CPSTEP_CUDA_TRY(cudaMalloc(dst, sizeof(T) * std::max<size_t>(n, 1)));
  if (n) CPSTEP_CUDA_TRY(cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice));
  return CPSTEP_OK;
}

bool inv3(const double* h, double* hi, double* det) {
  // column-major 3x3: h[r + 3c]
  double a = h[0], b = h[3], c = h[6], d = h[1], e = h[4], f = h[7], g = h[2], k = h[5], l = h[8];
  double A = e * l - f * k, B = -(d * l - f * g), C = d * k - e * g;
  double dt = a * A + b * B + c * C;
  if (!(std::fabs(dt) > 0)) return false;
  double inv[9] = {A, -(b * l - c * k), b * f - c * e,
                   B, a * l - c * g, -(a * f - c * d),
                   C, -(a * k - b * g), a * e - b * d};
  // inv is row-major (r*3+c); store column-major
  for (int r = 0; r < 3; ++r)
    for (int cc = 0; cc < 3; ++cc) hi[r + 3 * cc] = inv[r * 3 + cc] / dt;
  *det = dt;
  return true;
}

// one block per (line, state): copy the line's packed points into its z-line
__global__ void k_expand(double2* __restrict__ packed, double2* __restrict__ lines,
                         StateGeom g, int expand) {
  int l = blockIdx.x, s = blockIdx.y;
  double2* ps = packed + (size_t)s * g.npts;
  double2* ls = lines + ((size_t)s * g.nlines + l) * g.nz;
  int off = g.line_off[l], nn = g.line_nneg[l], np = g.line_npos[l];
  int zn = g.line_zneg[l], zp = g.line_zpos[l];
  if (expand) {
    for (int z = threadIdx.x; z < g.nz; z += blockDim.x) ls[z] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int q = threadIdx.x; q < nn + np; q += blockDim.x) {
      int z = (q < nn) ? zn + q : zp + (q - nn);
      ls[z] = ps[off + q];
    }
  } else {
    for (int q = threadIdx.x; q < nn + np; q += blockDim.x) {
      int z = (q < nn) ? zn + q : zp + (q - nn);
      ps[off + q] = ls[z];
    }
  }
}

__global__ void k_eke(double2* __restrict__ force, const double2* __restrict__ psi,
                      const double* __restrict__ occ, StateGeom g, double ecut,
                      double* __restrict__ part) {
  __shared__ double red[32];
  int s = blockIdx.y;
  double e = 0.0;
  double w = occ[s];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.npts; p += gridDim.x * blockDim.x) {
    size_t i = (size_t)s * g.npts + p;
    double g2 = g.g2[p];
    double2 f = force[i];
    if (g2 <= ecut) {
      double2 ps = psi[i];
      double wt = w * g.wpt[p] * g2;
      f.x -= wt * ps.x;
      f.y -= wt * ps.y;
      e += wt * (ps.x * ps.x + ps.y * ps.y);
    } else {
      f = make_double2(0.0, 0.0);
    }
    force[i] = f;
  }
  double t = block_sum(e, red);
  if (threadIdx.x == 0) part[(size_t)s * gridDim.x + blockIdx.x] = 0.5 * t;
}

__global__ void k_rowsum2(const double* __restrict__ part, int ncol, int nrow,
                          double* __restrict__ out) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nrow) {
    double a = 0.0;
    for (int c = 0; c < ncol; ++c) a += part[(size_t)r * ncol + c];
    out[r] = a;
  }
}

}  // namespace

// step intervals in time order -> phase numbers of the header (EES runs third)
static const int kPhaseOfInterval[CPSTEP_NPHASE] = {0, 1, 2, 6, 3, 4, 5};

int prof_fold(cpstep_ctx* c) {
  if (c->prof_pending == 0) return CPSTEP_OK;
  const int W = CPSTEP_NPHASE + 1;
  CPSTEP_CUDA_TRY(cudaEventSynchronize(c->prof_ev[(size_t)(c->prof_pending - 1) * W + CPSTEP_NPHASE]));
  for (int s = 0; s < c->prof_pending; ++s)
    for (int k = 0; k < CPSTEP_NPHASE; ++k) {
      float ms = 0.f;
      CPSTEP_CUDA_TRY(cudaEventElapsedTime(&ms, c->prof_ev[(size_t)s * W + k],
                                           c->prof_ev[(size_t)s * W + k + 1]));
      c->prof_ms[kPhaseOfInterval[k]] += ms;
    }
  c->prof_steps += c->prof_pending;
  c->prof_pending = 0;
  return CPSTEP_OK;
}

void graph_drop(cpstep_ctx* c) {
  c->gen += 1;
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  c->gexec = nullptr;
  c->graph_warm = 0;
}

extern "C" {

int cpstep_version(void) { return 100; }

unsigned long long cpstep_launch_count(void) {
  return __atomic_load_n(&g_cpstep_launches, __ATOMIC_RELAXED);
}

int cpstep_ctx_profile(cpstep_ctx* c, int enable) {
  if (!c) return CPSTEP_ERR_ARG;
  graph_drop(c);
  if (enable && c->prof_ev.empty()) {
    c->prof_ev.resize((size_t)cpstep_ctx::PROF_RING * (CPSTEP_NPHASE + 1));
    for (auto& e : c->prof_ev) CPSTEP_CUDA_TRY(cudaEventCreate(&e));
  }
  c->profile = enable ? 1 : 0;
  for (int i = 0; i < CPSTEP_NPHASE; ++i) c->prof_ms[i] = 0.0;
  c->prof_steps = 0;
  c->prof_pending = 0;
  return CPSTEP_OK;
}

int cpstep_phase_times(cpstep_ctx* c, double* ms, int* steps) {
  if (!c || !ms) return CPSTEP_ERR_ARG;
  if (int rc = prof_fold(c)) return rc;
  for (int i = 0; i < CPSTEP_NPHASE; ++i) ms[i] = c->prof_ms[i];
  if (steps) *steps = c->prof_steps;
  return CPSTEP_OK;
}

const char* cpstep_last_error(void) { return g_err; }

int cpstep_ctx_create(cpstep_ctx** out, int precision, int nstates, int npts, const int* kx,
                      const int* ky, const int* kz, int nruns, const int* runs, int nx, int ny,
                      int nz, const double* hmat, double ecut_ry) {
  g_err[0] = 0;
  if (!out || !kx || !ky || !kz || !runs || !hmat || nstates <= 0 || npts <= 0 || nruns <= 0 ||
      (nruns & 1) || nx <= 0 || ny <= 0 || nz <= 0 ||
      (precision != CPSTEP_PREC_FP64 && precision != CPSTEP_PREC_MIXED)) {
    cpstep_set_error("ctx_create: bad argument");
    return CPSTEP_ERR_ARG;
  }
  *out = nullptr;
  cpstep_ctx* c = new cpstep_ctx();
  c->precision = precision;
  c->nstates = nstates;
  c->npts = npts;
  c->nx = nx; c->ny = ny; c->nz = nz;
  c->ecut_ry = ecut_ry;
  c->stream = 0;
  std::memcpy(c->hmat, hmat, sizeof(double) * 9);
  if (!inv3(hmat, c->hmati, &c->vol)) {
    delete c;
    cpstep_set_error("ctx_create: singular cell");
    return CPSTEP_ERR_ARG;
  }
  c->vol = std::fabs(c->vol);
  // --- line tables from the run descriptors (readStateIntoRuns pairs them)
  int nl = nruns / 2;
  std::vector<int> off(nl), nneg(nl), npos(nl), zneg(nl), zpos(nl), xy(nl);
  int nsub = nz - runs[6];
  int kxmax = 0, acc = 0;
  for (int l = 0; l < nl; ++l) {
    const int* rn = runs + 14 * l;
    const int* rp = rn + 7;
    if (rn[0] != rp[0] || rn[1] != rp[1] || rn[3] != acc || rp[3] != rn[3] + rn[4] ||
        rn[4] < 0 || rp[4] < 0 || rp[0] < 0 || rp[1] < 0 || rp[0] >= nx || rp[1] >= ny ||
        rn[2] + nsub + rn[4] > nz || rp[2] + rp[4] > nz || rp[2] < 0 || rn[2] + nsub < 0) {
      delete c;
      cpstep_set_error("ctx_create: run descriptor pair %d inconsistent", l);
      return CPSTEP_ERR_LAYOUT;
    }
    off[l] = rn[3];
    nneg[l] = rn[4];
    npos[l] = rp[4];
    zneg[l] = rn[2] + nsub;
    zpos[l] = rp[2];
    xy[l] = rp[0] | (rp[1] << 16);
    kxmax = std::max(kxmax, rp[0]);
    acc = rp[3] + rp[4];
  }
  if (acc != npts) {
    delete c;
    cpstep_set_error("ctx_create: runs cover %d points, npts %d", acc, npts);
    return CPSTEP_ERR_LAYOUT;
  }
  c->nlines = nl;
  c->nlpad = (nl + 3) & ~3;
  c->nplane_x = kxmax + 1;
  if (c->nplane_x > nx / 2) {
    delete c;
    cpstep_set_error("ctx_create: kx range %d exceeds nx/2", kxmax);
    return CPSTEP_ERR_LAYOUT;
  }
  c->h_kx.assign(kx, kx + npts);
  c->h_ky.assign(ky, ky + npts);
  c->h_kz.assign(kz, kz + npts);
  c->h_line_xy = xy;
  c->h_line_off = off;
  std::vector<double> g2(npts), wpt(npts);
  const double tpi = 2.0 * M_PI;
  const double* hi = c->hmati;
  for (int i = 0; i < npts; ++i) {
    double a = kx[i], b = ky[i], cc = kz[i];
    double gx = (a * hi[0] + b * hi[1] + cc * hi[2]) * tpi;
    double gy = (a * hi[3] + b * hi[4] + cc * hi[5]) * tpi;
    double gz = (a * hi[6] + b * hi[7] + cc * hi[8]) * tpi;
    g2[i] = gx * gx + gy * gy + gz * gz;
    wpt[i] = (kx[i] == 0) ? 1.0 : 2.0;
  }
  int rc = cudaGetDevice(&c->device) == cudaSuccess ? 0 : CPSTEP_ERR_CUDA;
  if (!rc) {
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
    if (c->num_sms <= 0) c->num_sms = 148;
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, c->device);
    c->tc_ok = major == 10;
    if (cudaMalloc(&c->d_dev_err, sizeof(int)) != cudaSuccess ||
        cudaMemset(c->d_dev_err, 0, sizeof(int)) != cudaSuccess)
      rc = CPSTEP_ERR_CUDA;
  }
  if (!rc) rc = upload(&c->d_line_off, off.data(), nl);
  if (!rc) rc = upload(&c->d_line_nneg, nneg.data(), nl);
  if (!rc) rc = upload(&c->d_line_npos, npos.data(), nl);
  if (!rc) rc = upload(&c->d_line_zneg, zneg.data(), nl);
  if (!rc) rc = upload(&c->d_line_zpos, zpos.data(), nl);
  if (!rc) rc = upload(&c->d_line_xy, xy.data(), nl);
  if (!rc) rc = upload(&c->d_kx, kx, npts);
  if (!rc) rc = upload(&c->d_ky, ky, npts);
  if (!rc) rc = upload(&c->d_kz, kz, npts);
  if (!rc) rc = upload(&c->d_g2, g2.data(), npts);
  if (!rc) rc = upload(&c->d_wpt, wpt.data(), npts);
  if (!rc) rc = statefft_init(c);
  if (!rc) rc = rho_init(c, std::fabs(hmat[0]), ecut_ry);
  if (!rc) rc = step_init_classes(c);
  if (rc) {
    cpstep_ctx_destroy(c);
    return rc;
  }
  *out = c;
  return CPSTEP_OK;
}

int cpstep_ctx_destroy(cpstep_ctx* c) {
  if (!c) return CPSTEP_OK;
  cudaFree(c->d_line_off); cudaFree(c->d_line_nneg); cudaFree(c->d_line_npos);
  cudaFree(c->d_line_zneg); cudaFree(c->d_line_zpos); cudaFree(c->d_line_xy);
  cudaFree(c->d_kx); cudaFree(c->d_ky); cudaFree(c->d_kz);
  cudaFree(c->d_g2); cudaFree(c->d_wpt);
  cudaFree(c->d_pc_part); cudaFree(c->d_ortho_ws); cudaFree(c->d_hmati);
  cudaFree(c->d_dev_err);
  cudaFree(c->d_split);
  cudaFree(c->d_lv);
  cudaFree(c->d_hlv[0]); cudaFree(c->d_hlv[1]); cudaFree(c->d_pdiag);
  cudaFree(c->d_ion_e);
  cudaFree(c->d_force_atoms);
  graph_drop(c);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  for (auto& e : c->prof_ev) cudaEventDestroy(e);
  nl_free(c);
  sf_free(c);
  nhc_free(c);
  atom_nvt_free(c);
  rho_free(c);
  step_free(c);
  statefft_free(c);
  delete c;
  return CPSTEP_OK;
}

int cpstep_ctx_set_stream(cpstep_ctx* c, void* stream) {
  if (!c) return CPSTEP_ERR_ARG;
  graph_drop(c);
  c->stream = reinterpret_cast<cudaStream_t>(stream);
  return CPSTEP_OK;
}

int cpstep_ctx_info(const cpstep_ctx* c, int* nlines, int* nplane_x) {
  if (!c) return CPSTEP_ERR_ARG;
  if (nlines) *nlines = c->nlines;
  if (nplane_x) *nplane_x = c->nplane_x;
  return CPSTEP_OK;
}

int cpstep_ctx_sync(cpstep_ctx* c) {
  if (!c) return CPSTEP_ERR_ARG;
  CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CPSTEP_OK;
}

int cpstep_expand_gspace(cpstep_ctx* c, const double* d_packed, double* d_lines, int nstates) {
  if (!c || !d_packed || !d_lines || nstates <= 0) return CPSTEP_ERR_ARG;
  k_expand<<<dim3(c->nlines, nstates), 128, 0, c->stream>>>(
      const_cast<double2*>(reinterpret_cast<const double2*>(d_packed)),
      reinterpret_cast<double2*>(d_lines), c->geom(), 1);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

int cpstep_pack_gspace(cpstep_ctx* c, const double* d_lines, double* d_packed, int nstates) {
  if (!c || !d_packed || !d_lines || nstates <= 0) return CPSTEP_ERR_ARG;
  k_expand<<<dim3(c->nlines, nstates), 128, 0, c->stream>>>(
      reinterpret_cast<double2*>(d_packed),
      const_cast<double2*>(reinterpret_cast<const double2*>(d_lines)), c->geom(), 0);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

int cpstep_stp_fft_gtor(cpstep_ctx* c, const double* d_psi, double* d_psi_r, int nstates) {
  if (!c || !d_psi || !d_psi_r || nstates <= 0 || nstates > c->nstates) return CPSTEP_ERR_ARG;
  return statefft_gtor(c, d_psi, d_psi_r, nstates);
}

int cpstep_stp_fft_rtog(cpstep_ctx* c, const double* d_f_r, double* d_fg, int nstates) {
  if (!c || !d_f_r || !d_fg || nstates <= 0 || nstates > c->nstates) return CPSTEP_ERR_ARG;
  return statefft_rtog(c, d_f_r, d_fg, nstates);
}

int cpstep_density(cpstep_ctx* c, const double* d_psi, const double* d_occ, double* d_rho) {
  if (!c || !d_psi || !d_occ || !d_rho) return CPSTEP_ERR_ARG;
  return statefft_density(c, d_psi, d_occ, d_rho);
}

int cpstep_vks_psi(cpstep_ctx* c, const double* d_psi, const double* d_vks, const double* d_occ,
                   double* d_force, double* d_eke) {
  if (!c || !d_psi || !d_vks || !d_occ || !d_force) return CPSTEP_ERR_ARG;
  return statefft_vpsi(c, d_psi, d_vks, d_occ, d_force, d_eke, 0);
}

int cpstep_eke(cpstep_ctx* c, double* d_force, const double* d_psi, const double* d_occ,
               double* d_eke) {
  if (!c || !d_force || !d_psi || !d_occ || !d_eke) return CPSTEP_ERR_ARG;
  int nb = std::max(1, std::min(64, cdiv(c->npts, 256)));
  if (nb > c->nblk_z) nb = c->nblk_z;  // d_eke_part holds nstates*nblk_z partials
  k_eke<<<dim3(nb, c->nstates), 256, 0, c->stream>>>(
      reinterpret_cast<double2*>(d_force), reinterpret_cast<const double2*>(d_psi), d_occ,
      c->geom(), c->ecut_ry, c->d_eke_part);
  CPSTEP_LAUNCH_CHECK();
  k_rowsum2<<<cdiv(c->nstates, 128), 128, 0, c->stream>>>(c->d_eke_part, nb, c->nstates, d_eke);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

int cpstep_pc_overlap(cpstep_ctx* c, const double* d_a, const double* d_b, int na, int nb,
                      double alpha, double beta, double* d_c, int ldc) {
  if (!c || !d_a || !d_b || !d_c || na <= 0 || nb <= 0 || ldc < na) return CPSTEP_ERR_ARG;
  return pc_overlap_launch(c, d_a, d_b, na, nb, 2 * c->npts, c->d_wpt, alpha, beta, d_c, ldc);
}

int cpstep_pc_backmultiply(cpstep_ctx* c, const double* d_m, int ldm, const double* d_in,
                           int nin, double* d_out, int nout, double alpha, double beta) {
  if (!c || !d_m || !d_in || !d_out || nin <= 0 || nout <= 0 || ldm < nin) return CPSTEP_ERR_ARG;
  const int K = 2 * c->npts;
  return pc_backmul_launch(c, d_m, ldm, d_in, K, d_out, K, nout, nin, K, alpha, beta);
}

int cpstep_dgemm(cpstep_ctx* c, char transa, char transb, int m, int n, int k, double alpha,
                 const double* d_a, int lda, const double* d_b, int ldb, double beta, double* d_c,
                 int ldc) {
  if (!c || !d_a || !d_b || !d_c || m < 0 || n < 0 || k < 0) return CPSTEP_ERR_ARG;
  int ta = (transa == 'T' || transa == 't' || transa == 'C' || transa == 'c');
  int tb = (transb == 'T' || transb == 't' || transb == 'C' || transb == 'c');
  if (lda < (ta ? k : m) || ldb < (tb ? n : k) || ldc < m) return CPSTEP_ERR_ARG;
  if (m == 0 || n == 0) return CPSTEP_OK;
  return dgemm_launch(c->stream, ta, tb, m, n, k, alpha, d_a, lda, d_b, ldb, beta, d_c, ldc);
}

int cpstep_ortho_tmat(cpstep_ctx* c, const double* d_s, double* d_t, int n, int mode,
                      double tol, int max_iter, int* iters, double* rms) {
  if (!c || !d_s || !d_t || n <= 0 || max_iter <= 0 || mode < 0 || mode > 3) return CPSTEP_ERR_ARG;
  return ortho_tmat(c, d_s, d_t, n, mode & 1, (mode >> 1) & 1, tol, max_iter, iters, rms, 1);
}

int cpstep_set_atoms(cpstep_ctx* c, int natm, int ntyp, const int* typ, const double* pos,
                     const double* q, int nspl, double gmin_spl, double dg_spl,
                     const double* vps, const double* gzvps, double alp_ewd) {
  if (c) graph_drop(c);
  if (!c || natm <= 0 || ntyp <= 0 || !typ || !pos || !q || nspl <= 1 || !(dg_spl > 0) || !vps ||
      !gzvps || !(alp_ewd > 0))
    return CPSTEP_ERR_ARG;
  return atoms_set(c, natm, ntyp, typ, pos, q, nspl, gmin_spl, dg_spl, vps, gzvps, alp_ewd);
}

int cpstep_rho_layout(const cpstep_ctx* c, int cap, int* npts, int* kx, int* ky, int* kz) {
  if (!c || !npts) return CPSTEP_ERR_ARG;
  *npts = c->rg.npts;
  if (!kx || !ky || !kz) return CPSTEP_OK;
  if (cap < c->rg.npts) return CPSTEP_ERR_ARG;
  CPSTEP_CUDA_TRY(cudaMemcpy(kx, c->rg.kx, sizeof(int) * c->rg.npts, cudaMemcpyDeviceToHost));
  CPSTEP_CUDA_TRY(cudaMemcpy(ky, c->rg.ky, sizeof(int) * c->rg.npts, cudaMemcpyDeviceToHost));
  CPSTEP_CUDA_TRY(cudaMemcpy(kz, c->rg.kz, sizeof(int) * c->rg.npts, cudaMemcpyDeviceToHost));
  return CPSTEP_OK;
}

int cpstep_exc_calc(cpstep_ctx* c, const double* d_rho, double* d_vxc, double* d_energies) {
  if (!c || !d_rho || !d_vxc || !d_energies) return CPSTEP_ERR_ARG;
  return rho_xc(c, d_rho, d_vxc, d_energies);
}

int cpstep_rho_fft_r2g(cpstep_ctx* c, const double* d_rho_r, double* d_rhog) {
  if (!c || !d_rho_r || !d_rhog) return CPSTEP_ERR_ARG;
  if (int rc = rho_r2g(c, d_rho_r)) return rc;
  return rho_conj_scale(c, reinterpret_cast<const double*>(c->rg.rhog), d_rhog, c->rg.npts, 1.0);
}

int cpstep_hart_eext(cpstep_ctx* c, const double* d_rhog, double* d_vksg, double* d_energies,
                     double* d_force) {
  if (!c || !d_rhog || !d_vksg || !d_energies) return CPSTEP_ERR_ARG;
  if (int rc = rho_conj_scale(c, d_rhog, reinterpret_cast<double*>(c->rg.rhog), c->rg.npts, 1.0))
    return rc;
  if (int rc = rho_hart(c, d_energies, d_force)) return rc;
  return rho_conj_scale(c, reinterpret_cast<const double*>(c->rg.vg), d_vksg, c->rg.npts, 1.0);
}

int cpstep_vks_fft_g2r(cpstep_ctx* c, const double* d_vksg, double* d_v_r) {
  if (!c || !d_vksg || !d_v_r) return CPSTEP_ERR_ARG;
  if (int rc = rho_conj_scale(c, d_vksg, reinterpret_cast<double*>(c->rg.vg), c->rg.npts, 1.0))
    return rc;
  return c->ops64.g2r(c, rho_job(c), reinterpret_cast<const double*>(c->rg.vg), d_v_r, 1);
}

int cpstep_vks_from_rho(cpstep_ctx* c, const double* d_rho_r, double* d_vks_r,
                        double* d_energies, double* d_force) {
  if (!c || !d_rho_r || !d_vks_r || !d_energies) return CPSTEP_ERR_ARG;
  if (int rc = rho_xc(c, d_rho_r, d_vks_r, d_energies)) return rc;
  if (int rc = rho_r2g(c, d_rho_r)) return rc;
  if (c->xc == CPSTEP_XC_BLYP)
    if (int rc = rho_gga(c, d_rho_r, d_vks_r, d_energies)) return rc;
  if (int rc = rho_hart(c, d_energies, d_force)) return rc;
  return rho_vks_r(c, d_vks_r);
}

int cpstep_eext_grid_size(int kmax, double scale, int n_interp) {
  if (kmax < 0 || n_interp < 2) return -1;
  return eext_grid_size(kmax, scale, n_interp);
}

int cpstep_set_local_ees(cpstep_ctx* c, int on, int ngrid, int n_interp) {
  if (!c) return CPSTEP_ERR_ARG;
  graph_drop(c);
  return eesloc_set(c, on, ngrid, n_interp);
}

int cpstep_set_xc(cpstep_ctx* c, int functional, double gradient_cutoff) {
  if (!c || (functional != CPSTEP_XC_PZ_LDA && functional != CPSTEP_XC_BLYP))
    return CPSTEP_ERR_ARG;
  graph_drop(c);
  if (functional == CPSTEP_XC_BLYP && !c->d_gga_r) {
    const size_t nr = (size_t)c->nx * c->ny * c->nz;
    CPSTEP_CUDA_TRY(cudaMalloc(&c->d_gga_r, sizeof(double) * 3 * nr));
    CPSTEP_CUDA_TRY(cudaMalloc(&c->d_gga_g, sizeof(double2) * 4 * (size_t)c->rg.npts));
  }
  c->xc = functional;
  c->gga_cut = gradient_cutoff > 0.0 ? gradient_cutoff : 5.0e-5;
  return CPSTEP_OK;
}

int cpstep_gga_functional(cpstep_ctx* c, const double* d_rho, double* d_gx, double* d_gy,
                          double* d_gz, double* d_vks, double* d_energies) {
  if (!c || !d_rho || !d_gx || !d_gy || !d_gz || !d_vks || !d_energies) return CPSTEP_ERR_ARG;
  return rho_gga_functional(c, d_rho, d_gx, d_gy, d_gz, d_vks, d_energies, 0);
}

int cpstep_nl_grid_size(int kmax, double scale, int n_interp) {
  return nl_grid_size(kmax, scale, n_interp);
}

int cpstep_set_nonlocal(cpstep_ctx* c, int nkf, int n_interp, int nchan, const int* ch_type,
                        const int* ch_l, const int* ch_m, const double* vnl, const double* gz0,
                        const double* vnorm) {
  if (c) graph_drop(c);
  if (!c || nchan <= 0 || !ch_type || !ch_l || !ch_m || !vnl || !gz0 || !vnorm) {
    cpstep_set_error("set_nonlocal: bad argument");
    return CPSTEP_ERR_ARG;
  }
  return nl_set(c, nkf, n_interp, nchan, ch_type, ch_l, ch_m, vnl, gz0, vnorm);
}

int cpstep_ion_forces(cpstep_ctx* c, double* d_fatm, double* d_energies) {
  if (!c || !d_fatm || !d_energies) return CPSTEP_ERR_ARG;
  return ion_forces(c, d_fatm, d_energies);
}

int cpstep_atoms_integrate(cpstep_ctx* c, int itime, double* d_pos, double* d_vel,
                           const double* d_fatm, const double* d_mass, double dt, double* d_ekin) {
  if (!c || itime < 0 || !d_pos || !d_vel || !d_fatm || !d_mass || !(dt > 0.0))
    return CPSTEP_ERR_ARG;
  return atoms_integrate(c, itime, d_pos, d_vel, d_fatm, d_mass, dt, d_ekin);
}

int cpstep_set_nonlocal_sf(cpstep_ctx* c, int nchan, const int* ch_type, const int* ch_l,
                           const int* ch_m, const double* vnl, const double* gz0,
                           const double* vnorm) {
  if (!c || nchan <= 0 || !ch_type || !ch_l || !ch_m || !vnl || !gz0 || !vnorm) {
    cpstep_set_error("set_nonlocal_sf: bad argument");
    return CPSTEP_ERR_ARG;
  }
  return sf_set(c, nchan, ch_type, ch_l, ch_m, vnl, gz0, vnorm);
}

int cpstep_sf_nonlocal(cpstep_ctx* c, const double* d_psi, const double* d_occ, double* d_fpsi,
                       double* d_energies, double* d_fatm) {
  if (!c || !d_psi || !d_occ || !d_fpsi || !d_energies) {
    cpstep_set_error("sf_nonlocal: bad argument");
    return CPSTEP_ERR_ARG;
  }
  return sf_run(c, d_psi, d_occ, d_fpsi, d_energies, d_fatm);
}

int cpstep_ees_nonlocal(cpstep_ctx* c, const double* d_psi, const double* d_occ, double* d_fpsi,
                        double* d_energies, double* d_fatm) {
  if (!c || !d_psi || !d_occ || !d_fpsi || !d_energies) {
    cpstep_set_error("ees_nonlocal: bad argument");
    return CPSTEP_ERR_ARG;
  }
  return nl_run(c, d_psi, d_occ, d_fpsi, d_energies, d_fatm);
}

int cpstep_set_cp_mass(cpstep_ctx* c, double tau_fs, double cut_ry) {
  if (!c || !(tau_fs > 0) || !(cut_ry > 0)) return CPSTEP_ERR_ARG;
  graph_drop(c);
  return step_set_mass(c, tau_fs, cut_ry);
}

int cpstep_set_cp_thermostat(cpstep_ctx* c, double te_ext, double tau_fs, int num_nhc, int nck,
                             int nres, int nyosh) {
  if (!c) return CPSTEP_ERR_ARG;
  if (te_ext > 0.0 && !c->d_cmass) {
    cpstep_set_error("set_cp_thermostat: CP masses not set (cpstep_set_cp_mass)");
    return CPSTEP_ERR_STATE;
  }
  graph_drop(c);
  return nhc_set(c, te_ext, tau_fs, num_nhc, nck, nres, nyosh);
}

int cpstep_set_atom_thermostat(cpstep_ctx* c, int len_nhc, int nres, int nyosh,
                               const double* h_kT, const double* h_mnhc) {
  if (!c) return CPSTEP_ERR_ARG;
  return atom_nvt_set(c, len_nhc, nres, nyosh, h_kT, h_mnhc);
}

int cpstep_atom_thermostat_state(cpstep_ctx* c, int set, double* h_vnhc, double* h_pos_kt,
                                 double* h_energies2) {
  if (!c) return CPSTEP_ERR_ARG;
  return atom_nvt_state(c, set, h_vnhc, h_pos_kt, h_energies2);
}

int cpstep_cp_thermostat_state(cpstep_ctx* c, int set, double* h_x, double* h_xp, double* h_v) {
  if (!c) return CPSTEP_ERR_ARG;
  return nhc_state(c, set, h_x, h_xp, h_v);
}

int cpstep_cp_integrate(cpstep_ctx* c, const double* d_force, double* d_psi, double* d_vpsi,
                        double dt, int iteration, double* d_fict_ke) {
  if (!c || !d_force || !d_psi || !d_vpsi || iteration < 1) return CPSTEP_ERR_ARG;
  return step_integrate(c, d_force, d_psi, d_vpsi, dt, iteration, d_fict_ke, nullptr);
}

int cpstep_cp_step(cpstep_ctx* c, double* d_psi, double* d_vpsi, const double* d_occ, double dt,
                   int iteration, double* d_energies, double* d_atom_force) {
  if (!c || !d_psi || !d_vpsi || !d_occ || !d_energies || iteration < 1) return CPSTEP_ERR_ARG;
  if (c->atoms.natm <= 0 || !c->d_cmass) {
    cpstep_set_error("cp_step: atoms and CP masses must be set first");
    return CPSTEP_ERR_STATE;
  }
  // the first step (no second half kick) and profiled steps run directly
  if (iteration <= 1 && c->dyn_form == CPSTEP_CONSTRAINT_ORTHO_T) {
    int rc = step_run(c, d_psi, d_vpsi, d_occ, dt, iteration, d_energies, d_atom_force, 0);
    if (rc) return rc;
    int fl[4] = {0, 0, 0, 0};
    double dev = 0.0;
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(fl, c->d_dyn_flags, sizeof(fl), cudaMemcpyDeviceToHost,
                                    c->stream));
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(&dev, c->d_dyn_dev, sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
    CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (fl[3]) {
      cpstep_set_error("cp_step: S fails cp_norb_tol on the first step (max |S - 2I| = %g >= %g)",
                       dev, c->tol_norb);
      return CPSTEP_ERR_NORB;
    }
    return CPSTEP_OK;
  }
  if (!c->use_graph || iteration <= 1 || c->profile)
    return step_run(c, d_psi, d_vpsi, d_occ, dt, iteration, d_energies, d_atom_force, 0);
  const cpstep_ctx::StepKey key{d_psi, d_vpsi, d_occ, dt, d_energies, d_atom_force};
  if (c->gexec && key == c->gkey) {
    CPSTEP_CUDA_TRY(cudaGraphLaunch(c->gexec, c->stream));
    __atomic_add_fetch(&g_cpstep_launches, c->gkernels, __ATOMIC_RELAXED);
    return CPSTEP_OK;
  }
  if (!c->graph_warm || !(key == c->gkey)) {  // one direct step: buffers allocated, sizes set
    graph_drop(c);
    int rc = step_run(c, d_psi, d_vpsi, d_occ, dt, iteration, d_energies, d_atom_force, 0);
    if (!rc) {
      c->graph_warm = 1;
      c->gkey = key;
    }
    return rc;
  }
  // capture on a private stream (the legacy default stream cannot be captured)
  if (!c->cap_stream) CPSTEP_CUDA_TRY(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  const cudaStream_t user = c->stream;
  const unsigned long long n0 = cpstep_launch_count();
  c->stream = c->cap_stream;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeRelaxed);
  int rc = e == cudaSuccess ? step_run(c, d_psi, d_vpsi, d_occ, dt, iteration, d_energies,
                                       d_atom_force, 0)
                            : CPSTEP_ERR_CUDA;
  if (e == cudaSuccess) e = cudaStreamEndCapture(c->cap_stream, &g);
  c->stream = user;
  const unsigned long long nk = cpstep_launch_count() - n0;
  __atomic_sub_fetch(&g_cpstep_launches, nk, __ATOMIC_RELAXED);  // captured, not run
  cudaGraphExec_t x = nullptr;
  if (!rc && e == cudaSuccess && g) e = cudaGraphInstantiate(&x, g, 0);
  if (g) cudaGraphDestroy(g);
  if (rc || e != cudaSuccess || !x) {  // not capturable here: direct launches from now on
    cudaGetLastError();
    if (x) cudaGraphExecDestroy(x);
    c->use_graph = 0;
    return step_run(c, d_psi, d_vpsi, d_occ, dt, iteration, d_energies, d_atom_force, 0);
  }
  c->gexec = x;
  c->gkernels = nk;
  CPSTEP_CUDA_TRY(cudaGraphLaunch(c->gexec, c->stream));
  __atomic_add_fetch(&g_cpstep_launches, c->gkernels, __ATOMIC_RELAXED);
  return CPSTEP_OK;
}

int cpstep_set_constraint(cpstep_ctx* c, int form, double tol_norb) {
  if (!c || (form != CPSTEP_CONSTRAINT_ORTHO_T && form != CPSTEP_CONSTRAINT_LOWDIN) ||
      !(tol_norb > 0.0))
    return CPSTEP_ERR_ARG;
  graph_drop(c);
  c->dyn_form = form;
  c->tol_norb = tol_norb;
  c->dyn_init = 0;
  c->dyn_loaded = 0;
  return CPSTEP_OK;
}

int cpstep_dyn_state(cpstep_ctx* c, int set, double* d_psi_no, double* d_tmat,
                     int* h_half_step) {
  if (!c || (set != 0 && set != 1)) return CPSTEP_ERR_ARG;
  const size_t ncoef = (size_t)c->nstates * c->npts;
  const size_t nt = (size_t)c->nstates * c->nstates;
  if (set) {
    if (!d_psi_no || !d_tmat) {
      cpstep_set_error("dyn_state: a load needs both psi_no and orthoT");
      return CPSTEP_ERR_ARG;
    }
    graph_drop(c);
    if (!c->d_psi_no) CPSTEP_CUDA_TRY(cudaMalloc(&c->d_psi_no, sizeof(double2) * ncoef));
    if (!c->d_tmat) CPSTEP_CUDA_TRY(cudaMalloc(&c->d_tmat, sizeof(double) * nt));
    if (!c->d_dyn_flags) CPSTEP_CUDA_TRY(cudaMalloc(&c->d_dyn_flags, 4 * sizeof(int)));
    if (!c->d_dyn_dev) CPSTEP_CUDA_TRY(cudaMalloc(&c->d_dyn_dev, sizeof(double)));
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(c->d_psi_no, d_psi_no, sizeof(double2) * ncoef,
                                    cudaMemcpyDeviceToDevice, c->stream));
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(c->d_tmat, d_tmat, sizeof(double) * nt,
                                    cudaMemcpyDeviceToDevice, c->stream));
    // flags: no reset pending, [1] = 1 - halfStepEvolve, no resets counted
    int fl[4] = {0, (h_half_step && *h_half_step == 0) ? 1 : 0, 0, 0};
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(c->d_dyn_flags, fl, sizeof(fl), cudaMemcpyHostToDevice,
                                    c->stream));
    CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));  // fl is on this stack frame
    c->dyn_init = 1;
    c->dyn_loaded = 1;
    return CPSTEP_OK;
  }
  if (!c->dyn_init) {
    cpstep_set_error("dyn_state: no state yet (run iteration 1 or load one)");
    return CPSTEP_ERR_STATE;
  }
  if (d_psi_no)
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(d_psi_no, c->d_psi_no, sizeof(double2) * ncoef,
                                    cudaMemcpyDeviceToDevice, c->stream));
  if (d_tmat)
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(d_tmat, c->d_tmat, sizeof(double) * nt,
                                    cudaMemcpyDeviceToDevice, c->stream));
  if (h_half_step) {
    int fl[4] = {0, 0, 0, 0};
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(fl, c->d_dyn_flags, sizeof(fl), cudaMemcpyDeviceToHost,
                                    c->stream));
    CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    *h_half_step = fl[1] ? 0 : 1;
  }
  return CPSTEP_OK;
}

int cpstep_dyn_status(cpstep_ctx* c, double* max_dev, int* resets) {
  if (!c) return CPSTEP_ERR_ARG;
  int fl[4] = {0, 0, 0, 0};
  double dev = 0.0;
  if (c->d_dyn_flags)
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(fl, c->d_dyn_flags, sizeof(fl), cudaMemcpyDeviceToHost,
                                    c->stream));
  if (c->d_dyn_dev)
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(&dev, c->d_dyn_dev, sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
  CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (max_dev) *max_dev = dev;
  if (resets) *resets = fl[2];
  return CPSTEP_OK;
}

int cpstep_ctx_set_graph(cpstep_ctx* c, int enable) {
  if (!c || (enable != 0 && enable != 1)) return CPSTEP_ERR_ARG;
  graph_drop(c);
  c->use_graph = enable;
  return CPSTEP_OK;
}

int cpstep_ctx_graph_status(cpstep_ctx* c, int* enabled, int* captured,
                            unsigned long long* kernels) {
  if (!c) return CPSTEP_ERR_ARG;
  if (enabled) *enabled = c->use_graph;
  if (captured) *captured = c->gexec != nullptr;
  if (kernels) *kernels = c->gkernels;
  return CPSTEP_OK;
}

int cpstep_set_positions(cpstep_ctx* c, const double* h_pos) {
  if (!c || !h_pos) return CPSTEP_ERR_ARG;
  return atoms_set_positions(c, h_pos);
}

int cpstep_cp_step_host(cpstep_ctx* c, double* d_psi, double* d_vpsi, const double* d_occ,
                        double dt, int iteration, const double* h_pos, double* h_energies,
                        double* h_atom_force) {
  if (!c || !d_psi || !d_vpsi || !d_occ || !h_energies || iteration < 1) return CPSTEP_ERR_ARG;
  if (h_pos) {
    if (int rc = atoms_set_positions(c, h_pos)) return rc;
  }
  if (!c->d_force_atoms) {
    CPSTEP_CUDA_TRY(cudaMalloc(&c->d_force_atoms, sizeof(double) * 3 * std::max(1, c->atoms.natm)));
  }
  if (int rc = cpstep_cp_step(c, d_psi, d_vpsi, d_occ, dt, iteration, c->d_energies,
                              h_atom_force ? c->d_force_atoms : nullptr))
    return rc;
  CPSTEP_CUDA_TRY(cudaMemcpyAsync(h_energies, c->d_energies, sizeof(double) * CPSTEP_NENERGY,
                                  cudaMemcpyDeviceToHost, c->stream));
  if (h_atom_force)
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(h_atom_force, c->d_force_atoms,
                                    sizeof(double) * 3 * c->atoms.natm, cudaMemcpyDeviceToHost,
                                    c->stream));
  CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CPSTEP_OK;
}

int cpstep_set_gemm_path(cpstep_ctx* c, int tensor_cores) {
  if (!c || (tensor_cores != 0 && tensor_cores != 1)) return CPSTEP_ERR_ARG;
  graph_drop(c);
  if (tensor_cores) {
    int major = 0;
    CPSTEP_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, c->device));
    if (major != 10) {
      cpstep_set_error("set_gemm_path: tensor-core products need compute capability 10.x");
      return CPSTEP_ERR_ARG;
    }
  }
  c->tc_ok = tensor_cores;
  return CPSTEP_OK;
}

int cpstep_device_errors(cpstep_ctx* c, int* flags) {
  if (!c || !flags) return CPSTEP_ERR_ARG;
  *flags = 0;
  CPSTEP_CUDA_TRY(cudaMemcpyAsync(flags, c->d_dev_err, sizeof(int), cudaMemcpyDeviceToHost,
                                  c->stream));
  CPSTEP_CUDA_TRY(cudaMemsetAsync(c->d_dev_err, 0, sizeof(int), c->stream));
  CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CPSTEP_OK;
}

int cpstep_step_status(cpstep_ctx* c, int* iters, int* converged) {
  if (!c) return CPSTEP_ERR_ARG;
  int st[2] = {0, 0};
  if (c->d_ortho_status) {
    CPSTEP_CUDA_TRY(cudaMemcpyAsync(st, c->d_ortho_status, sizeof(st), cudaMemcpyDeviceToHost,
                                    c->stream));
  }
  CPSTEP_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (iters) *iters = st[0];
  if (converged) *converged = st[1];
  return CPSTEP_OK;
}

}  // extern "C"
