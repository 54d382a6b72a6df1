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

void cpstep_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// defined in statefft.cu
int statefft_density(cpstep_ctx* c, const double* psi, const double* occ, double* rho);
int statefft_vpsi(cpstep_ctx* c, const double* psi, const double* vks, const double* occ,
                  double* force, double* eke, int pencils_ready);
int statefft_gtor(cpstep_ctx* c, const double* psi, double* psi_r, int nstates);
int statefft_rtog(cpstep_ctx* c, const double* f_r, double* fg, int nstates);

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

extern "C" {

int cpstep_version(void) { return 100; }

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
  statefft_free(c);
  delete c;
  return CPSTEP_OK;
}

int cpstep_ctx_set_stream(cpstep_ctx* c, void* stream) {
  if (!c) return CPSTEP_ERR_ARG;
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

}  // extern "C"
