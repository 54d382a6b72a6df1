// State FFT registry: supported grid sizes, twiddle tables, scratch, and the
// small helper kernels shared by all sizes.  The per-size kernels live in
// statefft_impl.cuh and are instantiated in statefft_n*.cu.
#include <cmath>
#include "statefft_impl.cuh"

namespace sfft {

__global__ void k_rho_reduce(const double* __restrict__ part, int ngroups, size_t nr,
                             double scale, double* __restrict__ rho) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; i < nr; i += stride) {
    double a = 0.0;
    for (int g = 0; g < ngroups; ++g) a += part[(size_t)g * nr + i];
    rho[i] = a * scale;
  }
}

// blockIdx.x = plane z, blockIdx.y = a slice of its n^2 points.  The blocks b
// whose item range [I b / B, I (b + 1) / B) (I = n S items, plane-major) meets
// the plane's items [z S, (z + 1) S) are b0 = block of item z S .. b1 = block
// of item (z + 1) S - 1, where the block of item i is ((i + 1) B - 1) / I; an
// empty block range is skipped.  Block b's partial of plane z is its segment
// z - (first item of b) / S.  The (partial) offsets of the plane are listed
// once per block in shared memory.
__global__ void k_rho_reduce_items(const double* __restrict__ part, int n, int nstates,
                                   int nblocks, int segs, double scale, double* __restrict__ rho) {
  constexpr int MAXP = 64;
  __shared__ long long offs[MAXP];
  __shared__ int np_s;
  const int z = blockIdx.x;
  const size_t n2 = (size_t)n * n;
  const long long items = (long long)n * nstates;
  if (threadIdx.x == 0) {
    const long long ia = (long long)z * nstates, ib = ia + nstates - 1;
    const int b0 = (int)(((ia + 1) * nblocks - 1) / items);
    const int b1 = (int)(((ib + 1) * nblocks - 1) / items);
    int np = 0;
    for (int b = b0; b <= b1 && np < MAXP; ++b) {
      const long long s0 = p16_item_start(items, b, nblocks);
      if (s0 >= p16_item_start(items, b + 1, nblocks)) continue;
      const int seg = z - (int)(s0 / nstates);
      offs[np++] = ((long long)b * segs + seg) * (long long)n2;
    }
    np_s = np;
  }
  __syncthreads();
  const int np = np_s;
  const size_t per = (n2 + gridDim.y - 1) / gridDim.y;
  const size_t o0 = blockIdx.y * per, o1 = min(n2, o0 + per);
  for (size_t off = o0 + threadIdx.x; off < o1; off += blockDim.x) {
    double a = 0.0;
    for (int q = 0; q < np; ++q) a += part[offs[q] + off];
    rho[(size_t)z * n2 + off] = a * scale;
  }
}

// per-state sum of block partials in a fixed order (deterministic)
__global__ void k_rowsum(const double* __restrict__ part, int ncol, int nrow,
                         double* __restrict__ out) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nrow) {
    double a = 0.0;
    for (int c = 0; c < ncol; ++c) a += part[(size_t)r * ncol + c];
    out[r] = a;
  }
}

__global__ void k_to_float(const double* __restrict__ in, float* __restrict__ out, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) out[i] = (float)in[i];
}

}  // namespace sfft

// explicit specialisations live in the statefft_n*.cu files
#define CPSTEP_DECLARE(N)                         \
  template <> StateFftOps statefft_ops<double, N>(); \
  template <> StateFftOps statefft_ops<float, N>();
#define CPSTEP_FOR_SIZES(X) \
  X(16) X(20) X(24) X(28) X(32) X(40) X(42) X(48) X(60) X(64) X(80) X(96) X(120) X(128) X(198) X(200)
CPSTEP_FOR_SIZES(CPSTEP_DECLARE)

static bool lookup_ops(int precision, int n, StateFftOps* o) {
#define CPSTEP_CASE(N)                                                              \
  case N:                                                                           \
    *o = (precision == CPSTEP_PREC_FP64) ? statefft_ops<double, N>() : statefft_ops<float, N>(); \
    return true;
  switch (n) {
    CPSTEP_FOR_SIZES(CPSTEP_CASE)
    default:
      return false;
  }
#undef CPSTEP_CASE
}

int statefft_lookup(int precision, int n, StateFftOps* o) { return lookup_ops(precision, n, o) ? 1 : 0; }

int statefft_supported(int n) {
  StateFftOps o;
  return lookup_ops(CPSTEP_PREC_FP64, n, &o) ? 1 : 0;
}

template <typename T>
static int upload_tw(int n, cplx<T>** dst) {
  std::vector<cplx<T>> h(n);
  for (int m = 0; m < n; ++m) {
    double a = -2.0 * M_PI * (double)m / (double)n;
    h[m] = mk<T>((T)cos(a), (T)sin(a));
  }
  CPSTEP_CUDA_TRY(cudaMalloc(dst, sizeof(cplx<T>) * n));
  CPSTEP_CUDA_TRY(cudaMemcpy(*dst, h.data(), sizeof(cplx<T>) * n, cudaMemcpyHostToDevice));
  return CPSTEP_OK;
}

int statefft_init(cpstep_ctx* c) {
  if (c->nx != c->ny || c->ny != c->nz) {
    cpstep_set_error("state FFT: only cubic grids are built (got %d x %d x %d)", c->nx, c->ny, c->nz);
    return CPSTEP_ERR_ARG;
  }
  if (!lookup_ops(c->precision, c->nx, &c->ops) || !lookup_ops(CPSTEP_PREC_FP64, c->nx, &c->ops64)) {
    cpstep_set_error("state FFT: grid size %d not built into libcpstep", c->nx);
    return CPSTEP_ERR_ARG;
  }
  if (int rc = upload_tw<double>(c->nx, &c->tw64.x)) return rc;
  if (int rc = upload_tw<float>(c->nx, &c->tw32.x)) return rc;
  c->tw64.y = c->tw64.z = c->tw64.x;
  c->tw32.y = c->tw32.z = c->tw32.x;
  size_t csz = (c->precision == CPSTEP_PREC_FP64) ? sizeof(cplx<double>) : sizeof(cplx<float>);
  size_t pen = (size_t)c->nstates * c->nz * c->nlpad * csz;
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_pen_a, pen));
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_pen_b, pen));
  size_t nr = (size_t)c->nx * c->ny * c->nz;
  c->ngroups_rho = std::max(1, std::min(c->nstates, 8));
  // the two-stage density pass writes one plane partial per (block, plane
  // touched): at most (ceil(items / B) / S + 2) per block, B <= 2 blocks per SM
  size_t n2 = (size_t)c->nx * c->ny;
  long long items = (long long)c->nz * c->nstates;
  long long nb = 2LL * c->num_sms;
  size_t p16 = (size_t)nb * (size_t)(cdiv((int)((items + c->num_sms - 1) / c->num_sms), c->nstates) + 1) * n2;
  c->rho_part_elems = std::max(nr * c->ngroups_rho, p16);
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_rho_part, sizeof(double) * c->rho_part_elems));
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_vks_t, sizeof(float) * nr));
  c->nblk_z = cdiv(c->nlines, c->ops.lb);
  CPSTEP_CUDA_TRY(cudaMalloc(&c->d_eke_part, sizeof(double) * (size_t)c->nstates * c->nblk_z));
  return CPSTEP_OK;
}

void statefft_free(cpstep_ctx* c) {
  cudaFree(c->tw64.x);
  cudaFree(c->tw32.x);
  cudaFree(c->d_pen_a); cudaFree(c->d_pen_b); cudaFree(c->d_rho_part);
  cudaFree(c->d_vks_t); cudaFree(c->d_eke_part);
}

int statefft_density(cpstep_ctx* c, const double* psi, const double* occ, double* rho) {
  return c->ops.density(c, psi, occ, rho);
}
int statefft_vpsi(cpstep_ctx* c, const double* psi, const double* vks, const double* occ,
                  double* force, double* eke, int pencils_ready) {
  return c->ops.vpsi(c, psi, vks, occ, force, eke, pencils_ready);
}
int statefft_gtor(cpstep_ctx* c, const double* psi, double* psi_r, int nstates) {
  return c->ops.gtor(c, psi, psi_r, nstates);
}
int statefft_rtog(cpstep_ctx* c, const double* f_r, double* fg, int nstates) {
  return c->ops.rtog(c, f_r, fg, nstates);
}
