// Internal definition of the cpstep context.
#pragma once
#include <vector>
#include "common.cuh"
#include "fft_smem.cuh"

// Geometry of the packed state layout as the kernels see it.
struct StateGeom {
  int nx, ny, nz;
  int nlines, nlpad, nplane_x, npts;
  const int* line_off;   // packed offset of the first (negative-kz) point of the line
  const int* line_nneg;  // points in the negative-kz run
  const int* line_npos;  // points in the non-negative-kz run
  const int* line_zneg;  // z index of the first negative-kz point
  const int* line_zpos;  // z index of the first non-negative-kz point
  const int* line_xy;    // x | (y << 16), both wrapped to [0, n)
  const double* g2;      // |G|^2 per packed point
  const double* wpt;     // double-pack weight per point (1 on Gx=0, 2 elsewhere)
};

struct cpstep_ctx;

// Per-grid-size state FFT entry points (compile-time N inside).
struct StateFftOps {
  int (*density)(cpstep_ctx*, const double*, const double*, double*);
  int (*vpsi)(cpstep_ctx*, const double*, const double*, const double*, double*, double*, int);
  int (*gtor)(cpstep_ctx*, const double*, double*, int);
  int (*rtog)(cpstep_ctx*, const double*, double*, int);
  int lb;  // z-lines per block of the z-passes
};
template <typename T, int N>
StateFftOps statefft_ops();

template <typename T>
struct Twiddles {
  cplx<T>* x = nullptr;
  cplx<T>* y = nullptr;
  cplx<T>* z = nullptr;
};

struct cpstep_ctx {
  int precision;  // CPSTEP_PREC_FP64 or CPSTEP_PREC_MIXED
  int nstates;
  int npts;
  int nx, ny, nz;
  int nlines, nlpad, nplane_x;
  double vol;
  double hmat[9];
  double hmati[9];
  double ecut_ry;
  cudaStream_t stream;
  int device;
  int num_sms;

  // layout tables (device)
  int *d_line_off, *d_line_nneg, *d_line_npos, *d_line_zneg, *d_line_zpos, *d_line_xy;
  int *d_kx, *d_ky, *d_kz;
  double *d_g2, *d_wpt;
  std::vector<int> h_kx, h_ky, h_kz;
  std::vector<int> h_line_xy, h_line_off;

  StateFftOps ops;
  Twiddles<double> tw64;
  Twiddles<float> tw32;

  // state-FFT scratch (bytes sized for the working precision)
  void* d_pen_a;         // [nstates][nz][nlpad] complex  (psi z-pencils)
  void* d_pen_b;         // [nstates][nz][nlpad] complex  (V.psi z-pencils)
  double* d_rho_part;    // [ngroups_rho][nz*ny*nx]
  int ngroups_rho;
  void* d_vks_t;         // V_KS in working precision [nz][ny][nx]
  double* d_eke_part;    // [nstates][nblk_z]
  int nblk_z;
  double* d_red;         // small reduction scratch

  StateGeom geom() const {
    StateGeom g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.nlines = nlines; g.nlpad = nlpad; g.nplane_x = nplane_x; g.npts = npts;
    g.line_off = d_line_off; g.line_nneg = d_line_nneg; g.line_npos = d_line_npos;
    g.line_zneg = d_line_zneg; g.line_zpos = d_line_zpos; g.line_xy = d_line_xy;
    g.g2 = d_g2; g.wpt = d_wpt;
    return g;
  }
};

// statefft.cu
int statefft_init(cpstep_ctx* c);
void statefft_free(cpstep_ctx* c);
