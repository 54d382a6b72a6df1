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

// One FFT geometry with its pencil buffers (state sphere or density sphere).
struct FftJob {
  StateGeom g;
  void* pen_a;  // [nstates][nz][nlpad] pencils of the G->R pass
  void* pen_b;  // [nstates][nz][nlpad] pencils of the R->G pass
};

// EES non-local: the atoms' B-spline factors on the NL grid (per atom a, axis
// d = a, b, c and interpolation point j < 8; eesAtmBsplineRgrp,
// cp_ees_nonlocal.C:256-580) as the NL plane kernels read them.
constexpr int kNlInterp = 8;
// Mn and its gradient at one stencil point of one atom (see nl_point).
struct __align__(16) NlVal {
  double mn, dx, dy, dz;
};

struct NlAtoms {
  int natm;
  const int* typ;      // [natm]
  const int* ig;       // [natm][3][8] 0-based grid index along a, b, c
  const double* mn;    // [natm][3][8] M_n factors
  const double* dmn;   // [natm][3][8] their derivatives
  double hmati[9];
  double grid;         // NL grid size (cubic)
  // per (type, plane): the atoms of the type with an interpolation plane there,
  // atom | (jc << 16) in atom order, and their count
  const int* plist;    // [ntyp][nkf][natm]
  const int* pcount;   // [ntyp][nkf]
  // per-plane stencil tables of the channel's type (k_nl_table), tcap entries
  // per plane: entry e*64 + q is point q = jb*8 + ja of atom slot e of plist:
  // its plane cell tcell (y*N + x) and tval (Mn, dMn/dx, dMn/dy, dMn/dz as in
  // nl_point); the gather list: the gcount touched cells gcell in increasing
  // order, their entries gent[goff[c] .. goff[c+1]) in atom-slot order
  int tcap;
  const int* tcell;          // [nkf][tcap]
  const NlVal* tval;         // [nkf][tcap]
  const int* gcell;          // [nkf][tcap]
  const int* goff;           // [nkf][tcap + 1]
  const int* gent;           // [nkf][tcap]
  const int* gcount;         // [nkf]
};

// The B-spline product of one stencil point, in the reference's order
// (eesAtmBsplineRgrp IV, cp_ees_nonlocal.C:523-532): mn and dmn_{x,y,z}.
__device__ __forceinline__ void nl_point(const NlAtoms& A, int a, int ja, int jb, int jc,
                                         double& mn, double& dx, double& dy, double& dz) {
  const double* m = A.mn + (size_t)a * 3 * kNlInterp;
  const double* d = A.dmn + (size_t)a * 3 * kNlInterp;
  const double ma = m[ja], mb = m[kNlInterp + jb], mc = m[2 * kNlInterp + jc];
  const double at = d[ja] * mb * mc * A.grid;
  const double bt = ma * d[kNlInterp + jb] * mc * A.grid;
  const double ct = ma * mb * d[2 * kNlInterp + jc] * A.grid;
  mn = ma * mb * mc;
  const double* h = A.hmati;
  dx = at * h[0] + bt * h[1] + ct * h[2];
  dy = at * h[3] + bt * h[4] + ct * h[5];
  dz = at * h[6] + bt * h[7] + ct * h[8];
}

// One channel's NL pass on the NL grid: geometry, pencils, twiddles, atoms.
struct NlJob {
  FftJob f;
  const void* tw;      // [nkf] twiddles in working precision
  NlAtoms A;
  int ctype;           // atom type of the channel
};

// Per-grid-size FFT entry points (compile-time N inside).
struct StateFftOps {
  int (*density)(cpstep_ctx*, const double*, const double*, double*);
  int (*vpsi)(cpstep_ctx*, const double*, const double*, const double*, double*, double*, int);
  int (*gtor)(cpstep_ctx*, const double*, double*, int);
  int (*rtog)(cpstep_ctx*, const double*, double*, int);
  int (*g2r)(cpstep_ctx*, const FftJob&, const double*, double*, int);
  int (*r2g)(cpstep_ctx*, const FftJob&, const double*, double*, int, double);
  // EES on this grid size: conj(dyp psi) -> NL grid -> per-plane atom sums
  // zpart[s][atom][8][4]; scatter of zs[s][atom] -> NL grid -> fpsi +=
  int (*nl_proj)(cpstep_ctx*, const NlJob&, const double*, const double2*, int, double*);
  int (*nl_force)(cpstep_ctx*, const NlJob&, const double*, const double2*, int, double*);
  size_t (*nl_smem)(int nplane_x);
  int lb;  // z-lines per block of the z-passes
};
template <typename T, int N>
StateFftOps statefft_ops();

// Density sphere geometry and buffers (FP64 in both precision modes).
struct RhoGeom {
  int npts = 0, nlines = 0, nlpad = 0, nplane_x = 0;
  int *line_off = nullptr, *line_nneg = nullptr, *line_npos = nullptr;
  int *line_zneg = nullptr, *line_zpos = nullptr, *line_xy = nullptr;
  int *kx = nullptr, *ky = nullptr, *kz = nullptr;
  double *g2 = nullptr, *wpt = nullptr;
  void *pen_a = nullptr, *pen_b = nullptr;
  double2* rhog = nullptr;   // transformed density (conj of the reference rho(G))
  double2* vg = nullptr;     // conj of the reference vks(G)
  double4* fterm = nullptr;  // per-point force terms of CP_hart_eext_calc
  double* vhl = nullptr;     // Hartree + local potential on the grid
  double* part = nullptr;    // reduction partials
  int nblk_xc = 0, nblk_h = 0;
  int kz_runs = 0;           // every line's points have consecutive kz (phase recurrence)
};

// Atoms, pseudopotential spline tables and structure-factor phase tables.
struct AtomData {
  int natm = 0, ntyp = 0, nspl = 0;
  double gmin = 0, dg = 0, alp_ewd = 0;
  int* typ = nullptr;
  double *frac = nullptr, *q = nullptr, *vps = nullptr, *gzvps = nullptr;
  int kxm = 0, kym = 0, kzm = 0;
  double2 *ex = nullptr, *ey = nullptr, *ez = nullptr;
  double2* ezt = nullptr;  // [natm][2 kzm + 1], atoms in type order
  int* rank = nullptr;     // atom -> position in type order
  int tstart[CPSTEP_MAX_TYPES + 1] = {};  // type t holds ranks [tstart[t], tstart[t+1])
  int nfblk = 0;           // blocks (rows of fpart) of the force pass
  double* fpart = nullptr;
  double* pos = nullptr;  // Cartesian positions [natm][3] (bohr)
  std::vector<double> h_q;  // charges, host copy
};

// Isokinetic NHC thermostat of the CP coefficients (cpstep_set_cp_thermostat):
// initCPNHC's constants, the per-point chunk map and per-(state, chunk) chains.
struct CpNhc {
  int on = 0;
  int num = 0, nck = 0, nres = 0, nyosh = 0;
  double kT = 0.0, m[2] = {0.0, 0.0};
  double v0[8] = {0}, a2[8] = {0}, a4[8] = {0}, dfs[8] = {0};
  signed char* d_ck = nullptr;  // chunk of each point, -1 on the redundant half
  double *d_x = nullptr, *d_xp = nullptr, *d_vn = nullptr;  // [S][nck][num][2]
  int nsplit = 0, span = 0;       // KE blocks per state and points per block
  double* d_part = nullptr;       // [S][nsplit][nck]
  double* d_scale = nullptr;      // [S][nck][2]
  double* d_eout = nullptr;       // [S][nck][3]
  double* d_fm = nullptr;         // [npts] (dt/2) / cmass of the current step
};

// Massive Nose-Hoover chains of the atoms (cpstep_set_atom_thermostat).
struct AtomNvt {
  int len = 0, nres = 0, nyosh = 0;  // len 0: NVE
  int natm = 0;                      // atoms the chains were set for
  double *d_kT = nullptr, *d_mnhc = nullptr;  // [natm], [natm][len]
  double *d_vn = nullptr, *d_pkt = nullptr;   // [natm][3][len], [natm]
  double* d_e = nullptr;                      // {E_kin NHC, pot NHC} of the last step
};

// Structure-factor (non-EES) non-local state, l = 0 (cpstep_set_nonlocal_sf).
struct SfData {
  int on = 0, n = 0, ldz = 0;       // n non-local atoms (type order)
  int* atom = nullptr;              // [n] atom index
  int* ptab = nullptr;              // [n] projector table of the atom's type
  double* proj = nullptr;           // [tables][npts] y00 v_0(|G|)
  double* vn = nullptr;             // [n] vnorm / vol
  double* rows = nullptr;           // [4 n][2 npts] S, S^x, S^y, S^z (real view)
  double* z = nullptr;              // [nstates][4 n] projections
  double* zs = nullptr;             // [nstates][ldz] 2 vnorm/vol z
  double* enl_s = nullptr;          // [nstates]
  double* fnl = nullptr;            // [nstates][natm][3]
};

// EES non-local state of a context (cpstep_set_nonlocal).
struct NlData {
  int on = 0, nkf = 0, nchan = 0;
  std::vector<int> ch_type;
  std::vector<double> ch_vn;        // vnorm / vol per channel
  double2* dyp = nullptr;           // [nchan][npts] projector b(G) Ylm v_l(g)
  int *line_zneg = nullptr, *line_zpos = nullptr, *line_xy = nullptr;  // NL-grid lines
  void *pen_a = nullptr, *pen_b = nullptr;  // [nstates][nkf][nlpad]
  void* tw = nullptr;               // [nkf] twiddles, working precision
  StateFftOps ops;
  int* ig = nullptr;                // [natm][3][8]
  int *plist = nullptr, *pcount = nullptr;  // per-plane atom lists (NlAtoms)
  double *mn = nullptr, *dmn = nullptr;
  double* zpart = nullptr;          // [nstates][natm][8][4]
  double* zs = nullptr;             // [nstates][natm]
  double* enl_s = nullptr;          // [nstates]
  double* fnl = nullptr;            // [nstates][natm][3]
  int natm = 0;
  // stencil tables (NlAtoms), one block per type: type t starts at entry
  // tab_off[t] (nkf * tab_cap[t] entries), tab_cap[t] = 64 * atoms of type t
  int *tcell = nullptr, *gcell = nullptr, *goff = nullptr, *gent = nullptr, *gcount = nullptr;
  NlVal* tval = nullptr;
  std::vector<size_t> tab_off;
  std::vector<int> tab_cap;
  // G-space evaluation of the same sums (mixed contexts on the tensor cores,
  // ees_gspace_run): per atom separable transforms, S matrices (FP32) of each
  // type [v][atom of type][ld_s], each type's channels with contiguous dyp
  int km = 0;                       // largest |k| of the state sphere on an axis
  double2* sep = nullptr;           // [natm][3][2][2 km + 1]
  float* sv = nullptr;              // per type at sv_off[t]
  long long ld_s = 0;               // floats per S row (2 npts rounded up to 4)
  std::vector<long long> sv_off;
  std::vector<std::vector<int>> tch;  // channels of each type, in channel order
  std::vector<float2*> tdyp;        // [nch_t][ld_d32] per type, FP32 (tensor-core path)
  std::vector<float> tdmax;         // largest |dyp| of each type's channels (FP16 scales)
  std::vector<std::vector<float>> tdmax_c;  // the same per channel of the type
  float* d_hmax = nullptr;          // [2][ntyp] bound of |S| (Mn rows) and largest |Z| entry
                                    // per type (float bits, atomicMax), written every pass
  // FP16 levels of the S rows of every type (rows v natm_t + a, the pre-split
  // image) at blv + blv_off[t], their scales and inverses at tsc / tinv +
  // tsoff[t]; the A operand of the sums (w psi dyp_c) at alv
  uint8_t* blv = nullptr;
  std::vector<size_t> blv_off;
  float *tsc = nullptr, *tinv = nullptr;
  std::vector<long long> tsoff;
  uint8_t* alv = nullptr;
  size_t alv_bytes = 0;
  // the psi force's operand levels: Z and the transposed Mn rows (largest type)
  uint8_t *pf_z = nullptr, *pf_st = nullptr;
  size_t pf_zbytes = 0, pf_stbytes = 0;
  int ld_d32 = 0;                   // npts rounded up to even
  int* d_order = nullptr;           // atom of each type-order rank
  int* d_tch = nullptr;             // [ntyp][4] channel indices (-1 unused)
  double* d_vn = nullptr;           // [nchan] vnorm / vol
  double* csum = nullptr;           // sums of one type [nch 4 natm_t][nstates]
  double* zt = nullptr;             // scaled Z of two types, [nstates][ldz] each
  size_t zt_slot = 0;               // doubles per type
  int gspace_ok = 0;                // every type has at most 4 channels
};

// EES form of the Hartree + local + Ewald pass (cpstep_set_local_ees, the
// reference's cp_eext_ees_opt): the atoms' B-splines on the EES grid and their
// separable transforms with the EES weights folded in, per axis d and atom a,
//   t_d[k][a] = bden_d(k) sum_j Mn_d[a][j] e^{+2 pi i k ig_d[a][j] / ngrid}
// and dt_d the same sum of dMn, over the density sphere's k extents.
struct EesLocal {
  int on = 0, ngrid = 0, natm = 0;
  int* ig = nullptr;                // [natm][3][8]
  double *mn = nullptr, *dmn = nullptr;
  double2* bden = nullptr;          // [ngrid] get_bspline_wght1d
  double2 *tx = nullptr, *ty = nullptr, *tz = nullptr;     // [k][natm]
  double2 *dtx = nullptr, *dty = nullptr, *dtz = nullptr;
  double2* tzt = nullptr;           // [type-order rank][2 kzm + 1]
};

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

  StateFftOps ops;    // working precision
  StateFftOps ops64;  // FP64 (density path)
  RhoGeom rg;
  AtomData atoms;
  EesLocal eloc;
  NlData nl;
  SfData sf;
  CpNhc nhc;
  AtomNvt atom_nvt;
  int rho_izero = -1;
  // exchange-correlation functional (CPSTEP_XC_*) and the BLYP scratch: the
  // three gradient grids [3][N_r] and four packed density-sphere arrays
  int xc = 0;
  double gga_cut = 5.0e-5;
  double* d_ion_e = nullptr;  // [natm] real-space Ewald pair energies
  double* d_gga_r = nullptr;
  double2* d_gga_g = nullptr;
  double* d_energies = nullptr;  // [CPSTEP_NENERGY]
  // electronic step
  int* d_cls = nullptr;      // point class (0 redundant Gx=0, 1 G=0, 2 unique Gx=0, 3 Gx>0)
  int* d_red_idx = nullptr;  // redundant points and their stored partners
  int* d_red_src = nullptr;
  int nred = 0;
  double* d_cmass = nullptr;
  int nblk_ke = 0;
  double* d_step_part = nullptr;
  double *d_lambda = nullptr, *d_smat = nullptr, *d_tmat = nullptr;
  double *d_psi_tmp = nullptr, *d_rho = nullptr, *d_vks = nullptr, *d_eke = nullptr;
  double* d_force = nullptr;
  double* d_force_atoms = nullptr;  // staging of cpstep_cp_step_host
  // the orthonormality constraint of the step (cpstep_set_constraint):
  // CPSTEP_CONSTRAINT_ORTHO_T carries the non-orthogonal coefficients d_psi_no
  // and orthoT (d_tmat, the previous step's T) between steps;
  // CPSTEP_CONSTRAINT_LOWDIN needs neither
  int dyn_form = 0;
  double tol_norb = 0.003;
  int dyn_init = 0;             // d_psi_no / d_tmat hold a state (iteration 1 or loaded)
  int dyn_loaded = 0;           // loaded by cpstep_dyn_state since the last step
  double* d_psi_no = nullptr;   // [nstates][npts] complex
  double* d_gamma = nullptr;    // gamma = orthoT lambda, S x S column-major
  int* d_dyn_flags = nullptr;   // [0] reset in this step, [1] next integrate skips the
                                // second half kick, [2] resets so far, [3] first-step failure
  double* d_dyn_dev = nullptr;  // max |S - 2I| of the last step
  // phase timing (cpstep_ctx_profile): events recorded on the context's stream
  // (a ring of PROF_RING steps' events, folded into prof_ms when it fills or
  // when cpstep_phase_times is called, so profiling adds no per-step sync)
  static constexpr int PROF_RING = 64;
  int profile = 0;
  std::vector<cudaEvent_t> prof_ev;  // [PROF_RING][CPSTEP_NPHASE + 1]
  int prof_pending = 0;
  double prof_ms[CPSTEP_NPHASE] = {};
  int prof_steps = 0;
  double* d_hmati = nullptr;
  Twiddles<double> tw64;
  Twiddles<float> tw32;

  // state-FFT scratch (bytes sized for the working precision)
  void* d_pen_a;         // [nstates][nz][nlpad] complex  (psi z-pencils)
  void* d_pen_b;         // [nstates][nz][nlpad] complex  (V.psi z-pencils)
  double* d_rho_part;    // [ngroups_rho][nz*ny*nx], or the two-stage density's plane partials
  int ngroups_rho;
  size_t rho_part_elems = 0;  // doubles in d_rho_part
  int p16_blocks_k2 = 0, p16_blocks_k3 = 0;  // resident blocks of the two-stage plane passes
  void* d_vks_t;         // V_KS in working precision [nz][ny][nx]
  double* d_eke_part;    // [nstates][nblk_z]
  int nblk_z;
  double* d_red;         // small reduction scratch

  // PairCalculator / Ortho scratch (grown on demand)
  double* d_pc_part = nullptr;
  size_t pc_part_elems = 0;
  void* d_split = nullptr;  // plane buffer of the split plane passes (k_split_*)
  size_t split_bytes = 0;
  uint8_t* d_lv = nullptr;  // BF16 levels of pre-split tensor-core operands (k_presplit)
  size_t lv_bytes = 0;
  // BF16 level images of the two operands of a many-state overlap (k_presplit)
  // and the FP64 row sums of its diagonal
  uint8_t* d_hlv[2] = {nullptr, nullptr};
  size_t hlv_bytes[2] = {0, 0};
  double* d_pdiag = nullptr;
  size_t pdiag_elems = 0;
  double* d_ortho_ws = nullptr;
  size_t ortho_ws_elems = 0;
  int* d_ortho_status = nullptr;  // [iterations, converged] of the last Ortho launch
  // tensor-core PairCalc products (mixed precision on sm_100): on by default
  // where the device is compute capability 10.x; cpstep_set_gemm_path
  int tc_ok = 0;
  int* d_dev_err = nullptr;  // error bits set by kernels (bounded waits that timed out)

  // CUDA graph of cpstep_cp_step (iteration > 1): captured after one direct
  // step with the same arguments, replayed while they stay the same; dropped
  // by every call that changes what it holds (graph_drop)
  struct StepKey {
    double *psi, *vpsi;
    const double* occ;
    double dt;
    double *energies, *atom_force;
    bool operator==(const StepKey& o) const {
      return psi == o.psi && vpsi == o.vpsi && occ == o.occ && dt == o.dt &&
             energies == o.energies && atom_force == o.atom_force;
    }
  };
  // launch choices (cpstep_autotune, cpstep_tune_get/set); the defaults are
  // the fixed heuristics
  struct Tune {
    int shfl = 2;         // state plane passes (density, V.psi): register shuffle FFT (1),
                          // shared-memory Stockham (0), or the two-stage form of
                          // fft_p16.cuh (2: FP32 and N = 32, 64, 128; elsewhere as 1)
    int plane_waves = 3;  // state plane passes: blocks ~ plane_waves x SMs
    int nl_blocks = 6;    // EES plane kernels: blocks ~ nl_blocks x SMs
    int pc_split = 1;     // PairCalc overlap split-K: CTAs ~ pc_split x SMs
    int ees_gspace = 1;   // mixed contexts on the tensor cores: EES in G space (1) or
                          // through the NL-grid FFTs (0)
  } tune;
  int use_graph = 1;
  int graph_warm = 0;              // a direct step with gkey ran
  StepKey gkey{};
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t gexec = nullptr;
  unsigned long long gkernels = 0;  // kernels in the graph
  unsigned gen = 0;                 // counts graph_drop calls (batch graphs recapture)
  // batches: the Ortho launch (cooperative, grid-wide barriers) waits for
  // ortho_wait and records ortho_signal, so no two contexts' Ortho kernels run
  // at the same time
  cudaEvent_t ortho_wait = nullptr, ortho_signal = nullptr;

  FftJob state_job() const {
    FftJob j;
    j.g = geom();
    j.pen_a = d_pen_a;
    j.pen_b = d_pen_b;
    return j;
  }

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
int statefft_density(cpstep_ctx* c, const double* psi, const double* occ, double* rho);
int statefft_vpsi(cpstep_ctx* c, const double* psi, const double* vks, const double* occ,
                  double* force, double* eke, int pencils_ready);
int statefft_gtor(cpstep_ctx* c, const double* psi, double* psi_r, int nstates);
int statefft_rtog(cpstep_ctx* c, const double* f_r, double* fg, int nstates);

int statefft_lookup(int precision, int n, StateFftOps* o);

// ees.cu
int nl_set(cpstep_ctx* c, int nkf, int n_interp, int nchan, const int* ch_type, const int* ch_l,
           const int* ch_m, const double* vnl, const double* gz0, const double* vnorm);
void nl_free(cpstep_ctx* c);
int sf_set(cpstep_ctx* c, int nchan, const int* ch_type, const int* ch_l, const int* ch_m,
           const double* vnl, const double* gz0, const double* vnorm);
void sf_free(cpstep_ctx* c);
int sf_run(cpstep_ctx* c, const double* psi, const double* occ, double* fpsi, double* energies,
           double* fatm);
int nl_run(cpstep_ctx* c, const double* psi, const double* occ, double* fpsi, double* energies,
           double* fatm);
int nl_grid_size(int kmax, double scale, int n_interp);
int eext_grid_size(int kmax, double scale, int n_interp);
// eesAtmBsplineRgrp's indices, Mn and dMn of every atom on an nkf grid
// (order kNlInterp) from fractional coordinates [natm][3]
int ees_bspline_launch(cpstep_ctx* c, const double* frac, int natm, int nkf, int* ig, double* mn,
                       double* dmn);
// get_bspline_wght1d: the complex EES weights of one axis, m = 0 .. ngrid-1
void ees_bspline_weights(int n_interp, int ngrid, std::vector<double>& br,
                         std::vector<double>& bi);

// rhopath.cu
int rho_init(cpstep_ctx* c, double box_len, double ecut_ry);
void rho_free(cpstep_ctx* c);
FftJob rho_job(const cpstep_ctx* c);
int atoms_set(cpstep_ctx* c, int natm, int ntyp, const int* typ, const double* pos,
              const double* q, int nspl, double gmin, double dg, const double* vps,
              const double* gzvps, double alp_ewd);
int atoms_set_positions(cpstep_ctx* c, const double* h_pos);
int rho_xc(cpstep_ctx* c, const double* rho_r, double* vxc, double* energies);
int rho_r2g(cpstep_ctx* c, const double* rho_r);
int rho_gga(cpstep_ctx* c, const double* rho_r, double* vks_r, double* energies);
int atoms_set_positions_dev(cpstep_ctx* c, const double* d_pos);
int ion_forces(cpstep_ctx* c, double* fatm, double* energies);
int atoms_integrate(cpstep_ctx* c, int itime, double* pos, double* vel, const double* fatm,
                    const double* mass, double dt, double* ekin);
int rho_gga_functional(cpstep_ctx* c, const double* rho_r, double* gx, double* gy, double* gz,
                       double* vks_r, double* energies, int add_to_exc);
int rho_hart(cpstep_ctx* c, double* energies, double* force);
int eesloc_set(cpstep_ctx* c, int on, int ngrid, int n_interp);
void eesloc_free(cpstep_ctx* c);
int rho_vks_r(cpstep_ctx* c, double* vks_r);
int rho_conj_scale(cpstep_ctx* c, const double* in, double* out, int n, double s);

// paircalc.cu
int pc_overlap_launch(cpstep_ctx* c, const double* a, const double* b, int M, int N, int K,
                      const double* w, double alpha, double beta, double* C, int ldc);
int pc_backmul_launch(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                      double* out, int ldo, int nout, int nin, int K, double alpha, double beta);
void graph_drop(cpstep_ctx* c);
int pc_part_reserve(cpstep_ctx* c, size_t elems);
size_t pc_part_need(int nsplit, size_t mn);  // partials plus the reduction's group sums
int split_reserve(cpstep_ctx* c, size_t bytes);
int lv_reserve(cpstep_ctx* c, size_t bytes);
// one atom type's operands of the EES psi force (paircalc_tc.cu)
struct EesForceType {
  const float* sv;      // FP32 Mn rows sv[a ld_s + k]
  long long ld_s;
  const float2* dyp;    // channel c at dyp + c ld_d
  int nch, natm_t;
  const double* Z;      // [S][ldz], inner index c natm_t + a
  int ldz;
  const float* smax;    // largest |S| and |Z| (float bits)
  const float* zmax;
  uint8_t* zlv;         // level buffers of Z and S^T
  uint8_t* stlv;
};
int ees_tc_force_pre(cpstep_ctx* c, int ntyp, const EesForceType* ty, int ld_d, double alpha,
                     double* fpsi, size_t zlv_bytes, size_t stlv_bytes);
size_t ees_pf_zbytes(int nstates, int natm_t);
size_t ees_pf_stbytes(int npts, int natm_t);
size_t ees_lv_bytes(int rows, int K);
int ees_tc_presplit_a(cpstep_ctx* c, const double* psi, int ntyp, const float2* const* dyp,
                      int ld_d, const int* nch, const float* const* dmax, uint8_t* const* alv,
                      size_t alv_bytes);
int ees_tc_sums_pre(cpstep_ctx* c, int nch, const float* dmax, const uint8_t* blv, int jp,
                    const float* cinv, const uint8_t* alv, double* C);
int pc_splitk_reduce_launch(cpstep_ctx* c, int nsplit, int M, int N, double alpha, double beta,
                            double* C, int ldc, int sym, const double* diag = nullptr);
// paircalc_tc.cu (tensor-core products; *used = false when the SIMT path must run)
bool pc_tc_usable(const cpstep_ctx* c);
int pc_overlap_tc_launch(cpstep_ctx* c, const double* a, const double* b, int M, int N, int K,
                         const double* w, double alpha, double beta, double* C, int ldc,
                         bool* used);
int pc_backmul_tc_launch(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                         double* out, int ldo, int nout, int nin, int K, double alpha,
                         double beta, const double* w, bool* used);
int pc_backmul_psiv_tc_launch(cpstep_ctx* c, const double* Tcm, int ldt, double* psi_no,
                              double* psi, int K, int n, const int* flag, double* v, double rdt,
                              bool* used);
int dgemm_launch(cudaStream_t s, int ta, int tb, int m, int n, int k, double alpha,
                 const double* A, int lda, const double* B, int ldb, double beta, double* C,
                 int ldc);

int pc_backmul_w_launch(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                        double* out, int ldo, int nout, int nin, int K, double alpha, double beta,
                        const double* w);

// api.cu
int prof_fold(cpstep_ctx* c);

// step.cu
int step_init_classes(cpstep_ctx* c);
void step_free(cpstep_ctx* c);
int step_set_mass(cpstep_ctx* c, double tau_fs, double cut_ry);
int step_integrate(cpstep_ctx* c, const double* force, double* psi, double* vpsi, double dt,
                   int iteration, double* d_fict_ke, double* d_enhc,
                   const int* d_skip_half = nullptr);

// nhc.cu
int nhc_set(cpstep_ctx* c, double te_ext, double tau_fs, int num, int nck, int nres, int nyosh);
void nhc_free(cpstep_ctx* c);
int nhc_state(cpstep_ctx* c, int set, double* h_x, double* h_xp, double* h_vn);
void nhc_yosh(int nyosh, double* w);  // set_yosh weights, unscaled
int atom_nvt_set(cpstep_ctx* c, int len, int nres, int nyosh, const double* h_kT,
                 const double* h_mnhc);
void atom_nvt_free(cpstep_ctx* c);
int atom_nvt_state(cpstep_ctx* c, int set, double* h_vn, double* h_pkt, double* h_e2);
int nhc_integrate(cpstep_ctx* c, const double* force, double* psi, double* vpsi, double dt,
                  int iteration, double* d_fict_ke, double* d_enhc, const int* d_skip_half);
int step_run(cpstep_ctx* c, double* psi, double* vpsi, const double* occ, double dt,
             int iteration, double* energies, double* atom_force, int ortho_check);

// ortho.cu
int ortho_tmat(cpstep_ctx* c, const double* S, double* T, int n, int mixed, int scale,
               double tol, int max_iter, int* iters_out, double* rms_out, int check_host);
