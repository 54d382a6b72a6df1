/*
 * libcpstep -- C ABI of the B200 (sm_100a) Car-Parrinello electronic step.
 *
 * Drop-in for the FFT, density, V.psi, kinetic, PairCalculator and Ortho
 * routines of OpenAtom.  Each entry names the reference routine it replaces
 * (paths relative to the OpenAtom tree).  Conventions, for every entry:
 *   - returns 0 (CPSTEP_OK) or an error code; cpstep_last_error() gives text.
 *     Nothing exits or aborts (the reference's CkExit/EXIT paths become codes).
 *   - coefficient arrays keep the reference's packed G-sphere layout: for every
 *     state the npts complex128 values (re, im interleaved) in the order of the
 *     kx/ky/kz arrays given to cpstep_ctx_create (the order processState
 *     produces, src_charm_driver/utility/util.C:1331-1642), states one after
 *     the other: psi[state][npts].
 *   - "d_" pointers are device pointers; work is queued on the context's
 *     stream (cpstep_ctx_set_stream) and is asynchronous unless stated.
 *   - the caller owns every buffer it passes.  A context owns its scratch.
 *   - one context per stream/thread; calls on one context are not re-entrant.
 *   - real-space grids are dense [nz][ny][nx] FP64 arrays (x fastest).  The
 *     reference keeps the same values in x-rows padded to nx+2
 *     (CP_Rho_RealSpacePlane.C:630-650).
 */
#ifndef CPSTEP_H
#define CPSTEP_H

#if defined(__GNUC__)
#define CPSTEP_API __attribute__((visibility("default")))
#else
#define CPSTEP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CPSTEP_OK 0
#define CPSTEP_ERR_ARG 1      /* bad size/pointer/argument */
#define CPSTEP_ERR_CUDA 2     /* CUDA runtime error */
#define CPSTEP_ERR_LAYOUT 3   /* inconsistent G-vector layout (util.C:956-1052 checks) */
#define CPSTEP_ERR_NOCONV 4   /* Ortho S->T iteration did not converge (ortho.C:129-133) */
#define CPSTEP_ERR_STATE 5    /* call out of order */
#define CPSTEP_ERR_NORB 6     /* S fails cp_norb_tol on the first dynamics step
                                 (Ortho::maxCheck, orthog_ctrl/ortho.C:477-482) */

/* slots of the energies array (Hartree): the reference's Iter [n] names */
#define CPSTEP_E_EXC 0     /* EEXC       (CP_exc_calc exc_ret)                */
#define CPSTEP_E_MUXC 1    /* muxc       (CP_exc_calc muxc_ret)               */
#define CPSTEP_E_HART 2    /* EHART      (CP_hart_eext_calc ehart_ret)        */
#define CPSTEP_E_EXT 3     /* EExt       (CP_hart_eext_calc eext_ret)         */
#define CPSTEP_E_EWD 4     /* reciprocal Ewald (CP_hart_eext_calc ewd_ret)    */
#define CPSTEP_E_EXT_G0 5  /* reserved                                        */
#define CPSTEP_E_KE 6      /* EKE        (sum of CP_eke_calc)                 */
#define CPSTEP_E_NL 7      /* ENL        (EES non-local)                      */
#define CPSTEP_E_TOT 8     /* ELEC_ENERGY_TOT = EKE+ENL+EHART+EExt+EEXC       */
#define CPSTEP_E_FICT 9    /* fictitious kinetic energy (get_fictKE)          */
#define CPSTEP_E_EXC_GGA 10 /* gradient correction part of EEXC (BLYP:
                               CP_getGGAFunctional exc_gga_ret)               */
#define CPSTEP_E_EWD_RS 11 /* real-space Ewald + self + background (CP_getionforce:
                               pot_ewd_rs + vself + vbgr)                    */
#define CPSTEP_E_NHC_KE 12 /* ekeNhc: CP thermostat kinetic energy (get_fictKE) */
#define CPSTEP_E_NHC_POT 13 /* potNHC: CP thermostat potential (get_fictKE)     */
#define CPSTEP_NENERGY 14

/* Exchange-correlation functionals (cpstep_set_xc).  PZ-LDA is the default;
 * BLYP is Slater exchange (CP_exc_calc with cp_lyp = 1) plus the Becke 88
 * exchange gradient correction and LYP correlation of CP_getGGAFunctional,
 * with the density gradients and the White-Bird divergence on the density
 * sphere (CP_Rho_GSpacePlane divRhoVksGspace / acceptWhiteByrd). */
#define CPSTEP_XC_PZ_LDA 0
#define CPSTEP_XC_BLYP 1

#define CPSTEP_MAX_TYPES 16   /* atom types a context accepts (cpstep_set_atoms) */

#define CPSTEP_PREC_FP64 0    /* plain FP64 path: the drop-in */
#define CPSTEP_PREC_MIXED 1   /* FP32 FFT/density/V.psi, FP64 accumulation, split GEMMs */

typedef struct cpstep_ctx cpstep_ctx;

/* Library version (major*10000 + minor*100 + patch). */
CPSTEP_API int cpstep_version(void);

/* Text of the last error on this thread ("" if none). */
CPSTEP_API const char* cpstep_last_error(void);

/* Kernels the library has launched since it was loaded (all contexts). */
CPSTEP_API unsigned long long cpstep_launch_count(void);

/* Phases of cpstep_cp_step timed with CUDA events on the context's stream when
 * profiling is on (cpstep_ctx_profile(ctx, 1) resets the sums):
 *   0 density (state FFTs G->R, rho)   1 V_KS (XC, rho FFT, Hartree/local/Ewald)
 *   2 V.psi + kinetic (state FFTs R->G) 3 lambda + constraint (PairCalc)
 *   4 integrate                         5 S + Ortho + psi.T (PairCalc, Ortho)
 *   6 EES non-local (runs between phases 2 and 3)
 * cpstep_phase_times returns the summed milliseconds per phase and the number
 * of profiled steps (synchronises the stream).  The Ortho S->T iteration has
 * no counterpart timer in the reference beyond TimeKeeper's substeps
 * (main/TimeKeeper.h:1-181). */
#define CPSTEP_NPHASE 7
CPSTEP_API int cpstep_ctx_profile(cpstep_ctx* ctx, int enable);
CPSTEP_API int cpstep_phase_times(cpstep_ctx* ctx, double* ms, int* steps);

/* ---------------------------------------------------------------------------
 * G-vector layout (host, no GPU needed).
 *
 * cpstep_layout_sizes: kmax of calc_cutoff (src_piny_physics_v1.0/interface/
 * cp_ewald/set_cp_ewald.C:124-225), the radixme FFT size (set_cp_ewald.C:751-818,
 * set_fftsizes :1505-1690), the half-sphere count of countkvec3d_sm
 * (set_cp_ewald.C:825-952) and the packed point count after flip_data_set
 * (src_charm_driver/utility/para_grp_parse.C:178-286) for a cubic box of side
 * box_len bohr and a cutoff ecut_ry Rydberg.
 */
CPSTEP_API int cpstep_layout_sizes(double box_len, double ecut_ry, int* kmax, int* nfft,
                        int* nktot_half, int* npts);

/*
 * cpstep_layout_build: the packed order of one state: setkvec3d_sm
 * (set_cp_ewald.C:523-680) -> flip_data_set (para_grp_parse.C:178-286) ->
 * processState (util.C:1331-1642, nchareG chunks, get_chareG_line_prms
 * para_grp_parse.C:21-170, sort_kxky util.C:2223-2247) -> RunDescriptors of
 * readStateIntoRuns (util.C:861-1099; 7 ints per run: x, y, z, offset,
 * length, inc, nz).  kx/ky/kz have room for npts_cap points and runs for
 * runs_cap runs.  nfft is the z size written into the run descriptors.
 */
CPSTEP_API int cpstep_layout_build(double box_len, double ecut_ry, int nchareG, int nfft,
                        int npts_cap, int* kx, int* ky, int* kz, int* npts,
                        int runs_cap, int* runs, int* nruns);

/* ---------------------------------------------------------------------------
 * State files (host, no GPU), one state per file as the reference writes them.
 *
 * cpstep_state_write: writeStateFile (src_charm_driver/utility/util.C:1955-
 *   2180) for one state: the packed points sorted as sort_psi_output
 *   (:2180-2220) orders them, the stored half sphere after G=0 and G=0 last;
 *   header "npts nx ny nz".  format: CPSTEP_STATE_TEXT ("%g %g %d %d %d"
 *   lines, as lossy as the reference's), CPSTEP_STATE_BINARY (int header,
 *   records double re, double im, int kx, ky, kz), and the _GZ variants
 *   (zlib, ".gz" appended to path).  The reference's TimeStamp side file is
 *   not written.
 * cpstep_state_read: readState (util.C:1107-1330) into the caller's packed
 *   layout (kx/ky/kz of npts points, as cpstep_layout_build or the reference
 *   produces it): every point takes the record with its (kx,ky,kz), the
 *   redundant Gx=0 half the conjugate of its partner (flip_data_set,
 *   para_grp_parse.C:178-286).  coef: npts complex (interleaved doubles).
 *   nx/ny/nz (may be NULL) receive the header's grid.  A layout point missing
 *   from the file returns CPSTEP_ERR_LAYOUT (the reference exits).
 */
#define CPSTEP_STATE_TEXT 0
#define CPSTEP_STATE_BINARY 1
#define CPSTEP_STATE_TEXT_GZ 2
#define CPSTEP_STATE_BINARY_GZ 3
CPSTEP_API int cpstep_state_write(const char* path, int format, int npts, const double* coef,
                                  const int* kx, const int* ky, const int* kz, int nx, int ny,
                                  int nz);
CPSTEP_API int cpstep_state_read(const char* path, int format, int npts, const int* kx,
                                 const int* ky, const int* kz, double* coef, int* nx, int* ny,
                                 int* nz);

/* ---------------------------------------------------------------------------
 * Context: the layout tables on the device plus the step's scratch.
 *
 * kx/ky/kz/runs: as produced by the reference (or cpstep_layout_build), copied.
 * hmat: the 3x3 cell matrix, column-major as PINY's gencell->hmat (bohr).
 * ecut_ry: the state cutoff of CP_eke_calc (g^2 <= ecut, cp_eke.C:77-91).
 * Replaces the FFTcache group set-up (src_charm_driver/fft_slab_ctrl/fftCache.C:100-330)
 * and the GStateSlab/RealStateSlab allocations (stateSlab.C:33-231).
 */
CPSTEP_API int cpstep_ctx_create(cpstep_ctx** ctx, int precision, int nstates, int npts,
                      const int* kx, const int* ky, const int* kz, int nruns,
                      const int* runs, int nx, int ny, int nz, const double* hmat,
                      double ecut_ry);
CPSTEP_API int cpstep_ctx_destroy(cpstep_ctx* ctx);
/* stream: a cudaStream_t (NULL = legacy default stream). */
CPSTEP_API int cpstep_ctx_set_stream(cpstep_ctx* ctx, void* stream);
/* Sizes the context derived: nlines, nplane_x. */
CPSTEP_API int cpstep_ctx_info(const cpstep_ctx* ctx, int* nlines, int* nplane_x);
/* Wait for the context's stream; returns a pending CUDA error if any. */
CPSTEP_API int cpstep_ctx_sync(cpstep_ctx* ctx);

/* ---------------------------------------------------------------------------
 * FFTcache / state chare mirrors.
 *
 * cpstep_expand_gspace: FFTcache::expandGSpace (fftCache.C:460-507) for all
 * states: packed [nstates][npts] -> z-lines [nstates][nlines][nz] (zero fill).
 * cpstep_pack_gspace: FFTcache::packGSpace (fftCache.C:517-553), the inverse.
 */
CPSTEP_API int cpstep_expand_gspace(cpstep_ctx* ctx, const double* d_packed, double* d_lines,
                         int nstates);
CPSTEP_API int cpstep_pack_gspace(cpstep_ctx* ctx, const double* d_lines, double* d_packed,
                       int nstates);

/*
 * cpstep_stp_fft_gtor: psi(G) -> psi(r) for nstates states, the composition of
 * doStpFFTGtoR_Gchare (fftCache.C:1133-1159), the G->R transpose
 * (CP_State_GSpacePlane.C:1473-1498, CP_State_RealSpacePlane.C:248-268) and
 * doStpFFTGtoR_Rchare (fftCache.C:1167-1243).  d_psi_r: [nstates][nz][ny][nx].
 * cpstep_stp_fft_rtog: the reverse composition doStpFFTRtoG_Rchare
 * (fftCache.C:1252-1319) -> transpose -> doStpFFTRtoG_Gchare (fftCache.C:1099-1123),
 * unscaled.  nstates <= the context's nstates.
 */
CPSTEP_API int cpstep_stp_fft_gtor(cpstep_ctx* ctx, const double* d_psi, double* d_psi_r,
                        int nstates);
CPSTEP_API int cpstep_stp_fft_rtog(cpstep_ctx* ctx, const double* d_f_r, double* d_fg,
                        int nstates);

/*
 * cpstep_density: rho(r) = sum_s occ[s] psi_s(r)^2 / vol, FP64 accumulation.
 * Replaces CP_State_RealSpacePlane::doFFT's square (CP_State_RealSpacePlane.C:349-355),
 * the density reduction (doReduction :484-500, CP_Rho_RealSpacePlane::acceptDensity
 * :398-447) and scaleData with probScale = 1/vol (:630-650).  d_occ: [nstates]
 * (occ*wght_kpt).  d_rho: [nz][ny][nx].
 */
CPSTEP_API int cpstep_density(cpstep_ctx* ctx, const double* d_psi, const double* d_occ,
                   double* d_rho);

/*
 * cpstep_vks_psi: F(G) = wpt * (-2/(nx ny nz)) * FFT^-1[occ * V_KS(r) * psi(r)],
 * wpt = 2 off the Gx=0 plane (GStateSlab::addForces, stateSlab.C:240-272, with
 * no non-local term).  Replaces unpackVks (CP_State_RealSpacePlane.C:530-597),
 * doVksFFT, the inverse transpose and CP_State_GSpacePlane::doIFFT
 * (CP_State_GSpacePlane.C:1590-1612).  If d_eke is not NULL the kinetic term of
 * CP_eke_calc (cp_eke.C:30-140) is fused in: F -= occ*wpt*g^2*psi and
 * d_eke[s] = sum occ*wpt*g^2*|psi|^2 / 2.  d_vks: [nz][ny][nx].
 */
CPSTEP_API int cpstep_vks_psi(cpstep_ctx* ctx, const double* d_psi, const double* d_vks,
                   const double* d_occ, double* d_force, double* d_eke);

/*
 * cpstep_eke: CPNONLOCAL::CP_eke_calc (cp_eke.C:30-140) for all states:
 * F -= occ*wpt*g^2*psi (zero beyond ecut), d_eke[s] = E_kin of state s.
 */
CPSTEP_API int cpstep_eke(cpstep_ctx* ctx, double* d_force, const double* d_psi,
               const double* d_occ, double* d_eke);

/* ---------------------------------------------------------------------------
 * PairCalculator and Ortho.
 *
 * cpstep_pc_overlap: d_c(i,j) = alpha * sum_p wpt_p Re(conj a_i(p) b_j(p))
 *   + beta * d_c(i,j), column-major with leading dimension ldc; a: [na][npts],
 *   b: [nb][npts] packed complex, wpt = 1 on Gx=0 and 2 elsewhere.  With
 *   alpha = 1 this is the reference's forward product: S = 2 psi_r^T psi_r
 *   (symmetric) or lambda = 2 psi_r^T F_r (asymmetric) over the real view with
 *   the Gx=0 rows scaled by 1/sqrt(2) (psi) and sqrt(2) (F)
 *   (PairCalculator::multiplyForward, paircalc/ckPairCalculator.C:682-802;
 *   scaling cp_state_ctrl/CP_State_GSpacePlane.C:1933-1954, :3120-3123).
 *   Split over G with a fixed-order reduction: deterministic.
 * cpstep_pc_backmultiply: out_i(p) = alpha * sum_{j<nin} M(j,i) in_j(p)
 *   + beta * out_i(p) for i < nout, M column-major (ldm): the backward
 *   products psi.T, F.T and psi.gamma (bwMultiplyHelper :1189-1425,
 *   bwMultiplyDynOrthoT :1444-1510).  in/out: [n][npts] packed complex.
 * cpstep_dgemm: column-major BLAS DGEMM semantics on device pointers, the
 *   myGEMM wrapper (ckPairCalculator.C:57-66).
 */
/*
 * cpstep_set_gemm_path: on a CPSTEP_PREC_MIXED context the overlap and
 *   back-multiply products run on the tensor cores (tensor_cores = 1, the
 *   default on compute capability 10.x) as split-BF16 compensated products:
 *   each FP64 element split into BF16 hi + lo, the three products
 *   lo*hi + hi*lo + hi*hi accumulated in FP32 over chunks of 32 reals, the
 *   chunks summed in FP64; the back-multiply adds the diagonal of M in FP64.
 *   tensor_cores = 0 selects the FP64 products.  FP64 contexts always use
 *   FP64.  No counterpart in the reference (its products are DGEMM calls).
 * cpstep_device_errors: error bits recorded by kernels since the last call
 *   (1: a bounded wait of a tensor-core product timed out and its tile was not
 *   written); clears them.  Synchronises the context's stream.
 */
CPSTEP_API int cpstep_set_gemm_path(cpstep_ctx* ctx, int tensor_cores);
CPSTEP_API int cpstep_device_errors(cpstep_ctx* ctx, int* flags);
CPSTEP_API int cpstep_pc_overlap(cpstep_ctx* ctx, const double* d_a, const double* d_b,
                                 int na, int nb, double alpha, double beta, double* d_c,
                                 int ldc);
CPSTEP_API int cpstep_pc_backmultiply(cpstep_ctx* ctx, const double* d_m, int ldm,
                                      const double* d_in, int nin, double* d_out, int nout,
                                      double alpha, double beta);
CPSTEP_API int cpstep_dgemm(cpstep_ctx* ctx, char transa, char transb, int m, int n, int k,
                            double alpha, const double* d_a, int lda, const double* d_b,
                            int ldb, double beta, double* d_c, int ldc);

/*
 * cpstep_ortho_tmat: T = (S/2)^(-1/2) for a symmetric n x n S (device FP64),
 * CPORTHOG::get_iter_Tmat (src_piny_physics_v1.0/abinito_physics/cp_orthog/
 * cp_lowdin.C:180-265) and the Ortho chare iteration (orthog_ctrl/ortho.C:
 * 153-269, :862-985): A = I, B = S/2, C = 3I - A B, B <- B C / 2,
 * A <- C A / 2 until rms(dA) <= tol or max_iter (reference: 1e-15, 10;
 * ortho.h:86-87).  mode bit 0: FP32 iteration followed by an FP64
 * correction that restores T^T (S/2) T = I to FP64 rounding; bit 1: scale
 * by a Gershgorin bound of the spectrum first (converges for eig(S/2) >= 2,
 * where the reference's iteration diverges).  Blocks the host until done.
 * Returns CPSTEP_ERR_NOCONV (T still written) where the reference aborts.
 * iters / rms (may be NULL) receive the iteration count and final rms.
 */
CPSTEP_API int cpstep_ortho_tmat(cpstep_ctx* ctx, const double* d_s, double* d_t, int n,
                                 int mode, double tol, int max_iter, int* iters, double* rms);

/* ---------------------------------------------------------------------------
 * Density side: XC, density FFT, Hartree + local pseudopotential + Ewald.
 *
 * cpstep_set_atoms: atoms and local pseudopotential tables, the data
 *   CP_hart_eext_calc reads from PINY (cp_local/cp_hart_ext.C:72-110):
 *   typ[natm] (0-based type), pos[natm][3] (bohr), q[ntyp] (ionic charges),
 *   spline tables vps[ntyp][4][nspl] = vps0..vps3 on g = gmin_spl + i*dg_spl
 *   (cppseudo->vps0..3, CP_get_vpsnow :433-475), gzvps[ntyp] (the G=0 term)
 *   and the Ewald alpha (genewald->alp_ewd).  Host pointers, copied.
 *   At most CPSTEP_MAX_TYPES types.
 * cpstep_rho_layout: the density sphere's packed order (|G|^2/2 <= 4 Ecut,
 *   countkvec3d/setkvec3d set_cp_ewald.C:230-500, flip_data_set order):
 *   npts, and kx/ky/kz (host, room for cap) when given.
 * cpstep_exc_calc: CPXCFNCTS::CP_exc_calc (cp_xc_fnctl/cp_pz_lda.C:23-170) on
 *   the dense [nz][ny][nx] grid: d_vxc = v_xc(r); d_energies[EXC], [MUXC].
 * cpstep_rho_fft_r2g: rho(G) = (vol/N) sum_r rho(r) e^{-iG.r} on the packed
 *   density sphere (CP_Rho_RealSpacePlane::fftRhoRtoRhoG, CP_Rho_RealSpacePlane.C:831-864).
 * cpstep_hart_eext: CPLOCAL::CP_hart_eext_calc (cp_local/cp_hart_ext.C:56-405):
 *   d_vksg = vks(G) (Hartree + local), d_energies[HART], [EXT], [EWD], and
 *   when d_force is not NULL the local + Ewald atom forces [natm][3].
 * cpstep_vks_fft_g2r: V(r) = sum_G vks(G) e^{+iG.r} (CP_Rho_GHartExt::FFTVks,
 *   CP_Rho_GHartExt.C:532-540).
 * cpstep_vks_from_rho: the chain CP_exc_calc -> fftRhoRtoRhoG -> CP_hart_eext_calc
 *   -> FFTVks -> acceptHartVks (CP_Rho_RealSpacePlane.C:1365-1415):
 *   d_vks_r = v_xc + V_H + V_loc on the grid, the five energies, forces.
 *   With BLYP the gradient correction joins after fftRhoRtoRhoG: the density
 *   gradients (divRhoVksGspace), CP_getGGAFunctional, the White-Bird
 *   divergence (whiteByrdFFT, acceptWhiteByrd); EEXC then includes EXC_GGA.
 * cpstep_set_xc: CPSTEP_XC_PZ_LDA (default) or CPSTEP_XC_BLYP; the BLYP
 *   density cut-off gradient_cutoff (the reference's \gradient_cutoff,
 *   5e-5 when <= 0).  Applies to cpstep_exc_calc, cpstep_vks_from_rho and
 *   the step.
 * cpstep_gga_functional: CPXCFNCTS::CP_getGGAFunctional
 *   (cp_xc_fnctl/cp_grad_rho_ctrl.C:32-193) with Becke 88 and LYP on the dense
 *   grid: d_vks += df/drho; d_gx, d_gy, d_gz (the density gradient on entry)
 *   <- unit(grad rho) df/d|grad rho|; d_energies[EXC_GGA] = E_GGA.  Points
 *   with an exactly zero gradient get zero there (the reference divides 0 by 0).
 * cpstep_eext_grid_size: the EES grid of init_eext_ees
 *   (interface/cp_ewald/set_cp_ewald.C:1419-1497) for a cubic box: the first
 *   set_fftsizes entry >= int(2 scale (2 kmax + 1)) (+1 if below 2 (2 kmax + 1)),
 *   kmax the states' largest |k| on an axis.  Returns the size, or -1.
 * cpstep_set_local_ees: the EES form of cpstep_hart_eext (cp_eext_ees_opt on:
 *   CP_Rho_RHartExt::computeAtmSF, CP_Rho_GHartExt::getHartEextEes,
 *   CPLOCAL::eesAtmBsplineRgrp / eesPackGridRchare / eesHartEextGchare /
 *   eesEwaldGchare / eesAtmForceRchare, cp_hart_ext.C:521-1470): the atoms'
 *   structure factors interpolated by B-splines of order n_interp (8 is
 *   built) on an ngrid^3 grid (cpstep_eext_grid_size) with the Euler weights
 *   b(G); energies, vks(G) and atom forces as the reference computes them in
 *   that form.  Applies to cpstep_hart_eext, cpstep_vks_from_rho and the step
 *   until called with on = 0 (the explicit structure factors, the default).
 *   Needs cpstep_set_atoms first; CPSTEP_ERR_ARG for another order or
 *   ngrid < n_interp.
 * d_energies: device array of CPSTEP_NENERGY doubles; only the named slots are written.
 */
CPSTEP_API int cpstep_set_atoms(cpstep_ctx* ctx, int natm, int ntyp, const int* typ,
                                const double* pos, const double* q, int nspl, double gmin_spl,
                                double dg_spl, const double* vps, const double* gzvps,
                                double alp_ewd);
CPSTEP_API int cpstep_rho_layout(const cpstep_ctx* ctx, int cap, int* npts, int* kx, int* ky,
                                 int* kz);
CPSTEP_API int cpstep_exc_calc(cpstep_ctx* ctx, const double* d_rho, double* d_vxc,
                               double* d_energies);
CPSTEP_API int cpstep_rho_fft_r2g(cpstep_ctx* ctx, const double* d_rho_r, double* d_rhog);
CPSTEP_API int cpstep_hart_eext(cpstep_ctx* ctx, const double* d_rhog, double* d_vksg,
                                double* d_energies, double* d_force);
CPSTEP_API int cpstep_vks_fft_g2r(cpstep_ctx* ctx, const double* d_vksg, double* d_v_r);
CPSTEP_API int cpstep_vks_from_rho(cpstep_ctx* ctx, const double* d_rho_r, double* d_vks_r,
                                   double* d_energies, double* d_force);
CPSTEP_API int cpstep_set_xc(cpstep_ctx* ctx, int functional, double gradient_cutoff);
CPSTEP_API int cpstep_eext_grid_size(int kmax, double scale, int n_interp);
CPSTEP_API int cpstep_set_local_ees(cpstep_ctx* ctx, int on, int ngrid, int n_interp);
CPSTEP_API int cpstep_gga_functional(cpstep_ctx* ctx, const double* d_rho, double* d_gx,
                                     double* d_gy, double* d_gz, double* d_vks,
                                     double* d_energies);

/* ---------------------------------------------------------------------------
 * EES non-local pseudopotential (Kleinman-Bylander s and p channels,
 * src_piny_physics_v1.0/abinito_physics/cp_nonlocal/cp_ees_nonlocal.C).
 *
 * cpstep_nl_grid_size: the NL FFT grid of init_nonlocal_ees
 *   (interface/cp_ewald/set_cp_ewald.C:1329-1400) for a cubic box: the first
 *   set_fftsizes entry >= int(2 scale (kmax+1)) (+1 if below 2 (kmax+1)).
 *   Returns the size, or -1 if the table has none.
 * cpstep_set_nonlocal: channels of the reference's iter_nl loop (lang_v,
 *   mang_v, ityp_v): ch_type (0-based type of cpstep_set_atoms), ch_l in
 *   {0, 1}, ch_m in [-l, l]; vnl[nchan][4][nspl] the channel's radial spline
 *   (vps0..vps3 of its type and l) on the g grid of cpstep_set_atoms; gz0[nchan]
 *   the G = 0 value of an s channel (gzvps0); vnorm[nchan] (vpsnorm).  nkf the
 *   NL grid (cpstep_nl_grid_size), n_interp the B-spline order (8).  Forms the
 *   projector dyp = Ylm b(G) v_l(|G|) of eesSetEesWghtGgrp / eesYlmOnD /
 *   eesProjGchare (:60-240, :594-1236) once.  Host pointers, copied.  Call
 *   after cpstep_set_atoms.  cpstep_cp_step includes the non-local pass once
 *   this is set.
 * cpstep_ees_nonlocal: for every state and channel, projPsiG = conj(dyp psi)
 *   -> NL grid (doNlFFTGtoR) -> Z = sum projPsiR Mn over each atom's
 *   8x8x8 B-spline stencil (eesAtmBsplineRgrp, eesZmatRchare) -> E_NL +=
 *   Z^2 vnorm/vol occ, F_atom -= Z' sum projPsiR dMn, scatter Z' Mn with
 *   Z' = 2 vnorm/vol occ Z (eesEnergyAtmForcRchare) -> NL R->G -> d_fpsi +=
 *   -w conj(dyp projPsiG') (eesPsiForcGspace).  d_energies[E_NL] is written,
 *   d_fatm[natm][3] (may be NULL) accumulated, d_fpsi accumulated.
 */
CPSTEP_API int cpstep_nl_grid_size(int kmax, double scale, int n_interp);
CPSTEP_API int cpstep_set_nonlocal(cpstep_ctx* ctx, int nkf, int n_interp, int nchan,
                                   const int* ch_type, const int* ch_l, const int* ch_m,
                                   const double* vnl, const double* gz0, const double* vnorm);
/* Structure-factor (non-EES) non-local path, l = 0 (the reference's path with
 * EES off: CP_calc_Struct_Fact cp_nonlocal/cp_struct_fact.C:33-221,
 * CP_enl_matrix_calc cp_nlmat.C:20-92, CP_enl_atm_forc_calc and
 * CP_enl_force_calc cp_nl_energy_forc.C:29-182).
 * cpstep_set_nonlocal_sf: channels as cpstep_set_nonlocal, each l = 0, m = 0,
 *   at most one per type; replaces an EES set-up (and cpstep_set_nonlocal
 *   replaces this one).  The step then adds this path's energy and forces.
 * cpstep_sf_nonlocal: for all states, d_energies[NL] = sum_s occ_s sum_a
 *   vnorm_a/vol z_a^2, d_fpsi -= sum_a z'_a S_a, d_fatm (if not NULL) += the
 *   atom forces; z'_a = 2 vnorm_a/vol z_a (no occupation factor in the
 *   forces, as in the reference). */
CPSTEP_API int cpstep_set_nonlocal_sf(cpstep_ctx* ctx, int nchan, const int* ch_type,
                                      const int* ch_l, const int* ch_m, const double* vnl,
                                      const double* gz0, const double* vnorm);
CPSTEP_API int cpstep_sf_nonlocal(cpstep_ctx* ctx, const double* d_psi, const double* d_occ,
                                  double* d_fpsi, double* d_energies, double* d_fatm);
CPSTEP_API int cpstep_ees_nonlocal(cpstep_ctx* ctx, const double* d_psi, const double* d_occ,
                                   double* d_fpsi, double* d_energies, double* d_fatm);

/* ---------------------------------------------------------------------------
 * Integrator and the fused electronic step.
 *
 * cpstep_set_cp_mass: CP coefficient masses of set_cpmass (src_piny_physics_v1.0/
 *   interface/cp_ewald/set_cp_ewald.C:32-74): cmass0 = 4 tau^2 CP_EMAGIC with
 *   tau = tau_fs / TIME_CONV, scaled by (g^2/2)/(cut/2) above cut (Ry), G=0 halved.
 * cpstep_cp_integrate: velocity Verlet of CPINTEGRATE::CP_integrate_dyn /
 *   cp_evolve_vel / get_fictKE (cp_integrate/cp_dynamics.C:29-258) on all
 *   states (with the isokinetic Nose-Hoover chains when cpstep_set_cp_thermostat
 *   switched them on, below): second half kick of the
 *   previous step when iteration > 1, fictitious KE (d_fict_ke, may be NULL),
 *   first half kick, psi += v dt, then the redundant lower Gx=0 half is
 *   overwritten by the conjugate of its partner (sendRedPsi/unpackRedPsi,
 *   CP_State_GSpacePlane.C:2862-3061).  d_force: the constrained force.
 * cpstep_cp_step: one electronic step on orthonormal psi (S = 2 I):
 *   rho -> V_KS (XC, Hartree, local, Ewald) -> F = V.psi + kinetic force
 *   (+ the EES non-local force when cpstep_set_nonlocal was called) ->
 *   lambda = <psi|F> -> the constraint of cpstep_set_constraint (below) ->
 *   Verlet -> S -> T = (S/2)^-1/2 -> psi = (the integrated coefficients).T.
 *   d_energies (CPSTEP_NENERGY doubles, device) receives every slot;
 *   d_atom_force (may be NULL) the local + Ewald (+ non-local) atom forces.
 *   Asynchronous: the Ortho convergence of the step is read by cpstep_step_status.
 *   With the orthoT constraint, iteration 1 returns CPSTEP_ERR_NORB (after the
 *   step) when S of the integrated coefficients fails cp_norb_tol.
 * cpstep_step_status: iterations and convergence flag of the last Ortho launch
 *   (synchronises the context's stream).
 */
CPSTEP_API int cpstep_set_cp_mass(cpstep_ctx* ctx, double tau_fs, double cut_ry);

/*
 * Isokinetic Nose-Hoover chain thermostat of the CP coefficients (ISOKIN_OPT = 1,
 * cp_integrate/cp_dynamics.C:19).  Replaces (ctx form, one chain set per state):
 *   CPINTEGRATE::initCPNHC         cp_integrate/cp_isokin.C:45-141
 *   CPINTEGRATE::cp_isoNHC_update  cp_integrate/cp_isokin.C:150-311
 *   cp_evolve_vel's thermostat calls (cp_dynamics.C:172-193) and the NHC part of
 *   get_fictKE (:231-240)
 * cpstep_set_cp_thermostat: te_ext (K; <= 0 switches the thermostat off and
 *   cpstep_cp_integrate / cpstep_cp_step return to plain velocity Verlet),
 *   tau_fs (cp_tau_nhc), num_nhc (cp_num_nhc_iso, 1..8), nck (cp_nhc_chunk,
 *   1..8), nres (cp_respa_steps_nhc >= 1), nyosh (cp_yosh_steps_nhc in
 *   {1,3,5,7,9}); reference defaults 2, 1, 4, 9 with tau 25 fs.  Each state's
 *   non-redundant coefficients (G=0, the unique Gx=0 points, the rest; each in
 *   packed order) form nck chunks as initCPNHC divides them; masses, barriers
 *   and degrees of freedom as initCPNHC.  The chains start at x = xp = 0,
 *   v = (sqrt(kT/mNHC[0]), 0) (on the isokinetic surface); CPSmplVel's random
 *   sample can be loaded with cpstep_cp_thermostat_state.  Needs the CP masses.
 *   Drops the step graph.
 * cpstep_cp_thermostat_state: set (set = 1) or read (set = 0) the chain state,
 *   host arrays [nstates][nck][num_nhc][2] (xNHC, xNHCP, vNHC; any may be NULL).
 * With the thermostat on, cpstep_cp_integrate and cpstep_cp_step apply
 * cp_isoNHC_update after the second half kick of the previous step (iteration
 * > 1) and before the first half kick, per state and chunk, and the step's
 * d_energies gain CPSTEP_E_NHC_KE and CPSTEP_E_NHC_POT (zero when off).
 */
CPSTEP_API int cpstep_set_cp_thermostat(cpstep_ctx* ctx, double te_ext, double tau_fs,
                                        int num_nhc, int nck, int nres, int nyosh);
CPSTEP_API int cpstep_cp_thermostat_state(cpstep_ctx* ctx, int set, double* h_x, double* h_xp,
                                          double* h_v);
CPSTEP_API int cpstep_cp_integrate(cpstep_ctx* ctx, const double* d_force, double* d_psi,
                                   double* d_vpsi, double dt, int iteration, double* d_fict_ke);
CPSTEP_API int cpstep_cp_step(cpstep_ctx* ctx, double* d_psi, double* d_vpsi,
                              const double* d_occ, double dt, int iteration,
                              double* d_energies, double* d_atom_force);
CPSTEP_API int cpstep_step_status(cpstep_ctx* ctx, int* ortho_iters, int* converged);

/*
 * The orthonormality constraint of cpstep_cp_step.
 * CPSTEP_CONSTRAINT_ORTHO_T (the default): the reference's CP dynamics
 *   (cp_min_opt = 0).  The context carries the non-orthogonal coefficients
 *   psi_no (CP_State_GSpacePlane's packedPlaneDataScr) and orthoT (the T of
 *   the previous step, Ortho::orthoT, orthog_ctrl/ortho.C:358-365).  Per step:
 *     gamma = orthoT lambda              Ortho::acceptSectionLambda (ortho.C:541-583)
 *     F_c = F.orthoT - W psi.gamma       PairCalculator::bwMultiplyDynOrthoT and the
 *                                        gamma product of bwMultiplyHelper
 *                                        (paircalc/ckPairCalculator.C:1444-1510,
 *                                        :1372-1420), unpackLambda / doLambda
 *                                        (CP_State_GSpacePlane.C:2060-2268):
 *                                        W = 1/2 on Gx=0, 1 elsewhere
 *     Verlet on psi_no with F_c; S = overlap(psi_no); T; psi = psi_no.T
 *     max |S - 2I| >= tol_norb (Ortho::maxCheck, ortho.C:461-483) after the
 *     first step: the finite-difference PsiV reset (finiteDifferencePsiV,
 *     CP_State_GSpacePlane.C:3707-3770, order 0): psi_no <- psi,
 *     v = (psi(t+dt) - psi(t)) / dt, orthoT <- I, and the next step has no
 *     second half kick (halfStepEvolve = 0, cp_dynamics.C:58).
 *   Iteration 1 starts from psi_no = psi and orthoT = I unless a state was
 *   loaded with cpstep_dyn_state since the last step.
 * CPSTEP_CONSTRAINT_LOWDIN: F <- F - W psi.lambda (the minimisation
 *   constraint, CP_State_GSpacePlane.C:2079-2088), Verlet on psi itself, then
 *   psi <- psi.T; no state between steps.
 * cpstep_set_constraint: form and tol_norb (cp_norb_tol, reference default
 *   0.003, set_sim_dict.C:1161-1162; > 0).  Drops the step graph and the
 *   carried state.
 * cpstep_dyn_state: read (set = 0) or load (set = 1) the carried state:
 *   device arrays d_psi_no [nstates][npts] complex128 and d_tmat (nstates^2,
 *   column-major), and the host int *h_half_step (the reference's
 *   halfStepEvolve: 0 after a reset, when the next step has no second half
 *   kick; 1 otherwise).  On a read any pointer may be NULL; a load needs both
 *   arrays (h_half_step NULL loads 1).  A load marks the state for the next
 *   step (iteration 1 then keeps it).
 * cpstep_dyn_status: max |S - 2I| of the last step's check and the PsiV
 *   resets so far (synchronises the context's stream); either may be NULL.
 */
#define CPSTEP_CONSTRAINT_ORTHO_T 0
#define CPSTEP_CONSTRAINT_LOWDIN 1
CPSTEP_API int cpstep_set_constraint(cpstep_ctx* ctx, int form, double tol_norb);
CPSTEP_API int cpstep_dyn_state(cpstep_ctx* ctx, int set, double* d_psi_no, double* d_tmat,
                                int* h_half_step);
CPSTEP_API int cpstep_dyn_status(cpstep_ctx* ctx, double* max_dev, int* resets);

/*
 * CUDA graph of the step (no reference counterpart; the reference's step is a
 * Charm++ message flow).  With graphs enabled (the default), cpstep_cp_step
 * and cpstep_cp_step_host with iteration > 1 run one step directly for a new
 * set of (psi, vpsi, occ, dt, energies, atom_force), capture the next one
 * into a graph and replay it while the arguments stay the same.  Setting
 * atoms, non-local data, CP masses, the stream, profiling or the GEMM path
 * drops the graph; profiled steps and iteration 1 always run directly.  If a
 * capture fails the context falls back to direct launches (enabled = 0).
 * cpstep_ctx_graph_status: enabled flag, whether a graph is held, and its
 * kernel count (cpstep_launch_count adds it per replay).
 */
CPSTEP_API int cpstep_ctx_set_graph(cpstep_ctx* ctx, int enable);

/*
 * Launch choices of a context (no reference counterpart; FFTW_MEASURE plans,
 * fftCache.C:252-255, are the nearest relative).  CPSTEP_NTUNE values:
 *   [0] state plane passes: register-shuffle line FFTs (1) or shared-memory
 *       Stockham (0) where both exist;  [1] state plane passes: blocks about
 *       this many times the SM count;  [2] EES plane kernels: the same;
 *   [3] PairCalc overlap split-K: CTAs about this many times the SM count;
 *   [4] mixed contexts: tensor-core products (1) or FP64 (0);
 *   [5] mixed contexts on the tensor cores: the EES non-local pass in G space
 *       (1: its grid sums by Parseval as tensor-core products with separable
 *       B-spline transforms) or through the NL-grid FFTs (0).
 * cpstep_autotune times the candidates of each choice on the caller's psi
 * (device, nstates x npts) and occ with CUDA events and keeps the fastest;
 * ms (may be NULL, CPSTEP_NTUNE doubles) receives the best time (ms) per
 * choice.  Synchronises the stream; uses scratch of about one psi.
 * Choices change results by rounding only; get/set reproduce a tuned run.
 */
#define CPSTEP_NTUNE 6
CPSTEP_API int cpstep_tune_get(const cpstep_ctx* ctx, int* vals, int n);
CPSTEP_API int cpstep_tune_set(cpstep_ctx* ctx, const int* vals, int n);
CPSTEP_API int cpstep_autotune(cpstep_ctx* ctx, const double* d_psi, const double* d_occ,
                               double* ms);

/*
 * Batches of independent systems (no reference counterpart beyond running
 * instances side by side): one context per system, one electronic step of
 * every context per cpstep_batch_step, captured into a single CUDA graph with
 * one branch per context and replayed while the arguments stay the same
 * (iteration 1 and a new argument set run directly; a context's setters force
 * a new capture).  Arrays are indexed by context; atom_force may be NULL (or
 * hold NULL entries).  The graph is launched on the batch's stream
 * (cpstep_batch_set_stream, default the legacy stream); the contexts' own
 * streams are not used by batch steps.  cpstep_batch_status as
 * cpstep_ctx_graph_status.
 */
typedef struct cpstep_batch cpstep_batch;
CPSTEP_API int cpstep_batch_create(cpstep_batch** batch, int nctx, cpstep_ctx* const* ctxs);
CPSTEP_API int cpstep_batch_destroy(cpstep_batch* batch);
CPSTEP_API int cpstep_batch_set_stream(cpstep_batch* batch, void* stream);
CPSTEP_API int cpstep_batch_set_graph(cpstep_batch* batch, int enable);
CPSTEP_API int cpstep_batch_status(cpstep_batch* batch, int* enabled, int* captured,
                                   unsigned long long* kernels);
CPSTEP_API int cpstep_batch_step(cpstep_batch* batch, double* const* d_psi,
                                 double* const* d_vpsi, const double* const* d_occ, double dt,
                                 int iteration, double* const* d_energies,
                                 double* const* d_atom_force);
CPSTEP_API int cpstep_ctx_graph_status(cpstep_ctx* ctx, int* enabled, int* captured,
                                       unsigned long long* kernels);

/*
 * cpstep_set_positions: new atom positions from host memory (natm x 3, bohr),
 *   copied on the context's stream (pinned memory makes it asynchronous); the
 *   structure-factor tables follow on the device.
 * cpstep_cp_step_host: the step as the reference's driver calls it, with host
 *   buffers for what crosses the boundary every MD step: positions in (h_pos,
 *   may be NULL to keep the current ones), energies (CPSTEP_NENERGY doubles)
 *   and atom forces (natm x 3, may be NULL) out.  The coefficients stay on the
 *   device between steps.  Synchronous.
 */
CPSTEP_API int cpstep_set_positions(cpstep_ctx* ctx, const double* h_pos);

/* Ions between electronic steps (CPAIMD).
 * cpstep_ion_forces: CPRSPACEION::CP_getionforce (cp_ions/cp_rspace_ion.C:25-250,
 *   fully periodic, no Grimme term) at the context's current positions and
 *   charges: d_fatm [natm][3] += the real-space Ewald forces;
 *   d_energies[EWD_RS] = pot_ewd_rs + vself + vbgr.
 * cpstep_atoms_integrate: the NVE step of ATOMINTEGRATE::ctrl_atom_integrate
 *   (integration_drivers.C:17-88): on device arrays [natm][3], v += dt/2 f/m
 *   (not when itime == 0), *d_ekin = 1/2 sum m v^2 (may be NULL), v += dt/2 f/m,
 *   x += dt v; the context's positions then follow d_pos (as
 *   cpstep_set_positions).  d_fatm holds the total atom forces (the step's
 *   local, reciprocal Ewald and non-local forces plus cpstep_ion_forces). */
CPSTEP_API int cpstep_ion_forces(cpstep_ctx* ctx, double* d_fatm, double* d_energies);
/*
 * Massive Nose-Hoover chains of the atoms: the NVT branch of ctrl_atom_integrate
 * (iextended_on = 1, isokin_opt = 0; integrate_nvt_2nd_half / _1st_half, applyNHC,
 * computeENHC: classical_physics/integrate/integration_drivers.C:89-190, :358-565).
 * cpstep_set_atom_thermostat: len_nhc (1..5; 0 returns to NVE), nres, nyosh
 *   ({1,3,5,7,9}), h_kT [natm] (AtomNHC::kT) and h_mnhc [natm][len_nhc]
 *   (AtomNHC::m, PhysicsAtomPosInit.C:229-256); needs the atoms; chain
 *   velocities and posKT start at zero.  cpstep_atoms_integrate then runs, per
 *   atom and Cartesian component: v += dt/2 f/m and applyNHC (itime > 0), E_kin,
 *   the NHC energies, applyNHC, v += dt/2 f/m, x += dt v.
 * cpstep_atom_thermostat_state: set (set = 1) or read the chain velocities
 *   h_vnhc [natm][3][len_nhc] (AtomNHC::vx/vy/vz) and h_pos_kt [natm]
 *   (AtomNHC::posKT); on read, h_energies2 (may be NULL) = {E_kin NHC, pot NHC}
 *   of the last cpstep_atoms_integrate.
 */
CPSTEP_API int cpstep_set_atom_thermostat(cpstep_ctx* ctx, int len_nhc, int nres, int nyosh,
                                          const double* h_kT, const double* h_mnhc);
CPSTEP_API int cpstep_atom_thermostat_state(cpstep_ctx* ctx, int set, double* h_vnhc,
                                            double* h_pos_kt, double* h_energies2);
CPSTEP_API int cpstep_atoms_integrate(cpstep_ctx* ctx, int itime, double* d_pos, double* d_vel,
                                      const double* d_fatm, const double* d_mass, double dt,
                                      double* d_ekin);
CPSTEP_API int cpstep_cp_step_host(cpstep_ctx* ctx, double* d_psi, double* d_vpsi,
                                   const double* d_occ, double dt, int iteration,
                                   const double* h_pos, double* h_energies,
                                   double* h_atom_force);

/*
 * cpstep_pc_overlap_noalloc: the overlap product of cpstep_pc_overlap,
 * d_c(i,j) = alpha * sum_p w_p Re(conj a_i(p) b_j(p)) + beta * d_c(i,j)
 * (column-major, ldc), for callers that must not allocate device memory: a
 * host application whose device memory is owned by its own pool or has a
 * fixed budget, or code running where cudaMalloc is not allowed (a host
 * callback, a library that promises its user no allocations).  It has no
 * counterpart in the reference, which always multiplies into memory its
 * chares own.  It needs no context and allocates nothing: the split-K
 * partial tiles go to a fixed 8 MiB device array inside libcpstep
 * (2^20 doubles), which every GPU that loads the library keeps until the
 * process exits.  Limit: na * nb <= 2^20 (e.g. 1024 x 1024 states); larger
 * sizes return CPSTEP_ERR_ARG.  d_a: [na][npts], d_b: [nb][npts] packed
 * complex128; d_w: per-point weights [npts] (1 on the Gx=0 plane and 2
 * elsewhere give the reference's S and lambda) or NULL for all 1;
 * stream: a cudaStream_t or NULL.
 * The first call on a device looks the array's device address up
 * (cudaGetSymbolAddress) with that device current, and so does the first call
 * after the device's current context has changed (its unique ID, cuCtxGetId,
 * is compared on every call: a cudaDeviceReset or a primary-context reset by
 * the application makes a new context with its own copy of the array): make
 * those calls before any stream capture.  Every call uses the same array: two
 * calls that can run at the same time on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.
 */
CPSTEP_API int cpstep_pc_overlap_noalloc(const double* d_a, const double* d_b, int na, int nb,
                                         int npts, const double* d_w, double alpha,
                                         double beta, double* d_c, int ldc, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CPSTEP_H */
