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

#define CPSTEP_PREC_FP64 0    /* plain FP64 path: the drop-in */
#define CPSTEP_PREC_MIXED 1   /* FP32 FFT/density/V.psi, FP64 accumulation, split GEMMs */

typedef struct cpstep_ctx cpstep_ctx;

/* Library version (major*10000 + minor*100 + patch). */
CPSTEP_API int cpstep_version(void);

/* Text of the last error on this thread ("" if none). */
CPSTEP_API const char* cpstep_last_error(void);

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

#ifdef __cplusplus
}
#endif
#endif /* CPSTEP_H */
