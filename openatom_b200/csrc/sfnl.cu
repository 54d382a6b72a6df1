// Structure-factor (non-EES) nonlocal pseudopotential, l = 0 channels (the
// reference's path when EES is off; it hard-wires l = 0):
//
//   CPNONLOCAL::CP_calc_Struct_Fact    src_piny_physics_v1.0/abinito_physics/cp_nonlocal/
//                                      cp_struct_fact.C:33-221 (get_rad_proj :225-258)
//   CPNONLOCAL::CP_enl_matrix_calc     cp_nlmat.C:20-92
//   CPNONLOCAL::CP_enl_atm_forc_calc   cp_nl_energy_forc.C:121-182
//   CPNONLOCAL::CP_enl_force_calc      cp_nl_energy_forc.C:29-114
//
// Per non-local atom a and packed point G (double pack, w = 1 on kx = 0, else 2):
//   S_a(G)   = conj(w e^{iG.R_a}) y00 v_0(|G|),  S_a^d(G) = -i g_d S_a(G)
//   z_a = <S_a|psi> over the real view, E_NL = sum_s occ_s sum_a vnorm_a/vol z_a^2,
//   z'_a = 2 vnorm_a/vol z_a, F_a^d -= z'_a z_a^d, F_psi -= sum_a z'_a S_a
// (the atom and psi forces carry no occupation factor, as in the reference).
// The reference's per-state DGEMVs become products over all states: the
// structure factors of the n non-local atoms and their gradient copies as one
// [4 n][2 npts] real matrix, Z = that . psi^T through the PairCalc overlap,
// the scaled Z back through the PairCalc back-multiply (tensor cores in a
// mixed context, FP64 otherwise).
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.cuh"

namespace sfnl {

// rows [4 n][2 npts]: r < n S_r, then S^x, S^y, S^z; blockIdx.y = row r < n
__global__ void k_sf(const int* __restrict__ kx, const int* __restrict__ ky,
                     const int* __restrict__ kz, int npts, const double* __restrict__ frac,
                     const int* __restrict__ atom, const int* __restrict__ ptab,
                     const double* __restrict__ proj, int n, const double* __restrict__ hmati,
                     double* __restrict__ rows) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (p >= npts) return;
  const int a = atom[r];
  const int x = kx[p], y = ky[p], z = kz[p];
  // G.R = 2 pi k.(hmati R), the argument reduced to [-1/2, 1/2] turns
  double t = (double)x * frac[3 * a] + (double)y * frac[3 * a + 1] + (double)z * frac[3 * a + 2];
  t -= rint(t);
  double sn, cs;
  sincospi(2.0 * t, &sn, &cs);
  const double pv = (x == 0 ? 1.0 : 2.0) * proj[(size_t)ptab[r] * npts + p];
  const size_t ld = 2 * (size_t)npts;
  rows[(size_t)r * ld + 2 * p] = pv * cs;
  rows[(size_t)r * ld + 2 * p + 1] = -pv * sn;
  const double tpi = 2.0 * M_PI;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double g = tpi * ((double)x * hmati[3 * d] + (double)y * hmati[3 * d + 1] +
                            (double)z * hmati[3 * d + 2]);
    double* o = rows + (size_t)((d + 1) * n + r) * ld + 2 * p;
    o[0] = -g * pv * sn;
    o[1] = -g * pv * cs;
  }
}

// one block per state: E_NL of the state, z' into zs[s][ldz], atom forces of
// the state into fnl[s][natm][3] (zero for atoms without an l = 0 channel)
__global__ void k_sf_glue(const double* __restrict__ Z, int n, int nstates,
                          const int* __restrict__ atom, const double* __restrict__ vn,
                          const double* __restrict__ occ, int natm, double* __restrict__ zs,
                          int ldz, double* __restrict__ enl_s, double* __restrict__ fnl) {
  __shared__ double red[32];
  const int s = blockIdx.x;
  const double* zc = Z + (size_t)s * 4 * n;
  double* f = fnl + (size_t)s * natm * 3;
  for (int i = threadIdx.x; i < 3 * natm; i += blockDim.x) f[i] = 0.0;
  __syncthreads();
  double e = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const double z = zc[r], norm = vn[r];
    e += z * z * norm;
    const double zp = 2.0 * norm * z;
    zs[(size_t)s * ldz + r] = zp;
    const int a = atom[r];
#pragma unroll
    for (int d = 0; d < 3; ++d) f[3 * a + d] = -zp * zc[(d + 1) * n + r];
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) enl_s[s] = e * occ[s];
}

// E_NL = sum over states, atom forces += sum over states (fixed order)
__global__ void k_sf_finish(const double* __restrict__ enl_s, const double* __restrict__ fnl,
                            int nstates, int natm, double* __restrict__ energies,
                            double* __restrict__ fatm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && energies) {
    double e = 0.0;
    for (int s = 0; s < nstates; ++s) e += enl_s[s];
    energies[CPSTEP_E_NL] = e;
  }
  if (fatm && i < 3 * natm) {
    double f = 0.0;
    for (int s = 0; s < nstates; ++s) f += fnl[(size_t)s * 3 * natm + i];
    fatm[i] += f;
  }
}

}  // namespace sfnl

void sf_free(cpstep_ctx* c) {
  SfData& f = c->sf;
  cudaFree(f.atom); cudaFree(f.ptab); cudaFree(f.proj); cudaFree(f.vn); cudaFree(f.rows);
  cudaFree(f.z); cudaFree(f.zs); cudaFree(f.enl_s); cudaFree(f.fnl);
  f = SfData{};
}

// Channels as cpstep_set_nonlocal's, every one l = 0 (m = 0), at most one per
// type; the projector y00 v_0(|G|) per type and point once (get_rad_proj).
int sf_set(cpstep_ctx* c, int nchan, const int* ch_type, const int* ch_l, const int* ch_m,
           const double* vnl, const double* gz0, const double* vnorm) {
  const AtomData& at = c->atoms;
  if (at.natm <= 0) {
    cpstep_set_error("set_nonlocal_sf: call cpstep_set_atoms first");
    return CPSTEP_ERR_STATE;
  }
  std::vector<int> chan_of_type(at.ntyp, -1);
  for (int k = 0; k < nchan; ++k) {
    if (ch_type[k] < 0 || ch_type[k] >= at.ntyp || ch_l[k] != 0 || ch_m[k] != 0 ||
        chan_of_type[ch_type[k]] >= 0) {
      cpstep_set_error("set_nonlocal_sf: channel %d (type %d, l %d, m %d): the structure-factor "
                       "path takes one l = 0 channel per type", k, ch_type[k], ch_l[k], ch_m[k]);
      return CPSTEP_ERR_ARG;
    }
    chan_of_type[ch_type[k]] = k;
  }
  // atom types on the host (the context keeps them on the device)
  std::vector<int> typ(at.natm);
  CPSTEP_CUDA_TRY(cudaMemcpy(typ.data(), at.typ, sizeof(int) * at.natm, cudaMemcpyDeviceToHost));
  std::vector<int> atom, ptab, tab_of_type(at.ntyp, -1);
  std::vector<double> vn;
  int ntab = 0;
  for (int t = 0; t < at.ntyp; ++t)
    if (chan_of_type[t] >= 0) tab_of_type[t] = ntab++;
  for (int t = 0; t < at.ntyp; ++t)  // non-local atoms in type order
    for (int a = 0; a < at.natm; ++a)
      if (typ[a] == t && chan_of_type[t] >= 0) {
        atom.push_back(a);
        ptab.push_back(tab_of_type[t]);
        vn.push_back(vnorm[chan_of_type[t]] / c->vol);
      }
  const int n = (int)atom.size(), np = c->npts;
  if (n == 0) {
    cpstep_set_error("set_nonlocal_sf: no atom has an l = 0 channel");
    return CPSTEP_ERR_ARG;
  }
  // y00 v_0(|G|) per projector table (get_rad_proj: the knot below g, cubic in h)
  std::vector<double> proj((size_t)ntab * np);
  const double y00 = 1.0 / sqrt(4.0 * M_PI), tpi = 2.0 * M_PI;
  const double* h = c->hmati;
  for (int t = 0; t < at.ntyp; ++t) {
    const int k = chan_of_type[t];
    if (k < 0) continue;
    const double* v = vnl + (size_t)k * 4 * at.nspl;
    for (int p = 0; p < np; ++p) {
      const int ka = c->h_kx[p], kb = c->h_ky[p], kc = c->h_kz[p];
      const double gx = tpi * (ka * h[0] + kb * h[1] + kc * h[2]);
      const double gy = tpi * (ka * h[3] + kb * h[4] + kc * h[5]);
      const double gz = tpi * (ka * h[6] + kb * h[7] + kc * h[8]);
      const double g = sqrt(gx * gx + gy * gy + gz * gz);
      double val;
      if (g != 0.0) {
        int iii = (int)((g - at.gmin) / at.dg) + 1;
        iii = std::min(iii, at.nspl);
        iii = std::max(iii, 1);
        const double hh = g - ((double)(iii - 1) * at.dg + at.gmin);
        const int i = iii - 1;
        val = ((v[3 * at.nspl + i] * hh + v[2 * at.nspl + i]) * hh + v[at.nspl + i]) * hh + v[i];
      } else {
        val = gz0[k];
      }
      proj[(size_t)tab_of_type[t] * np + p] = y00 * val;
    }
  }
  sf_free(c);
  graph_drop(c);
  SfData& f = c->sf;
  f.n = n;
  f.ldz = (n + 1) / 2 * 2;
  auto up = [&](auto** d, const auto& hv) -> int {
    CPSTEP_CUDA_TRY(cudaMalloc(d, sizeof(hv[0]) * hv.size()));
    CPSTEP_CUDA_TRY(cudaMemcpy(*d, hv.data(), sizeof(hv[0]) * hv.size(), cudaMemcpyHostToDevice));
    return CPSTEP_OK;
  };
  int rc;
  if ((rc = up(&f.atom, atom)) || (rc = up(&f.ptab, ptab)) || (rc = up(&f.proj, proj)) ||
      (rc = up(&f.vn, vn)))
    return rc;
  const int S = c->nstates;
  CPSTEP_CUDA_TRY(cudaMalloc(&f.rows, sizeof(double) * 4 * (size_t)n * 2 * np));
  CPSTEP_CUDA_TRY(cudaMalloc(&f.z, sizeof(double) * 4 * (size_t)n * S));
  CPSTEP_CUDA_TRY(cudaMalloc(&f.zs, sizeof(double) * (size_t)f.ldz * S));
  CPSTEP_CUDA_TRY(cudaMemset(f.zs, 0, sizeof(double) * (size_t)f.ldz * S));
  CPSTEP_CUDA_TRY(cudaMalloc(&f.enl_s, sizeof(double) * S));
  CPSTEP_CUDA_TRY(cudaMalloc(&f.fnl, sizeof(double) * (size_t)S * at.natm * 3));
  f.on = 1;
  nl_free(c);  // the EES path and this one exclude each other
  return CPSTEP_OK;
}

// E_NL -> energies[NL], fpsi -= sum_a z'_a S_a, fatm += atom forces (if given)
int sf_run(cpstep_ctx* c, const double* psi, const double* occ, double* fpsi, double* energies,
           double* fatm) {
  SfData& f = c->sf;
  if (!f.on) {
    cpstep_set_error("sf_nonlocal: call cpstep_set_nonlocal_sf first");
    return CPSTEP_ERR_STATE;
  }
  const int S = c->nstates, np = c->npts, K = 2 * np, n = f.n, natm = c->atoms.natm;
  sfnl::k_sf<<<dim3(cdiv(np, 128), n), 128, 0, c->stream>>>(c->d_kx, c->d_ky, c->d_kz, np,
                                                            c->atoms.frac, f.atom, f.ptab,
                                                            f.proj, n, c->d_hmati, f.rows);
  CPSTEP_LAUNCH_CHECK();
  if (int rc = pc_overlap_launch(c, f.rows, psi, 4 * n, S, K, nullptr, 1.0, 0.0, f.z, 4 * n))
    return rc;
  sfnl::k_sf_glue<<<S, 128, 0, c->stream>>>(f.z, n, S, f.atom, f.vn, occ, natm, f.zs, f.ldz,
                                            f.enl_s, f.fnl);
  CPSTEP_LAUNCH_CHECK();
  if (int rc = pc_backmul_launch(c, f.zs, f.ldz, f.rows, K, fpsi, K, S, n, K, -1.0, 1.0))
    return rc;
  sfnl::k_sf_finish<<<cdiv(std::max(1, 3 * natm), 128), 128, 0, c->stream>>>(
      f.enl_s, f.fnl, S, natm, energies, fatm);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}
