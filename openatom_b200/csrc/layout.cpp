// Host-side construction of the reference's packed G-vector layout.
//
// setkvec3d_sm        src_piny_physics_v1.0/interface/cp_ewald/set_cp_ewald.C:523-680
// calc_cutoff/radixme set_cp_ewald.C:124-225, :751-818, set_fftsizes :1505-1690
// flip_data_set       src_charm_driver/utility/para_grp_parse.C:178-286
// processState        src_charm_driver/utility/util.C:1331-1642
// get_chareG_line_prms para_grp_parse.C:21-170
// sort_kxky           util.C:2223-2247
// readStateIntoRuns   util.C:861-1099
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>
#include "../../include/cpstep.h"

void cpstep_set_error(const char* fmt, ...);

namespace {

// the reference's FFT size table (set_fftsizes): sizes whose factors the
// reference FFT libraries handle, ascending (112 repeated and 100 absent there)
const int kFftSizes[] = {
    4,   6,   8,   10,  12,  14,  16,  18,  20,  22,  24,  28,  30,  32,  36,  40,  42,  44,
    48,  56,  60,  64,  66,  70,  72,  80,  84,  88,  90,  96,  112, 112, 120, 128, 128, 132,
    140, 144, 154, 160, 168, 176, 180, 192, 198, 210, 220, 224, 240, 252, 256, 264, 280, 288,
    308, 320, 330, 336, 352, 360, 384, 396, 420, 440, 448, 462, 480, 504, 512, 528, 560, 576,
    616, 630, 640, 660, 672, 704, 720, 768, 770, 792, 840, 880, 896, 924, 960, 990, 1008, 1024};

// init_nonlocal_ees (set_cp_ewald.C:1329-1400), one axis
int nl_grid_size_of(int kmax, double scale, int n_interp) {
  const int nk = kmax + 1;
  int nkf = (int)(2.0 * scale * (double)nk);
  if (nkf < 2 * nk) ++nkf;
  for (int k : kFftSizes)
    if (k >= nkf) return k >= n_interp ? k : -1;
  return -1;
}

int kmax_of(double L, double ecut_ry) {
  double ecut_ha = 0.5 * ecut_ry;
  double temp = std::sqrt(ecut_ha * 0.5) / (M_PI * (1.0 / L));
  int it = (int)temp;
  if (temp - (double)it > 0.99) ++it;
  return it;
}

int radix_of(int kmax) {
  int kk = 2 * (2 * kmax + 1);
  for (int k : kFftSizes)
    if (k >= kk) return k;
  return -1;
}

struct K3 {
  int a, b, c;
};

std::vector<K3> half_sphere(double L, double ecut_ha, int kmax) {
  const double h = 1.0 / L, tpi = 2.0 * M_PI;
  auto en = [&](int a, int b, int c) {
    double x = a * h * tpi, y = b * h * tpi, z = c * h * tpi;
    return (x * x + y * y + z * z) * 0.5;
  };
  std::vector<K3> v;
  int i = 1;
  for (; i <= kmax; ++i)
    if (en(i, 0, 0) > ecut_ha) break;
  int kamax = i - 1;
  for (int ka = 0; ka <= kamax; ++ka) {
    int kbmin = (ka == 0) ? 0 : -kmax;
    for (i = kbmin; i <= 0; ++i)
      if (en(ka, i, 0) <= ecut_ha) break;
    kbmin = i;
    for (i = 1; i <= kmax; ++i)
      if (en(ka, i, 0) > ecut_ha) break;
    int kbmax = i - 1;
    for (int kb = kbmin; kb <= kbmax; ++kb) {
      int kcmin = (ka == 0 && kb == 0) ? 1 : -kmax;
      for (i = kcmin; i <= 0; ++i)
        if (en(ka, kb, i) <= ecut_ha) break;
      kcmin = i;
      for (i = 1; i <= kmax; ++i)
        if (en(ka, kb, i) > ecut_ha) break;
      int kcmax = i - 1;
      for (int kc = kcmin; kc <= kcmax; ++kc) v.push_back({ka, kb, kc});
    }
  }
  v.push_back({0, 0, 0});  // G=0 last, as PINY stores it
  return v;
}

// Gx=0 half plane mirrored in front, G=0 between, rest unchanged.
bool flip(const std::vector<K3>& in, std::vector<K3>& out) {
  int n = (int)in.size();
  int np0 = 0;
  for (const K3& k : in) np0 += (k.a == 0);
  const K3& last = in[n - 1];
  if (last.a || last.b || last.c) return false;
  for (int i = 0; i < np0 - 1; ++i)
    if (in[i].a != 0) return false;
  out.clear();
  out.reserve(n + np0 - 1);
  for (int i = 0; i < np0 - 1; ++i) {
    const K3& k = in[np0 - 2 - i];
    out.push_back({k.a, -k.b, -k.c});
  }
  out.push_back({0, 0, 0});
  for (int i = 0; i < n - 1; ++i) out.push_back(in[i]);
  return true;
}

bool chunk_params(int nktot, int nchunk, const std::vector<int>& npts, std::vector<int>& nline_grp) {
  int nline = (int)npts.size();
  if (nchunk > nline || nchunk < 1) return false;
  double dev_min = 0.0;
  int nbal_min = 0, first = 0;
  int mmm = nktot / nchunk;
  for (int ibal = 0; ibal <= mmm - 1; ++ibal) {
    int ntarg = nktot / nchunk;
    if (ntarg > ibal) ntarg -= ibal;
    int nmax = 0, nmin = nktot, nnow = 0, ic = 0;
    for (int i = 0; i < nline; ++i) {
      nnow += npts[i];
      if (nnow >= ntarg && ic < nchunk - 1) {
        ++ic;
        nmin = std::min(nmin, nnow);
        nmax = std::max(nmax, nnow);
        nnow = 0;
      }
    }
    nmin = std::min(nmin, nnow);
    nmax = std::max(nmax, nnow);
    double dev = 100.0 * (double)(nmax - nmin) / (double)std::max(nmin, 1);
    if (ic == nchunk - 1 && (dev < dev_min || first == 0)) {
      first = 1;
      dev_min = dev;
      nbal_min = ibal;
    }
  }
  if (!first) return false;
  int ntarg = nktot / nchunk;
  if (ntarg > nbal_min) ntarg -= nbal_min;
  nline_grp.assign(nchunk, 0);
  std::vector<int> pts(nchunk, 0);
  int ic = 0;
  for (int i = 0; i < nline; ++i) {
    pts[ic] += npts[i];
    nline_grp[ic] += 1;
    if (pts[ic] >= ntarg && ic < nchunk - 1) ++ic;
  }
  for (int i = 0; i < nchunk; ++i)
    if (nline_grp[i] == 0 || pts[i] == 0) return false;
  return true;
}

struct Line {
  int start, end;
};

std::vector<Line> lines_of(const std::vector<K3>& k) {
  std::vector<Line> L;
  int s = 0;
  for (int i = 1; i <= (int)k.size(); ++i) {
    if (i == (int)k.size() || k[i].a != k[i - 1].a || k[i].b != k[i - 1].b) {
      L.push_back({s, i});
      s = i;
    }
  }
  return L;
}

bool process(const std::vector<K3>& in, int nchunk, std::vector<K3>& out) {
  for (size_t i = 1; i < in.size(); ++i) {
    if (in[i].a < in[i - 1].a) return false;
    if (in[i].a == in[i - 1].a && in[i].b < in[i - 1].b) return false;
    if (in[i].a == in[i - 1].a && in[i].b == in[i - 1].b && in[i].c != in[i - 1].c + 1) return false;
  }
  std::vector<Line> L = lines_of(in);
  int nline = (int)L.size();
  if (nchunk > nline) return false;
  // round-robin deal of the lines to the chunks
  std::vector<K3> dealt;
  dealt.reserve(in.size());
  for (int i = 0; i < nchunk; ++i)
    for (int j = i; j < nline; j += nchunk)
      for (int p = L[j].start; p < L[j].end; ++p) dealt.push_back(in[p]);
  std::vector<Line> L2 = lines_of(dealt);
  std::vector<int> npts(L2.size());
  for (size_t i = 0; i < L2.size(); ++i) npts[i] = L2[i].end - L2[i].start;
  std::vector<int> nline_grp;
  if (!chunk_params((int)dealt.size(), nchunk, npts, nline_grp)) return false;
  // sort the lines of every chunk on (kx, ky)
  out.clear();
  out.reserve(dealt.size());
  int loff = 0;
  for (int c = 0; c < nchunk; ++c) {
    std::vector<int> idx(nline_grp[c]);
    std::iota(idx.begin(), idx.end(), loff);
    std::sort(idx.begin(), idx.end(), [&](int a, int b) {
      const K3 &ka = dealt[L2[a].start], &kb = dealt[L2[b].start];
      return ka.a != kb.a ? ka.a < kb.a : ka.b < kb.b;
    });
    for (int l : idx)
      for (int p = L2[l].start; p < L2[l].end; ++p) out.push_back(dealt[p]);
    loff += nline_grp[c];
  }
  return true;
}

bool make_runs(const std::vector<K3>& k, int nx, int ny, int nz, std::vector<int>& runs) {
  runs.clear();
  auto wrap = [](int v, int m) { return v < 0 ? v + m : v; };
  auto push = [&](int x, int y, int z, int off, int len) {
    int r[7] = {x, y, z, off, len, 1, nz};
    runs.insert(runs.end(), r, r + 7);
  };
  int n = (int)k.size();
  int cx = wrap(k[0].a, nx), cy = wrap(k[0].b, ny), cz = wrap(k[0].c, nz);
  int tmpz = cz, rsum = 0, rlen = 1;
  if (k[0].c >= 0) push(cx, cy, cz, rsum, 0);
  for (int p = 1; p < n; ++p) {
    int x = wrap(k[p].a, nx), y = wrap(k[p].b, ny), z = wrap(k[p].c, nz);
    if (z == tmpz + 1 && x == cx && y == cy) {
      ++rlen;
      ++tmpz;
    } else {
      push(cx, cy, cz, rsum, rlen);
      rsum += rlen;
      if ((cx != x || cy != y) && k[p - 1].c < 0) push(cx, cy, 0, rsum, 0);
      if ((cx != x || cy != y) && k[p].c >= 0) push(x, y, 0, rsum, 0);
      cx = x; cy = y; cz = z; tmpz = z; rlen = 1;
    }
  }
  push(cx, cy, cz, rsum, rlen);
  rsum += rlen;
  if (k[n - 1].c < 0) push(cx, cy, 0, rsum, 0);
  return rsum == n && (runs.size() / 7) % 2 == 0;
}

}  // namespace

int nl_grid_size(int kmax, double scale, int n_interp) {
  return nl_grid_size_of(kmax, scale, n_interp);
}

// init_eext_ees (set_cp_ewald.C:1419-1497), one axis: the same rule on the
// density sphere's 2 (2 kmax + 1)
int eext_grid_size(int kmax, double scale, int n_interp) {
  const int nk = 2 * kmax + 1;
  int nkf = (int)(2.0 * scale * (double)nk);
  if (nkf < 2 * nk) ++nkf;
  for (int k : kFftSizes)
    if (k >= nkf) return k >= n_interp ? k : -1;
  return -1;
}

extern "C" int cpstep_layout_sizes(double box_len, double ecut_ry, int* kmax, int* nfft,
                                   int* nktot_half, int* npts) {
  if (!(box_len > 0) || !(ecut_ry > 0)) {
    cpstep_set_error("layout_sizes: box and cutoff must be positive");
    return CPSTEP_ERR_ARG;
  }
  int km = kmax_of(box_len, ecut_ry);
  std::vector<K3> hs = half_sphere(box_len, 0.5 * ecut_ry, km);
  int np0 = 0;
  for (const K3& k : hs) np0 += (k.a == 0);
  if (kmax) *kmax = km;
  if (nfft) *nfft = radix_of(km);
  if (nktot_half) *nktot_half = (int)hs.size() - 1;
  if (npts) *npts = (int)hs.size() + np0 - 1;
  return CPSTEP_OK;
}

extern "C" int cpstep_layout_build(double box_len, double ecut_ry, int nchareG, int nfft,
                                   int npts_cap, int* kx, int* ky, int* kz, int* npts,
                                   int runs_cap, int* runs, int* nruns) {
  if (!(box_len > 0) || !(ecut_ry > 0) || !kx || !ky || !kz || !npts) {
    cpstep_set_error("layout_build: bad argument");
    return CPSTEP_ERR_ARG;
  }
  int km = kmax_of(box_len, ecut_ry);
  if (nfft < 2 * (2 * km + 1)) {
    cpstep_set_error("layout_build: nfft %d below 2*(2*kmax+1) = %d", nfft, 2 * (2 * km + 1));
    return CPSTEP_ERR_ARG;
  }
  std::vector<K3> hs = half_sphere(box_len, 0.5 * ecut_ry, km), fl, pr;
  if (!flip(hs, fl)) {
    cpstep_set_error("layout_build: flip_data_set check failed");
    return CPSTEP_ERR_LAYOUT;
  }
  if (nchareG <= 0) {
    int kxmax = 0;
    for (const K3& k : fl) kxmax = std::max(kxmax, k.a);
    nchareG = kxmax + 1;  // gExpandFact = 1
  }
  if (!process(fl, nchareG, pr)) {
    cpstep_set_error("layout_build: processState failed (nchareG %d)", nchareG);
    return CPSTEP_ERR_LAYOUT;
  }
  if ((int)pr.size() > npts_cap) {
    cpstep_set_error("layout_build: npts_cap %d < %d", npts_cap, (int)pr.size());
    return CPSTEP_ERR_ARG;
  }
  for (size_t i = 0; i < pr.size(); ++i) {
    kx[i] = pr[i].a;
    ky[i] = pr[i].b;
    kz[i] = pr[i].c;
  }
  *npts = (int)pr.size();
  if (runs) {
    std::vector<int> rv;
    if (!make_runs(pr, nfft, nfft, nfft, rv)) {
      cpstep_set_error("layout_build: run descriptors broken");
      return CPSTEP_ERR_LAYOUT;
    }
    int nr = (int)rv.size() / 7;
    if (nr > runs_cap) {
      cpstep_set_error("layout_build: runs_cap %d < %d", runs_cap, nr);
      return CPSTEP_ERR_ARG;
    }
    std::copy(rv.begin(), rv.end(), runs);
    if (nruns) *nruns = nr;
  }
  return CPSTEP_OK;
}

// Density sphere |G|^2/2 <= 4 ecut_Ha (countkvec3d/setkvec3d, set_cp_ewald.C:230-500,
// with the kmaxv = 2 kmax_cp loop bounds of calc_cutoff :205-207), in flip_data_set
// order as one chunk: its z-lines are already contiguous and (kx, ky)-sorted.
int cpstep_density_layout(double box_len, double ecut_ry, int nfft, std::vector<int>& kx,
                          std::vector<int>& ky, std::vector<int>& kz, std::vector<int>& runs) {
  int km = kmax_of(box_len, ecut_ry);
  std::vector<K3> hs = half_sphere(box_len, 2.0 * ecut_ry, 2 * km), fl;
  if (!flip(hs, fl)) return CPSTEP_ERR_LAYOUT;
  int kxmax = 0, kymax = 0, kzmax = 0;
  for (const K3& k : fl) {
    kxmax = std::max(kxmax, std::abs(k.a));
    kymax = std::max(kymax, std::abs(k.b));
    kzmax = std::max(kzmax, std::abs(k.c));
  }
  if (2 * kxmax + 2 > nfft || 2 * kymax + 1 > nfft || 2 * kzmax + 1 > nfft) return CPSTEP_ERR_ARG;
  kx.resize(fl.size());
  ky.resize(fl.size());
  kz.resize(fl.size());
  for (size_t i = 0; i < fl.size(); ++i) {
    kx[i] = fl[i].a;
    ky[i] = fl[i].b;
    kz[i] = fl[i].c;
  }
  return make_runs(fl, nfft, nfft, nfft, runs) ? CPSTEP_OK : CPSTEP_ERR_LAYOUT;
}
