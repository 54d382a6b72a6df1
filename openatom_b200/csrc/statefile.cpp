// State files in the reference's format (host code, no GPU).
//
//   write: writeStateFile (src_charm_driver/utility/util.C:1955-2180) with
//          sort_psi_output (:2180-2220): the points sorted by
//          (kz - kzmin) + (ky - kymin) nz + (kx - kxmin) nz ny, the ones after
//          G=0 in that order (the stored half sphere) and then G=0; header
//          "npts nx ny nz".  Text lines "%g %g %d %d %d \n"; binary records
//          double re, double im, int kx, ky, kz (28 bytes, no padding) after
//          four int header words; the gz variants through zlib with ".gz"
//          appended to the name (options 2 and 3 of the reference).
//   read:  readState (util.C:1107-1330): header, then records up to and
//          including G=0 (double pack), and the packing of processState /
//          flip_data_set (para_grp_parse.C:178-286): every point of the
//          caller's packed layout takes the record with its (kx,ky,kz); the
//          redundant Gx=0 points (kx = 0 and ky < 0, or ky = 0 and kz < 0)
//          take the conjugate of their partner (0,-ky,-kz).
#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/cpstep.h"

void cpstep_set_error(const char* fmt, ...);

namespace {

struct Rec {
  double re, im;
  int x, y, z;
};

long long key3(int x, int y, int z) {
  return ((long long)(x + 4096) << 26) | ((long long)(y + 4096) << 13) | (long long)(z + 4096);
}

bool redundant(int x, int y, int z) { return x == 0 && (y < 0 || (y == 0 && z < 0)); }

// Output order of writeStateFile: indices sorted by the sort_psi_output key
// (unique per point), then the position of G=0 in that order.
void out_order(int n, const int* kx, const int* ky, const int* kz, std::vector<int>& idx,
               int& istrt) {
  int xmin = kx[0], ymin = ky[0], zmin = kz[0], ymax = ky[0], zmax = kz[0];
  for (int i = 0; i < n; ++i) {
    xmin = std::min(xmin, kx[i]);
    ymin = std::min(ymin, ky[i]);
    zmin = std::min(zmin, kz[i]);
    ymax = std::max(ymax, ky[i]);
    zmax = std::max(zmax, kz[i]);
  }
  const long long ny = ymax - ymin + 1, nz = zmax - zmin + 1;
  std::vector<long long> key(n);
  for (int i = 0; i < n; ++i)
    key[i] = (kz[i] - zmin) + (long long)(ky[i] - ymin) * nz + (long long)(kx[i] - xmin) * nz * ny;
  idx.resize(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return key[a] < key[b]; });
  istrt = 0;
  for (int i = 0; i < n; ++i)
    if (kx[idx[i]] == 0 && ky[idx[i]] == 0 && kz[idx[i]] == 0) {
      istrt = i;
      break;
    }
}

// one writer over FILE* or gzFile
struct Out {
  FILE* fp = nullptr;
  gzFile gz = nullptr;
  bool ok = true;
  void text(const char* s) {
    const size_t n = strlen(s);
    if (fp) ok = ok && fwrite(s, 1, n, fp) == n;
    if (gz) ok = ok && gzwrite(gz, s, (unsigned)n) == (int)n;
  }
  void bin(const void* p, size_t n) {
    if (fp) ok = ok && fwrite(p, 1, n, fp) == n;
    if (gz) ok = ok && gzwrite(gz, p, (unsigned)n) == (int)n;
  }
  bool close() {
    if (fp) ok = (fclose(fp) == 0) && ok;
    if (gz) ok = (gzclose(gz) == Z_OK) && ok;
    return ok;
  }
};

struct In {
  FILE* fp = nullptr;
  gzFile gz = nullptr;
  bool read(void* p, size_t n) {
    if (fp) return fread(p, 1, n, fp) == n;
    return gzread(gz, p, (unsigned)n) == (int)n;
  }
  bool line(char* buf, int cap) {
    if (fp) return fgets(buf, cap, fp) != nullptr;
    return gzgets(gz, buf, cap) != nullptr;
  }
  void close() {
    if (fp) fclose(fp);
    if (gz) gzclose(gz);
  }
};

std::string file_name(const char* path, int format) {
  std::string s(path);
  if (format == CPSTEP_STATE_TEXT_GZ || format == CPSTEP_STATE_BINARY_GZ) s += ".gz";
  return s;
}

}  // namespace

extern "C" {

int cpstep_state_write(const char* path, int format, int npts, const double* coef, const int* kx,
                       const int* ky, const int* kz, int nx, int ny, int nz) {
  if (!path || !coef || !kx || !ky || !kz || npts <= 0 || format < 0 || format > 3) {
    cpstep_set_error("state_write: bad argument");
    return CPSTEP_ERR_ARG;
  }
  std::vector<int> idx;
  int istrt = 0;
  out_order(npts, kx, ky, kz, idx, istrt);
  if (!(kx[idx[istrt]] == 0 && ky[idx[istrt]] == 0 && kz[idx[istrt]] == 0)) {
    cpstep_set_error("state_write: no G=0 point");
    return CPSTEP_ERR_LAYOUT;
  }
  const int ntrue = npts - istrt;
  const std::string name = file_name(path, format);
  Out o;
  const bool text = format == CPSTEP_STATE_TEXT || format == CPSTEP_STATE_TEXT_GZ;
  if (format == CPSTEP_STATE_TEXT || format == CPSTEP_STATE_BINARY)
    o.fp = fopen(name.c_str(), text ? "w" : "wb");
  else
    o.gz = gzopen(name.c_str(), "wb");
  if (!o.fp && !o.gz) {
    cpstep_set_error("state_write: cannot open %s", name.c_str());
    return CPSTEP_ERR_ARG;
  }
  auto rec = [&](int p) {
    const double re = coef[2 * (size_t)p], im = coef[2 * (size_t)p + 1];
    if (text) {
      char b[160];
      snprintf(b, sizeof(b), "%g %g %d %d %d \n", re, im, kx[p], ky[p], kz[p]);
      o.text(b);
    } else {
      o.bin(&re, sizeof(double));
      o.bin(&im, sizeof(double));
      o.bin(&kx[p], sizeof(int));
      o.bin(&ky[p], sizeof(int));
      o.bin(&kz[p], sizeof(int));
    }
  };
  if (text) {
    char b[96];
    snprintf(b, sizeof(b), "%d %d %d %d\n", ntrue, nx, ny, nz);
    o.text(b);
  } else {
    const int h[4] = {ntrue, nx, ny, nz};
    o.bin(h, sizeof(h));
  }
  for (int i = istrt + 1; i < npts; ++i) rec(idx[i]);
  rec(idx[istrt]);
  if (!o.close()) {
    cpstep_set_error("state_write: write to %s failed", name.c_str());
    return CPSTEP_ERR_ARG;
  }
  return CPSTEP_OK;
}

int cpstep_state_read(const char* path, int format, int npts, const int* kx, const int* ky,
                      const int* kz, double* coef, int* nx, int* ny, int* nz) {
  if (!path || !coef || !kx || !ky || !kz || npts <= 0 || format < 0 || format > 3) {
    cpstep_set_error("state_read: bad argument");
    return CPSTEP_ERR_ARG;
  }
  const std::string name = file_name(path, format);
  const bool text = format == CPSTEP_STATE_TEXT || format == CPSTEP_STATE_TEXT_GZ;
  In in;
  if (format == CPSTEP_STATE_TEXT || format == CPSTEP_STATE_BINARY)
    in.fp = fopen(name.c_str(), text ? "r" : "rb");
  else
    in.gz = gzopen(name.c_str(), "rb");
  if (!in.fp && !in.gz) {
    cpstep_set_error("state_read: cannot open %s", name.c_str());
    return CPSTEP_ERR_ARG;
  }
  int h[4] = {0, 0, 0, 0};
  char buf[1000];  // the reference's line buffer size
  bool ok;
  if (text) {
    ok = in.line(buf, sizeof(buf)) && sscanf(buf, "%d%d%d%d", &h[0], &h[1], &h[2], &h[3]) == 4;
  } else {
    ok = in.read(h, sizeof(h));
  }
  if (!ok || h[0] <= 0) {
    in.close();
    cpstep_set_error("state_read: cannot parse the size line of %s", name.c_str());
    return CPSTEP_ERR_LAYOUT;
  }
  std::unordered_map<long long, Rec> recs;
  recs.reserve((size_t)h[0] * 2);
  bool g0 = false;
  for (int p = 0; p < h[0] && !g0; ++p) {
    Rec r;
    if (text) {
      ok = in.line(buf, sizeof(buf)) &&
           sscanf(buf, "%lg%lg%d%d%d", &r.re, &r.im, &r.x, &r.y, &r.z) == 5;
    } else {
      ok = in.read(&r.re, 8) && in.read(&r.im, 8) && in.read(&r.x, 4) && in.read(&r.y, 4) &&
           in.read(&r.z, 4);
    }
    if (!ok) {
      in.close();
      cpstep_set_error("state_read: cannot parse record %d of %s", p, name.c_str());
      return CPSTEP_ERR_LAYOUT;
    }
    recs[key3(r.x, r.y, r.z)] = r;
    g0 = r.x == 0 && r.y == 0 && r.z == 0;  // double pack: G=0 closes the list
  }
  in.close();
  for (int p = 0; p < npts; ++p) {
    const bool red = redundant(kx[p], ky[p], kz[p]);
    const auto it = red ? recs.find(key3(-kx[p], -ky[p], -kz[p]))
                        : recs.find(key3(kx[p], ky[p], kz[p]));
    if (it == recs.end()) {
      cpstep_set_error("state_read: point (%d,%d,%d) of the layout not in %s", kx[p], ky[p],
                       kz[p], name.c_str());
      return CPSTEP_ERR_LAYOUT;
    }
    coef[2 * (size_t)p] = it->second.re;
    coef[2 * (size_t)p + 1] = red ? -it->second.im : it->second.im;
  }
  if (nx) *nx = h[1];
  if (ny) *ny = h[2];
  if (nz) *nz = h[3];
  return CPSTEP_OK;
}

}  // extern "C"
