/* Extra stand-ins for compiling the reference's EES sources
 * (cp_ees_nonlocal.C, set_cp_ewald.C) with plain g++: PUP, PE queries, the
 * PINY allocator names, CkAssert and the two Charm++ types their headers name.
 * Forced into those translation units by build_ref.sh.  Test infrastructure
 * only. */
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
namespace PUP {
class er {
 public:
  bool isUnpacking() const { return false; }
  template <class T>
  void operator()(T*, int) {}
};
}  // namespace PUP
template <class T>
inline PUP::er& operator|(PUP::er& p, T&) { return p; }
inline int CkMyPe() { return 0; }
inline int CkNumPes() { return 1; }
inline void* cmalloc(size_t n, const char*) { return malloc(n); }
inline void cfree(void* p, const char*) { free(p); }
#define PUPmarshall(x)
class CkCallback {};
#define CkAssert(x)                                                   \
  do {                                                                \
    if (!(x)) {                                                       \
      fprintf(stderr, "CkAssert failed: %s\n", #x);                  \
      exit(1);                                                        \
    }                                                                 \
  } while (0)
/* the Charm-FFT library's point record (external, not in the tree): kz, ky,
 * kx of a density-sphere point and its offset in the caller's array */
struct gridPoint {
  int d1, d2, d3;
  int offset;
};
double getdeth(double*);
