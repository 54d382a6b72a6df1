/* Stand-in for the FFTcache group of fft_slab_ctrl/fftCacheSlab.h, reduced to
 * the two member functions the oracle compiles from fftCache.C
 * (expandGSpace, packGSpace; declared there at fftCacheSlab.h:374-379 with
 * these signatures) and the Charm++ calls their bodies make.  Test
 * infrastructure only. */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "ckcomplex.h"
namespace PUP {
class er;
}
#include "RunDescriptor.h"
#ifndef CkAssert
#define CkAssert(x)                                   \
  do {                                                \
    if (!(x)) {                                       \
      fprintf(stderr, "CkAssert failed: %s\n", #x);  \
      exit(1);                                        \
    }                                                 \
  } while (0)
#endif
#ifndef CkExit
#define CkExit() exit(1)
#endif
class FFTcache {
 public:
  void expandGSpace(complex* data, complex* packedData, RunDescriptor* runs, int numRuns,
                    int numFull, int numPoints, int nfftz);
  void packGSpace(complex* data, complex* packedData, RunDescriptor* runs, int numRuns,
                  int numFull, int numPoints, int nfftz);
};
