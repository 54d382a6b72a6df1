/* Stand-in for PINY's standard_include.h: the C headers and the PRINTF /
 * EXIT / memory macros the compiled reference leaves use.  Test
 * infrastructure only. */
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "charm++.h"
#define PRINTF printf
#define FFLUSH fflush
#define EXIT(N) exit(N)
