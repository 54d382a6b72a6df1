/* Minimal stand-in for the Charm++ header, so that self-contained reference
 * leaves (para_grp_parse.C) compile with plain g++ for the oracle.  Test
 * infrastructure only. */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#define CkPrintf printf
#define CkExit() exit(1)
#define CkAbort(m) do { fprintf(stderr, "%s\n", m); exit(1); } while (0)
#define CmiMemcpy memcpy
#ifndef CHARM_OFF
#define CHARM_OFF
#endif
