// C entry points around reference routines that build_ref.sh compiles from
// their own sources under the reference tree.  Test infrastructure only: the
// oracle's restatements (oracle/layout.py, oracle/ortho.py) are pinned to them.
#include <cstdlib>
#include "ckcomplex.h"
#include "para_grp_parse.h"                 // src_charm_driver/utility
#include "CP_OPERATIONS/class_cporthog.h"   // src_piny_physics_v1.0/include/class_defs

void sort_commence(int, int*, int*);  // src_mathlib/lst_sort_clean.C:97

extern "C" {

// ParaGrpParse::flip_data_set (para_grp_parse.C:178-286).  kx/ky/kz hold nktot
// points on entry and room for the flipped set; returns the new count.
int ref_flip_data_set(int nktot, int* kx, int* ky, int* kz) {
  int n_ret = 0;
  ParaGrpParse::flip_data_set(nktot, &n_ret, kx, ky, kz, nullptr, 0);
  return n_ret;
}

// ParaGrpParse::get_chareG_line_prms (para_grp_parse.C:21-170).
void ref_get_chareG_line_prms(int nktot, int nchareG, int nline, int* npts, int* istrt,
                              int* iend, int* npts_lgrp, int* nline_lgrp) {
  ParaGrpParse::get_chareG_line_prms(nktot, nchareG, nline, npts, istrt, iend, npts_lgrp,
                                     nline_lgrp, true);
}

// sort_commence (lst_sort_clean.C:97): sorts a ascending carrying b along.
void ref_sort_commence(int n, int* a, int* b) { sort_commence(n, a, b); }

// CPORTHOG::get_iter_Tmat (cp_lowdin.C:180-265): T = (S/2)^(-1/2) by Schulz.
void ref_get_iter_Tmat(const double* S, double* T, int n) { CPORTHOG::get_iter_Tmat(S, T, n); }
}
