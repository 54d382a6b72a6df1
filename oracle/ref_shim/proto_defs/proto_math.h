/* Declarations of the math routines the compiled reference leaves call.  The
 * definitions (a plain column-major DGEMM for GENMATMUL, an error stub for the
 * EISPACK eigensolver RS, cputime) are in oracle/ref_mathlib.c.  Test
 * infrastructure only. */
#pragma once
#define GENMATMUL genmatmul_
#define RS rs_
extern "C" {
void genmatmul_(double* X, int* ldx, int* ityp_x, double* Y, int* ldy, int* ityp_y, double* Z,
                int* ldz, int* nrz, int* ncz, int* nxy, double* alpha, double* beta);
void rs_(int* nm, int* n, double* a, double* w, int* matz, double* z, double* fv1, double* fv2,
         int* ierr);
void cputime(double* t);
}
