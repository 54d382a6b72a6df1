/* Math routines the compiled reference leaves call, written from their
 * published definitions.  Test infrastructure only.
 *
 * genmatmul_: src_mathlib/genmatmul.f:5-40 -- Z = alpha op(X) op(Y) + beta Z,
 *   column-major, op = transpose when the type flag is 0 (the routine maps
 *   ITYP 0 -> 'T', anything else -> 'N' before calling BLAS DGEMM).
 * rs_: the EISPACK symmetric eigensolver is not needed by the oracle
 *   (get_iter_Tmat never calls it); the stub reports an error.
 */
#include <stdio.h>
#include <time.h>

void genmatmul_(double* X, int* ldx, int* tx, double* Y, int* ldy, int* ty, double* Z, int* ldz,
                int* nrz, int* ncz, int* nxy, double* alpha, double* beta) {
  int m = *nrz, n = *ncz, k = *nxy;
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < m; ++i) {
      double acc = 0.0;
      for (int l = 0; l < k; ++l) {
        double x = (*tx == 0) ? X[l + (long)i * *ldx] : X[i + (long)l * *ldx];
        double y = (*ty == 0) ? Y[j + (long)l * *ldy] : Y[l + (long)j * *ldy];
        acc += x * y;
      }
      double z = Z[i + (long)j * *ldz];
      Z[i + (long)j * *ldz] = *alpha * acc + (*beta == 0.0 ? 0.0 : *beta * z);
    }
  }
}

void rs_(int* nm, int* n, double* a, double* w, int* matz, double* z, double* fv1, double* fv2,
         int* ierr) {
  (void)nm; (void)n; (void)a; (void)w; (void)matz; (void)z; (void)fv1; (void)fv2;
  fprintf(stderr, "rs_: not available in the oracle build\n");
  *ierr = 1;
}

void cputime(double* t) { *t = (double)clock() / CLOCKS_PER_SEC; }

/* DGEMV (BLAS): y = alpha op(A) x + beta y, A column-major lda x n (m rows),
 * op = A for 'N', A^T for 'T'; y is not read when beta is 0. */
void DGEMV(char* trans, int* m, int* n, double* alpha, double* a, int* lda, double* x,
           int* incx, double* beta, double* y, int* incy) {
  const int t = (*trans == 'T' || *trans == 't' || *trans == 'C' || *trans == 'c');
  const int leny = t ? *n : *m, lenx = t ? *m : *n;
  for (int i = 0; i < leny; ++i) {
    double acc = 0.0;
    for (int l = 0; l < lenx; ++l) {
      const double av = t ? a[l + (long)i * *lda] : a[i + (long)l * *lda];
      acc += av * x[(long)l * *incx];
    }
    double* yi = &y[(long)i * *incy];
    *yi = *alpha * acc + (*beta == 0.0 ? 0.0 : *beta * *yi);
  }
}

/* ZGEMV: only the non-double-packed reference paths call it; the oracle
 * uses the double-packed ones. */
void ZGEMV(char* trans, int* m, int* n, void* alpha, void* a, int* lda, void* x, int* incx,
           void* beta, void* y, int* incy) {
  (void)trans; (void)m; (void)n; (void)alpha; (void)a; (void)lda; (void)x; (void)incx;
  (void)beta; (void)y; (void)incy;
  fprintf(stderr, "ZGEMV is not provided by the oracle's math shim\n");
}
