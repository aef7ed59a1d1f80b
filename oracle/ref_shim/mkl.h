/* mkl.h -- the few Intel MKL declarations the reference's f-basis solver
 * (source/cpp/CQdiss_os_dimer) uses, so that its unmodified sources compile without MKL for the
 * oracle pin.  Test infrastructure only: built into oracle/_ref by oracle/build_ref.py and never
 * linked into the product.  Semantics follow Intel's published documentation of these routines
 * (CSR "3-array variation", one-based indexing); the implementations are in mkl_shim.cpp. */
#pragma once

typedef struct {
    double real, imag;
} MKL_Complex16;

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

#ifdef __cplusplus
extern "C" {
#endif
/* y = op(A) x, A m x m real CSR (one-based ia, ja); op = A for 'N'/'n', A^T for 'T'/'t'/'C'/'c'. */
void mkl_dcsrgemv(const char *transa, const int *m, const double *a, const int *ia, const int *ja, const double *x,
                  double *y);
/* C = A + beta op(B), m x n complex CSR, one-based.  request 1: row pointers ic only; 2: jc and c
 * for the ic of a request-1 call; 0: everything, within nzmax entries. */
void mkl_zcsradd(const char *trans, const int *request, const int *sort, const int *m, const int *n,
                 MKL_Complex16 *a, int *ja, int *ia, MKL_Complex16 *beta, MKL_Complex16 *b, int *jb, int *ib,
                 MKL_Complex16 *c, int *jc, int *ic, const int *nzmax, int *info);
/* C = op(A) B, op(A) m x n (A m x n for 'N', n x m for 'T'/'C'), B n x k, complex CSR, one-based;
 * request as for mkl_zcsradd. */
void mkl_zcsrmultcsr(const char *trans, const int *request, const int *sort, const int *m, const int *n,
                     const int *k, MKL_Complex16 *a, int *ja, int *ia, MKL_Complex16 *b, int *jb, int *ib,
                     MKL_Complex16 *c, int *jc, int *ic, const int *nzmax, int *info);
/* Eigenvalues of the Floquet tasks only (not part of the pinned path): not available here. */
lapack_int LAPACKE_zgeev(int matrix_layout, char jobvl, char jobvr, lapack_int n, MKL_Complex16 *a, lapack_int lda,
                         MKL_Complex16 *w, MKL_Complex16 *vl, lapack_int ldvl, MKL_Complex16 *vr, lapack_int ldvr);
#ifdef __cplusplus
}
#endif
