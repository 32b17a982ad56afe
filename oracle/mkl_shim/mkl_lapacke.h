/* ORACLE TEST INFRASTRUCTURE — not product code.
 *
 * Stand-in for <mkl_lapacke.h>: the two LAPACKE routines PDFIIM's per-row
 * construction calls (PDFIIM/src/parPrec.cpp:288-290), row-major only.
 */
#ifndef FIIM_ORACLE_MKL_LAPACKE_H
#define FIIM_ORACLE_MKL_LAPACKE_H

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

#ifdef __cplusplus
extern "C" {
#endif

int LAPACKE_dgetrf(int matrix_layout, int m, int n, double *a, int lda, int *ipiv);
int LAPACKE_dgetrs(int matrix_layout, char trans, int n, int nrhs, const double *a, int lda,
                   const int *ipiv, double *b, int ldb);

#ifdef __cplusplus
}
#endif
#endif
