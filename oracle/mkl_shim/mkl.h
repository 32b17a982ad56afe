/* ORACLE TEST INFRASTRUCTURE — not product code.
 *
 * Stand-in for <mkl.h>: the CBLAS level-1 and VML routines the reference's
 * BiCGSTAB calls (AFIIM/src/bicgstab.cpp:153-271, ACIFIM/src/bicgstab.cpp:182-300,401-417,
 * PDFIIM/src/bicgstab.cpp:171-289), mkl_get_max_threads (PDFIIM/example/pdfiim.cpp:116)
 * and, through mkl_lapacke.h, the LAPACKE LU routines PDFIIM's construction calls
 * (PDFIIM/src/parPrec.cpp:288-290).
 */
#ifndef FIIM_ORACLE_MKL_H
#define FIIM_ORACLE_MKL_H

#include "mkl_spblas.h"
#include "mkl_lapacke.h"

#ifdef __cplusplus
extern "C" {
#endif

void cblas_dcopy(int n, const double *x, int incx, double *y, int incy);
void cblas_daxpy(int n, double a, const double *x, int incx, double *y, int incy);
void cblas_daxpby(int n, double a, const double *x, int incx, double b, double *y, int incy);
double cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
double cblas_dnrm2(int n, const double *x, int incx);
void vdMul(int n, const double *a, const double *b, double *y);
void vdSub(int n, const double *a, const double *b, double *y);
int mkl_get_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
