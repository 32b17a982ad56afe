// ORACLE TEST INFRASTRUCTURE — not product code.
//
// Project-written restatement of the Intel MKL entry points that the reference's
// BiCGSTAB solve phase and factor construction call. MKL (oneAPI; no version pinned
// anywhere in the reference, AFIIM/Makefile:12) is absent here, so the reference
// sources are compiled unmodified against this file and the headers beside it.
// Semantics follow MKL's published documentation; the arithmetic is the textbook
// definition of each routine (row-wise CSR sums in storage order, left-to-right
// dot products, sqrt of the sum of squares, unblocked LU with partial pivoting
// as in Golub & Van Loan, Alg. 3.4.1), NOT MKL's internal kernels, so results can
// differ from an MKL build in the last bits.
//
// Threading: SpMV rows and BLAS-1 loops are split into static contiguous blocks
// over OpenMP threads; reductions add the per-thread partials in thread order, so
// a run is deterministic for a fixed thread count and, with one thread, equals the
// sequential left-to-right sum that the plain-C restatement (fiim_oracle.c) uses.

#include "mkl.h"

#include <cmath>
#include <cstdlib>
#include <mutex>
#include <set>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

struct fiim_shim_sparse_matrix {
    int rows, cols, nnz;
    bool coo;
    int *rs, *re, *ci, *ri;
    double *v;
};

namespace {
std::mutex g_mu;
std::set<sparse_matrix_t> g_live;   // handles created and not yet destroyed

inline int nthreads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Static block [lo,hi) of thread t out of T for a range of n items.
inline void block_range(long n, int t, int T, long *lo, long *hi) {
    long q = n / T, r = n % T;
    *lo = t * q + std::min<long>(t, r);
    *hi = *lo + q + (t < r ? 1 : 0);
}

// Does entry (row i, col j) take part under the descriptor's fill mode?
inline bool in_triangle(const matrix_descr &d, int i, int j) {
    if (d.type == SPARSE_MATRIX_TYPE_TRIANGULAR || d.type == SPARSE_MATRIX_TYPE_SYMMETRIC) {
        if (d.mode == SPARSE_FILL_MODE_UPPER) return j >= i;
        if (d.mode == SPARSE_FILL_MODE_LOWER) return j <= i;
    }
    return true;
}
}  // namespace

extern "C" {

sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *A, sparse_index_base_t base, int rows,
                                        int cols, int *rows_start, int *rows_end, int *col_indx,
                                        double *values) {
    if (!A || base != SPARSE_INDEX_BASE_ZERO) return SPARSE_STATUS_NOT_SUPPORTED;
    auto *m = new fiim_shim_sparse_matrix{rows, cols, rows > 0 ? rows_end[rows - 1] : 0, false,
                                          rows_start, rows_end, col_indx, nullptr, values};
    std::lock_guard<std::mutex> lk(g_mu);
    g_live.insert(m);
    *A = m;
    return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_d_create_coo(sparse_matrix_t *A, sparse_index_base_t base, int rows,
                                        int cols, int nnz, int *row_indx, int *col_indx,
                                        double *values) {
    if (!A || base != SPARSE_INDEX_BASE_ZERO) return SPARSE_STATUS_NOT_SUPPORTED;
    auto *m = new fiim_shim_sparse_matrix{rows, cols, nnz, true, nullptr, nullptr, col_indx,
                                          row_indx, values};
    std::lock_guard<std::mutex> lk(g_mu);
    g_live.insert(m);
    *A = m;
    return SPARSE_STATUS_SUCCESS;
}

// Destroying a handle this shim never created is a no-op: PDFIIM/src/bicgstab.cpp:308
// destroys an uninitialised handle when A is symmetric.
sparse_status_t mkl_sparse_destroy(sparse_matrix_t A) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_live.find(A);
    if (it == g_live.end()) return SPARSE_STATUS_NOT_INITIALIZED;
    g_live.erase(it);
    delete A;
    return SPARSE_STATUS_SUCCESS;
}

// y = alpha*op(A)*x + beta*y under the descriptor: GENERAL uses every entry;
// TRIANGULAR uses the chosen triangle (UNIT diag: stored diagonal ignored, 1 used);
// SYMMETRIC uses the chosen triangle mirrored. beta == 0 overwrites y.
sparse_status_t mkl_sparse_d_mv(sparse_operation_t op, double alpha, sparse_matrix_t A,
                                struct matrix_descr d, const double *x, double beta,
                                double *y) {
    if (!A) return SPARSE_STATUS_NOT_INITIALIZED;
    const bool unit = (d.type == SPARSE_MATRIX_TYPE_TRIANGULAR && d.diag == SPARSE_DIAG_UNIT);
    const bool sym = (d.type == SPARSE_MATRIX_TYPE_SYMMETRIC);
    const int nout = (op == SPARSE_OPERATION_NON_TRANSPOSE) ? A->rows : A->cols;

    if (!A->coo && op == SPARSE_OPERATION_NON_TRANSPOSE && !sym) {
        // Row-parallel gather form: each row summed in storage order.
        const int T = nthreads();
#pragma omp parallel num_threads(T)
        {
#ifdef _OPENMP
            const int t = omp_get_thread_num();
#else
            const int t = 0;
#endif
            long lo, hi;
            block_range(A->rows, t, T, &lo, &hi);
            for (long i = lo; i < hi; ++i) {
                double s = 0.0;
                for (int k = A->rs[i]; k < A->re[i]; ++k) {
                    const int j = A->ci[k];
                    if (!in_triangle(d, (int)i, j)) continue;
                    if (unit && j == i) continue;
                    s += A->v[k] * x[j];
                }
                if (unit) s += x[i];
                y[i] = (beta == 0.0) ? alpha * s : alpha * s + beta * y[i];
            }
        }
        return SPARSE_STATUS_SUCCESS;
    }

    // Scatter forms (transpose, symmetric, COO): sequential, into a fresh accumulator.
    std::vector<double> acc(nout, 0.0);
    auto visit = [&](int i, int j, double v) {
        if (!in_triangle(d, i, j)) return;
        if (unit && i == j) return;
        if (op == SPARSE_OPERATION_NON_TRANSPOSE) {
            acc[i] += v * x[j];
            if (sym && i != j) acc[j] += v * x[i];
        } else {
            acc[j] += v * x[i];
            if (sym && i != j) acc[i] += v * x[j];
        }
    };
    if (A->coo) {
        for (int k = 0; k < A->nnz; ++k) visit(A->ri[k], A->ci[k], A->v[k]);
    } else {
        for (int i = 0; i < A->rows; ++i)
            for (int k = A->rs[i]; k < A->re[i]; ++k) visit(i, A->ci[k], A->v[k]);
    }
    if (unit)
        for (int i = 0; i < nout; ++i) acc[i] += x[i];
    for (int i = 0; i < nout; ++i) y[i] = (beta == 0.0) ? alpha * acc[i] : alpha * acc[i] + beta * y[i];
    return SPARSE_STATUS_SUCCESS;
}

// Solve op(T) y = alpha*x for triangular T stored in CSR (forward or backward substitution).
sparse_status_t mkl_sparse_d_trsv(sparse_operation_t op, double alpha, sparse_matrix_t A,
                                  struct matrix_descr d, const double *x, double *y) {
    if (!A || A->coo || op != SPARSE_OPERATION_NON_TRANSPOSE) return SPARSE_STATUS_NOT_SUPPORTED;
    const bool unit = (d.diag == SPARSE_DIAG_UNIT);
    const int n = A->rows;
    if (d.mode == SPARSE_FILL_MODE_LOWER) {
        for (int i = 0; i < n; ++i) {
            double s = alpha * x[i], dg = 1.0;
            for (int k = A->rs[i]; k < A->re[i]; ++k) {
                const int j = A->ci[k];
                if (j < i) s -= A->v[k] * y[j];
                else if (j == i && !unit) dg = A->v[k];
            }
            y[i] = s / dg;
        }
    } else {
        for (int i = n - 1; i >= 0; --i) {
            double s = alpha * x[i], dg = 1.0;
            for (int k = A->rs[i]; k < A->re[i]; ++k) {
                const int j = A->ci[k];
                if (j > i) s -= A->v[k] * y[j];
                else if (j == i && !unit) dg = A->v[k];
            }
            y[i] = s / dg;
        }
    }
    return SPARSE_STATUS_SUCCESS;
}

void cblas_dcopy(int n, const double *x, int incx, double *y, int incy) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) y[(long)i * incy] = x[(long)i * incx];
}

// y = y + a*x
void cblas_daxpy(int n, double a, const double *x, int incx, double *y, int incy) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) y[(long)i * incy] += a * x[(long)i * incx];
}

// y = a*x + b*y
void cblas_daxpby(int n, double a, const double *x, int incx, double b, double *y, int incy) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) y[(long)i * incy] = a * x[(long)i * incx] + b * y[(long)i * incy];
}

static double blocked_sum(int n, const double *x, int incx, const double *y, int incy) {
    const int T = nthreads();
    std::vector<double> part(T, 0.0);
#pragma omp parallel num_threads(T)
    {
#ifdef _OPENMP
        const int t = omp_get_thread_num();
#else
        const int t = 0;
#endif
        long lo, hi;
        block_range(n, t, T, &lo, &hi);
        double s = 0.0;
        for (long i = lo; i < hi; ++i) s += x[i * incx] * y[i * incy];
        part[t] = s;
    }
    double s = 0.0;
    for (int t = 0; t < T; ++t) s += part[t];
    return s;
}

double cblas_ddot(int n, const double *x, int incx, const double *y, int incy) {
    return blocked_sum(n, x, incx, y, incy);
}

double cblas_dnrm2(int n, const double *x, int incx) { return std::sqrt(blocked_sum(n, x, incx, x, incx)); }

void vdMul(int n, const double *a, const double *b, double *y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) y[i] = a[i] * b[i];
}

void vdSub(int n, const double *a, const double *b, double *y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) y[i] = a[i] - b[i];
}

int mkl_get_max_threads(void) { return nthreads(); }

// Row-major LU with partial pivoting, P*A = L*U (unit L below the diagonal, U on and above).
// ipiv is 1-based as in LAPACK; the pivot is the first entry of largest magnitude.
int LAPACKE_dgetrf(int layout, int m, int n, double *a, int lda, int *ipiv) {
    if (layout != LAPACK_ROW_MAJOR) return -1;
    int info = 0;
    const int kmax = std::min(m, n);
    for (int k = 0; k < kmax; ++k) {
        int p = k;
        double best = std::fabs(a[(long)k * lda + k]);
        for (int i = k + 1; i < m; ++i) {
            const double v = std::fabs(a[(long)i * lda + k]);
            if (v > best) { best = v; p = i; }
        }
        ipiv[k] = p + 1;
        if (a[(long)p * lda + k] == 0.0) {
            if (info == 0) info = k + 1;
            continue;
        }
        if (p != k)
            for (int j = 0; j < n; ++j) std::swap(a[(long)k * lda + j], a[(long)p * lda + j]);
        const double piv = a[(long)k * lda + k];
        for (int i = k + 1; i < m; ++i) {
            const double l = a[(long)i * lda + k] / piv;
            a[(long)i * lda + k] = l;
            for (int j = k + 1; j < n; ++j) a[(long)i * lda + j] -= l * a[(long)k * lda + j];
        }
    }
    return info;
}

// Solve A X = B ('N') or A^T X = B ('T') from the dgetrf factors; row-major B (n x nrhs).
int LAPACKE_dgetrs(int layout, char trans, int n, int nrhs, const double *a, int lda,
                   const int *ipiv, double *b, int ldb) {
    if (layout != LAPACK_ROW_MAJOR) return -1;
    for (int c = 0; c < nrhs; ++c) {
        auto B = [&](int i) -> double & { return b[(long)i * ldb + c]; };
        if (trans == 'N' || trans == 'n') {
            for (int k = 0; k < n; ++k)
                if (ipiv[k] - 1 != k) std::swap(B(k), B(ipiv[k] - 1));
            for (int i = 0; i < n; ++i) {          // L y = P b, unit L
                double s = B(i);
                for (int j = 0; j < i; ++j) s -= a[(long)i * lda + j] * B(j);
                B(i) = s;
            }
            for (int i = n - 1; i >= 0; --i) {     // U x = y
                double s = B(i);
                for (int j = i + 1; j < n; ++j) s -= a[(long)i * lda + j] * B(j);
                B(i) = s / a[(long)i * lda + i];
            }
        } else {
            for (int i = 0; i < n; ++i) {          // U^T z = b
                double s = B(i);
                for (int j = 0; j < i; ++j) s -= a[(long)j * lda + i] * B(j);
                B(i) = s / a[(long)i * lda + i];
            }
            for (int i = n - 1; i >= 0; --i) {     // L^T w = z, unit L
                double s = B(i);
                for (int j = i + 1; j < n; ++j) s -= a[(long)j * lda + i] * B(j);
                B(i) = s;
            }
            for (int k = n - 1; k >= 0; --k)       // x = P^T w
                if (ipiv[k] - 1 != k) std::swap(B(k), B(ipiv[k] - 1));
        }
    }
    return 0;
}

}  // extern "C"
