/* ORACLE TEST INFRASTRUCTURE — not product code.
 *
 * Minimal stand-in for the Intel MKL sparse BLAS header, declaring only the
 * entry points the reference's solve and construction code calls:
 *   AFIIM/src/bicgstab.cpp:136-147,151-195   ACIFIM/src/bicgstab.cpp:157-224,394-426
 *   PDFIIM/src/bicgstab.cpp:143-213,306-308  {AFIIM,ACIFIM,PDFIIM}/src/misc.cpp (form_model_rhs)
 * Intel MKL itself is not vendored by the reference, its version is not pinned
 * (AFIIM/Makefile:12, ACIFIM/Makefile:16, PDFIIM/Makefile:11-12) and it is absent
 * here; mkl_shim.cpp restates the published semantics of these calls.
 * Enumerator values are this shim's own; only the names are MKL's.
 */
#ifndef FIIM_ORACLE_MKL_SPBLAS_H
#define FIIM_ORACLE_MKL_SPBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fiim_shim_sparse_matrix *sparse_matrix_t;

typedef enum { SPARSE_STATUS_SUCCESS = 0, SPARSE_STATUS_NOT_INITIALIZED = 1,
               SPARSE_STATUS_INVALID_VALUE = 3, SPARSE_STATUS_NOT_SUPPORTED = 6 } sparse_status_t;
typedef enum { SPARSE_INDEX_BASE_ZERO = 0, SPARSE_INDEX_BASE_ONE = 1 } sparse_index_base_t;
typedef enum { SPARSE_OPERATION_NON_TRANSPOSE = 10, SPARSE_OPERATION_TRANSPOSE = 11,
               SPARSE_OPERATION_CONJUGATE_TRANSPOSE = 12 } sparse_operation_t;
typedef enum { SPARSE_MATRIX_TYPE_GENERAL = 20, SPARSE_MATRIX_TYPE_SYMMETRIC = 21,
               SPARSE_MATRIX_TYPE_HERMITIAN = 22, SPARSE_MATRIX_TYPE_TRIANGULAR = 23,
               SPARSE_MATRIX_TYPE_DIAGONAL = 24 } sparse_matrix_type_t;
typedef enum { SPARSE_FILL_MODE_LOWER = 40, SPARSE_FILL_MODE_UPPER = 41,
               SPARSE_FILL_MODE_FULL = 42 } sparse_fill_mode_t;
typedef enum { SPARSE_DIAG_NON_UNIT = 50, SPARSE_DIAG_UNIT = 51 } sparse_diag_type_t;

struct matrix_descr {
    sparse_matrix_type_t type;
    sparse_fill_mode_t mode;
    sparse_diag_type_t diag;
};

sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *A, sparse_index_base_t base,
                                        int rows, int cols, int *rows_start, int *rows_end,
                                        int *col_indx, double *values);
sparse_status_t mkl_sparse_d_create_coo(sparse_matrix_t *A, sparse_index_base_t base,
                                        int rows, int cols, int nnz, int *row_indx,
                                        int *col_indx, double *values);
sparse_status_t mkl_sparse_d_mv(sparse_operation_t op, double alpha, sparse_matrix_t A,
                                struct matrix_descr descr, const double *x, double beta,
                                double *y);
sparse_status_t mkl_sparse_d_trsv(sparse_operation_t op, double alpha, sparse_matrix_t A,
                                  struct matrix_descr descr, const double *x, double *y);
sparse_status_t mkl_sparse_destroy(sparse_matrix_t A);

#ifdef __cplusplus
}
#endif
#endif
