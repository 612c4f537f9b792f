/*
 * Stand-in for the oneMKL "inspector-executor" sparse BLAS subset used by LinQT
 * (src/mkl_sparse_matrix.cpp:13-105).  Enumerations and signatures follow the
 * public oneMKL developer reference; behaviour is implemented in mkl_standin.cpp:
 *
 *   - handles hold a CSR copy (0-based);
 *   - mkl_sparse_z_mv / _mm honour matrix_descr: with SPARSE_MATRIX_TYPE_HERMITIAN
 *     and SPARSE_FILL_MODE_UPPER only entries with col >= row are used, the
 *     diagonal counts once, and the strictly lower triangle is conj(upper);
 *   - mkl_sparse_z_add computes C = alpha*op(A) + B as a general CSR sum.
 *
 * Test infrastructure only (see mkl.h).
 */
#ifndef LINQT_ORACLE_MKL_SPBLAS_STANDIN_H
#define LINQT_ORACLE_MKL_SPBLAS_STANDIN_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SPARSE_STATUS_SUCCESS = 0,
  SPARSE_STATUS_NOT_INITIALIZED = 1,
  SPARSE_STATUS_ALLOC_FAILED = 2,
  SPARSE_STATUS_INVALID_VALUE = 3,
  SPARSE_STATUS_EXECUTION_FAILED = 4,
  SPARSE_STATUS_INTERNAL_ERROR = 5,
  SPARSE_STATUS_NOT_SUPPORTED = 6
} sparse_status_t;

typedef enum {
  SPARSE_OPERATION_NON_TRANSPOSE = 10,
  SPARSE_OPERATION_TRANSPOSE = 11,
  SPARSE_OPERATION_CONJUGATE_TRANSPOSE = 12
} sparse_operation_t;

typedef enum {
  SPARSE_MATRIX_TYPE_GENERAL = 20,
  SPARSE_MATRIX_TYPE_SYMMETRIC = 21,
  SPARSE_MATRIX_TYPE_HERMITIAN = 22,
  SPARSE_MATRIX_TYPE_TRIANGULAR = 23,
  SPARSE_MATRIX_TYPE_DIAGONAL = 24,
  SPARSE_MATRIX_TYPE_BLOCK_TRIANGULAR = 25,
  SPARSE_MATRIX_TYPE_BLOCK_DIAGONAL = 26
} sparse_matrix_type_t;

typedef enum { SPARSE_INDEX_BASE_ZERO = 0, SPARSE_INDEX_BASE_ONE = 1 } sparse_index_base_t;

typedef enum {
  SPARSE_FILL_MODE_LOWER = 40,
  SPARSE_FILL_MODE_UPPER = 41,
  SPARSE_FILL_MODE_FULL = 42
} sparse_fill_mode_t;

typedef enum { SPARSE_DIAG_NON_UNIT = 50, SPARSE_DIAG_UNIT = 51 } sparse_diag_type_t;

typedef enum { SPARSE_LAYOUT_ROW_MAJOR = 101, SPARSE_LAYOUT_COLUMN_MAJOR = 102 } sparse_layout_t;

struct matrix_descr {
  sparse_matrix_type_t type;
  sparse_fill_mode_t mode;
  sparse_diag_type_t diag;
};

struct sparse_matrix;
typedef struct sparse_matrix *sparse_matrix_t;

sparse_status_t mkl_sparse_z_create_csr(sparse_matrix_t *A, sparse_index_base_t indexing, MKL_INT rows,
                                        MKL_INT cols, MKL_INT *rows_start, MKL_INT *rows_end,
                                        MKL_INT *col_indx, MKL_Complex16 *values);
sparse_status_t mkl_sparse_z_create_coo(sparse_matrix_t *A, sparse_index_base_t indexing, MKL_INT rows,
                                        MKL_INT cols, MKL_INT nnz, MKL_INT *row_indx, MKL_INT *col_indx,
                                        MKL_Complex16 *values);
sparse_status_t mkl_sparse_convert_csr(const sparse_matrix_t source, sparse_operation_t operation,
                                       sparse_matrix_t *dest);
sparse_status_t mkl_sparse_destroy(sparse_matrix_t A);
sparse_status_t mkl_sparse_set_mv_hint(const sparse_matrix_t A, sparse_operation_t operation,
                                       struct matrix_descr descr, MKL_INT expected_calls);
sparse_status_t mkl_sparse_optimize(sparse_matrix_t A);
sparse_status_t mkl_sparse_z_mv(sparse_operation_t operation, MKL_Complex16 alpha, const sparse_matrix_t A,
                                struct matrix_descr descr, const MKL_Complex16 *x, MKL_Complex16 beta,
                                MKL_Complex16 *y);
sparse_status_t mkl_sparse_z_mm(sparse_operation_t operation, MKL_Complex16 alpha, const sparse_matrix_t A,
                                struct matrix_descr descr, sparse_layout_t layout, const MKL_Complex16 *B,
                                MKL_INT columns, MKL_INT ldb, MKL_Complex16 beta, MKL_Complex16 *C,
                                MKL_INT ldc);
sparse_status_t mkl_sparse_copy(const sparse_matrix_t source, struct matrix_descr descr, sparse_matrix_t *dest);
sparse_status_t mkl_sparse_z_add(sparse_operation_t operation, const sparse_matrix_t A, MKL_Complex16 alpha,
                                 const sparse_matrix_t B, sparse_matrix_t *C);

#ifdef __cplusplus
}
#endif

#endif
