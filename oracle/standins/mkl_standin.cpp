// Implementation of the oneMKL stand-in declared in mkl.h / mkl_spblas.h.
// Test infrastructure only: it lets the reference's own sources
// (src/mkl_sparse_matrix.cpp, src/mkl_linear_algebra.cpp) build and run as the
// oracle.  Semantics follow the public oneMKL reference:
//   mkl_sparse_z_mv   y = alpha*op(A)*x + beta*y, A interpreted through matrix_descr
//   mkl_sparse_z_add  C = alpha*op(A) + B
//   cblas_zdotc_sub   sum_i conj(x_i)*y_i
#include <complex>
#define MKL_Complex16 std::complex<double>
#include "mkl.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

typedef std::complex<double> cplx;

struct sparse_matrix {
  int rows = 0, cols = 0;
  std::vector<int> rowptr, col;  // CSR, 0-based, as stored by the caller
  std::vector<cplx> val;
  // Hermitian-upper expansion, built lazily at the first Hermitian mv/mm
  bool herm_ready = false;
  std::vector<int> hrowptr, hcol;
  std::vector<cplx> hval;
};

static void build_hermitian_upper(sparse_matrix *A) {
  if (A->herm_ready) return;
  const int n = A->rows;
  std::vector<int> count(n, 0);
  for (int i = 0; i < n; i++)
    for (int k = A->rowptr[i]; k < A->rowptr[i + 1]; k++) {
      const int j = A->col[k];
      if (j < i) continue;  // strictly lower entries are ignored
      count[i]++;
      if (j != i) count[j]++;
    }
  A->hrowptr.assign(n + 1, 0);
  for (int i = 0; i < n; i++) A->hrowptr[i + 1] = A->hrowptr[i] + count[i];
  A->hcol.resize(A->hrowptr[n]);
  A->hval.resize(A->hrowptr[n]);
  std::vector<int> fill(A->hrowptr.begin(), A->hrowptr.end() - 1);
  for (int i = 0; i < n; i++)
    for (int k = A->rowptr[i]; k < A->rowptr[i + 1]; k++) {
      const int j = A->col[k];
      if (j < i) continue;
      A->hcol[fill[i]] = j;
      A->hval[fill[i]++] = A->val[k];
      if (j != i) {
        A->hcol[fill[j]] = i;
        A->hval[fill[j]++] = std::conj(A->val[k]);
      }
    }
  A->herm_ready = true;
}

static void invalidate(sparse_matrix *A) {
  A->herm_ready = false;
  A->hrowptr.clear();
  A->hcol.clear();
  A->hval.clear();
}

extern "C" {

int mkl_get_max_threads(void) { return omp_get_max_threads(); }

void cblas_zscal(MKL_INT n, const void *a, void *x, MKL_INT incx) {
  const cplx s = *static_cast<const cplx *>(a);
  cplx *v = static_cast<cplx *>(x);
#pragma omp parallel for schedule(static)
  for (MKL_INT i = 0; i < n; i++) v[(long)i * incx] *= s;
}

void cblas_zaxpy(MKL_INT n, const void *a, const void *x, MKL_INT incx, void *y, MKL_INT incy) {
  const cplx s = *static_cast<const cplx *>(a);
  const cplx *vx = static_cast<const cplx *>(x);
  cplx *vy = static_cast<cplx *>(y);
#pragma omp parallel for schedule(static)
  for (MKL_INT i = 0; i < n; i++) vy[(long)i * incy] += s * vx[(long)i * incx];
}

void cblas_zcopy(MKL_INT n, const void *x, MKL_INT incx, void *y, MKL_INT incy) {
  const cplx *vx = static_cast<const cplx *>(x);
  cplx *vy = static_cast<cplx *>(y);
#pragma omp parallel for schedule(static)
  for (MKL_INT i = 0; i < n; i++) vy[(long)i * incy] = vx[(long)i * incx];
}

void cblas_zdotc_sub(MKL_INT n, const void *x, MKL_INT incx, const void *y, MKL_INT incy, void *dotc) {
  const cplx *vx = static_cast<const cplx *>(x);
  const cplx *vy = static_cast<const cplx *>(y);
  double re = 0.0, im = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : re, im)
  for (MKL_INT i = 0; i < n; i++) {
    const cplx t = std::conj(vx[(long)i * incx]) * vy[(long)i * incy];
    re += t.real();
    im += t.imag();
  }
  *static_cast<cplx *>(dotc) = cplx(re, im);
}

double cblas_dznrm2(MKL_INT n, const void *x, MKL_INT incx) {
  const cplx *vx = static_cast<const cplx *>(x);
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (MKL_INT i = 0; i < n; i++) s += std::norm(vx[(long)i * incx]);
  return std::sqrt(s);
}

void cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb, MKL_INT m, MKL_INT n,
                 MKL_INT k, const void *alpha, const void *a, MKL_INT lda, const void *b, MKL_INT ldb,
                 const void *beta, void *c, MKL_INT ldc) {
  const cplx al = *static_cast<const cplx *>(alpha), be = *static_cast<const cplx *>(beta);
  const cplx *A = static_cast<const cplx *>(a), *B = static_cast<const cplx *>(b);
  cplx *C = static_cast<cplx *>(c);
  // element accessors for op(A)(i,l) and op(B)(l,j) in either storage order
  auto elemA = [&](long i, long l) {
    cplx v;
    if (transa == CblasNoTrans)
      v = (layout == CblasRowMajor) ? A[i * lda + l] : A[l * lda + i];
    else
      v = (layout == CblasRowMajor) ? A[l * lda + i] : A[i * lda + l];
    return transa == CblasConjTrans ? std::conj(v) : v;
  };
  auto elemB = [&](long l, long j) {
    cplx v;
    if (transb == CblasNoTrans)
      v = (layout == CblasRowMajor) ? B[l * ldb + j] : B[j * ldb + l];
    else
      v = (layout == CblasRowMajor) ? B[j * ldb + l] : B[l * ldb + j];
    return transb == CblasConjTrans ? std::conj(v) : v;
  };
#pragma omp parallel for collapse(2) schedule(static)
  for (MKL_INT i = 0; i < m; i++)
    for (MKL_INT j = 0; j < n; j++) {
      cplx acc = 0.0;
      for (MKL_INT l = 0; l < k; l++) acc += elemA(i, l) * elemB(l, j);
      cplx &out = (layout == CblasRowMajor) ? C[(long)i * ldc + j] : C[(long)j * ldc + i];
      out = al * acc + be * out;
    }
}

sparse_status_t mkl_sparse_z_create_csr(sparse_matrix_t *A, sparse_index_base_t indexing, MKL_INT rows,
                                        MKL_INT cols, MKL_INT *rows_start, MKL_INT *rows_end,
                                        MKL_INT *col_indx, MKL_Complex16 *values) {
  if (!A || rows < 0 || cols < 0) return SPARSE_STATUS_INVALID_VALUE;
  const int base = (indexing == SPARSE_INDEX_BASE_ONE) ? 1 : 0;
  sparse_matrix *M = new sparse_matrix;
  M->rows = rows;
  M->cols = cols;
  M->rowptr.resize(rows + 1, 0);
  for (int i = 0; i < rows; i++) {
    const int b = rows_start[i] - base, e = rows_end[i] - base;
    for (int k = b; k < e; k++) {
      M->col.push_back(col_indx[k] - base);
      M->val.push_back(values[k]);
    }
    M->rowptr[i + 1] = (int)M->col.size();
  }
  *A = M;
  return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_z_create_coo(sparse_matrix_t *A, sparse_index_base_t indexing, MKL_INT rows,
                                        MKL_INT cols, MKL_INT nnz, MKL_INT *row_indx, MKL_INT *col_indx,
                                        MKL_Complex16 *values) {
  if (!A || rows < 0 || cols < 0 || nnz < 0) return SPARSE_STATUS_INVALID_VALUE;
  const int base = (indexing == SPARSE_INDEX_BASE_ONE) ? 1 : 0;
  std::vector<int> order(nnz);
  for (int k = 0; k < nnz; k++) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
    return row_indx[p] != row_indx[q] ? row_indx[p] < row_indx[q] : col_indx[p] < col_indx[q];
  });
  sparse_matrix *M = new sparse_matrix;
  M->rows = rows;
  M->cols = cols;
  M->rowptr.assign(rows + 1, 0);
  for (int t = 0; t < nnz; t++) {
    const int k = order[t];
    M->col.push_back(col_indx[k] - base);
    M->val.push_back(values[k]);
    M->rowptr[row_indx[k] - base + 1]++;
  }
  for (int i = 0; i < rows; i++) M->rowptr[i + 1] += M->rowptr[i];
  *A = M;
  return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_convert_csr(const sparse_matrix_t source, sparse_operation_t operation,
                                       sparse_matrix_t *dest) {
  if (!source || !dest) return SPARSE_STATUS_INVALID_VALUE;
  if (operation != SPARSE_OPERATION_NON_TRANSPOSE) return SPARSE_STATUS_NOT_SUPPORTED;
  sparse_matrix *M = new sparse_matrix(*source);
  invalidate(M);
  *dest = M;
  return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_destroy(sparse_matrix_t A) {
  delete A;
  return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_set_mv_hint(const sparse_matrix_t A, sparse_operation_t, struct matrix_descr,
                                       MKL_INT) {
  return A ? SPARSE_STATUS_SUCCESS : SPARSE_STATUS_NOT_INITIALIZED;
}

sparse_status_t mkl_sparse_optimize(sparse_matrix_t A) {
  return A ? SPARSE_STATUS_SUCCESS : SPARSE_STATUS_NOT_INITIALIZED;
}

// y = alpha*A*x + beta*y for one vector, through the descriptor's view of A
static sparse_status_t mv_one(sparse_matrix *A, struct matrix_descr descr, cplx alpha, const cplx *x,
                              cplx beta, cplx *y) {
  const int *rp, *cl;
  const cplx *vl;
  if (descr.type == SPARSE_MATRIX_TYPE_HERMITIAN) {
    if (descr.mode != SPARSE_FILL_MODE_UPPER || descr.diag != SPARSE_DIAG_NON_UNIT)
      return SPARSE_STATUS_NOT_SUPPORTED;
    build_hermitian_upper(A);
    rp = A->hrowptr.data();
    cl = A->hcol.data();
    vl = A->hval.data();
  } else if (descr.type == SPARSE_MATRIX_TYPE_GENERAL) {
    rp = A->rowptr.data();
    cl = A->col.data();
    vl = A->val.data();
  } else {
    return SPARSE_STATUS_NOT_SUPPORTED;
  }
  const int n = A->rows;
  const bool beta_zero = (beta == cplx(0.0, 0.0));
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    cplx acc = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; k++) acc += vl[k] * x[cl[k]];
    y[i] = beta_zero ? alpha * acc : alpha * acc + beta * y[i];
  }
  return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_z_mv(sparse_operation_t operation, MKL_Complex16 alpha, const sparse_matrix_t A,
                                struct matrix_descr descr, const MKL_Complex16 *x, MKL_Complex16 beta,
                                MKL_Complex16 *y) {
  if (!A) return SPARSE_STATUS_NOT_INITIALIZED;
  if (operation != SPARSE_OPERATION_NON_TRANSPOSE) return SPARSE_STATUS_NOT_SUPPORTED;
  return mv_one(A, descr, alpha, x, beta, y);
}

sparse_status_t mkl_sparse_z_mm(sparse_operation_t operation, MKL_Complex16 alpha, const sparse_matrix_t A,
                                struct matrix_descr descr, sparse_layout_t layout, const MKL_Complex16 *B,
                                MKL_INT columns, MKL_INT ldb, MKL_Complex16 beta, MKL_Complex16 *C,
                                MKL_INT ldc) {
  if (!A) return SPARSE_STATUS_NOT_INITIALIZED;
  if (operation != SPARSE_OPERATION_NON_TRANSPOSE) return SPARSE_STATUS_NOT_SUPPORTED;
  if (layout != SPARSE_LAYOUT_COLUMN_MAJOR) return SPARSE_STATUS_NOT_SUPPORTED;
  for (MKL_INT c = 0; c < columns; c++) {
    sparse_status_t s = mv_one(A, descr, alpha, B + (long)c * ldb, beta, C + (long)c * ldc);
    if (s != SPARSE_STATUS_SUCCESS) return s;
  }
  return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_copy(const sparse_matrix_t source, struct matrix_descr, sparse_matrix_t *dest) {
  if (!source || !dest) return SPARSE_STATUS_INVALID_VALUE;
  sparse_matrix *M = new sparse_matrix(*source);
  invalidate(M);
  *dest = M;
  return SPARSE_STATUS_SUCCESS;
}

sparse_status_t mkl_sparse_z_add(sparse_operation_t operation, const sparse_matrix_t A, MKL_Complex16 alpha,
                                 const sparse_matrix_t B, sparse_matrix_t *C) {
  if (!A || !B || !C) return SPARSE_STATUS_INVALID_VALUE;
  if (operation != SPARSE_OPERATION_NON_TRANSPOSE) return SPARSE_STATUS_NOT_SUPPORTED;
  if (A->rows != B->rows || A->cols != B->cols) return SPARSE_STATUS_INVALID_VALUE;
  sparse_matrix *M = new sparse_matrix;
  M->rows = A->rows;
  M->cols = A->cols;
  M->rowptr.assign(A->rows + 1, 0);
  std::vector<std::pair<int, cplx>> row;
  for (int i = 0; i < A->rows; i++) {
    row.clear();
    for (int k = A->rowptr[i]; k < A->rowptr[i + 1]; k++) row.push_back({A->col[k], alpha * A->val[k]});
    for (int k = B->rowptr[i]; k < B->rowptr[i + 1]; k++) row.push_back({B->col[k], B->val[k]});
    std::stable_sort(row.begin(), row.end(),
                     [](const std::pair<int, cplx> &p, const std::pair<int, cplx> &q) { return p.first < q.first; });
    for (size_t t = 0; t < row.size(); t++) {
      if (t > 0 && row[t].first == row[t - 1].first) {
        M->val.back() += row[t].second;
        continue;
      }
      M->col.push_back(row[t].first);
      M->val.push_back(row[t].second);
    }
    M->rowptr[i + 1] = (int)M->col.size();
  }
  *C = M;
  return SPARSE_STATUS_SUCCESS;
}

}  // extern "C"
