/*
 * Stand-in for the subset of Intel oneMKL's C interface that LinQT's hot path
 * calls (CBLAS level 1/3 on complex<double>, mkl_get_max_threads).  Written from
 * the public oneMKL developer reference; the implementation is ours and lives in
 * mkl_standin.cpp.  Test infrastructure only: it exists so that the reference's
 * own sources can be compiled unmodified into the oracle under oracle/_ref.
 *
 * The reference defines MKL_Complex16 as std::complex<double> before including
 * this header (include/sparse_matrix.hpp:45, include/linear_algebra.hpp:14).
 */
#ifndef LINQT_ORACLE_MKL_STANDIN_H
#define LINQT_ORACLE_MKL_STANDIN_H

#include <stddef.h>

#ifndef MKL_Complex16
typedef struct { double real, imag; } MKL_Complex16_standin;
#define MKL_Complex16 MKL_Complex16_standin
#endif

typedef int MKL_INT;

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

int mkl_get_max_threads(void);

void   cblas_zscal(MKL_INT n, const void *a, void *x, MKL_INT incx);
void   cblas_zaxpy(MKL_INT n, const void *a, const void *x, MKL_INT incx, void *y, MKL_INT incy);
void   cblas_zcopy(MKL_INT n, const void *x, MKL_INT incx, void *y, MKL_INT incy);
void   cblas_zdotc_sub(MKL_INT n, const void *x, MKL_INT incx, const void *y, MKL_INT incy, void *dotc);
double cblas_dznrm2(MKL_INT n, const void *x, MKL_INT incx);
void   cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb,
                   MKL_INT m, MKL_INT n, MKL_INT k, const void *alpha, const void *a, MKL_INT lda,
                   const void *b, MKL_INT ldb, const void *beta, void *c, MKL_INT ldc);

#ifdef __cplusplus
}
#endif

#include "mkl_spblas.h"

#endif
