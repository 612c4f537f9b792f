/*
 * Stand-in for the FFTW3 double-precision API subset used by LinQT
 * (include/fftw_wrapper.hpp:16-174).  Conventions follow the public FFTW3 manual:
 * a complex DFT of size n computes out[k] = sum_j in[j] * exp(sign * 2*pi*i*j*k/n),
 * unnormalised, with FFTW_FORWARD = -1 and FFTW_BACKWARD = +1; FFTW_REDFT01 is the
 * DCT-III out[k] = in[0] + 2*sum_{j>=1} in[j]*cos(pi*j*(k+1/2)/n).
 * The transforms are implemented in fftw_standin.cpp (iterative radix-2 for powers
 * of two, direct O(n^2) sums otherwise).  Test infrastructure only.
 */
#ifndef LINQT_ORACLE_FFTW3_STANDIN_H
#define LINQT_ORACLE_FFTW3_STANDIN_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef enum {
  FFTW_R2HC = 0,
  FFTW_HC2R = 1,
  FFTW_DHT = 2,
  FFTW_REDFT00 = 3,
  FFTW_REDFT01 = 4,
  FFTW_REDFT10 = 5,
  FFTW_REDFT11 = 6,
  FFTW_RODFT00 = 7,
  FFTW_RODFT01 = 8,
  FFTW_RODFT10 = 9,
  FFTW_RODFT11 = 10
} fftw_r2r_kind;

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

#ifdef __cplusplus
}
#endif

#endif
