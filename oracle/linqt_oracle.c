/*
 * linqt_oracle.c -- CPU restatement of LinQT's Chebyshev-moment hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 * Each function names the reference lines it restates (paths relative to the
 * adamecius/linqt checkout).  Arithmetic is IEEE double, complex numbers are C99
 * double _Complex; summation orders are those of the reference loops where the
 * reference fixes them, otherwise natural index order.
 *
 * Parity pins: tests/test_oracle_golden.py checks this file against the golden
 * tables shipped with the reference, tests/test_oracle_vs_ref.py against the
 * reference's own sources compiled under oracle/_ref.
 */
#include "linqt_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

struct lo_op {
  int n;
  long nnz;
  int *rowptr;
  int *col;
  cplx *val;
};

/* ---------------------------------------------------------------------------
 * Operators.  LinQT hands every CSR to MKL typed SPARSE_MATRIX_TYPE_HERMITIAN /
 * SPARSE_FILL_MODE_UPPER (include/sparse_matrix.hpp:52-54): entries below the
 * diagonal are ignored, the diagonal counts once, (H)_ji = conj(H_ij).  The
 * restatement expands that to a full CSR once.
 * ------------------------------------------------------------------------- */
lo_op *lo_op_from_upper(int n, const int *rowptr, const int *col, const double *val) {
  if (n < 0 || !rowptr) return NULL;
  if (rowptr[0] != 0) return NULL;
  for (int i = 0; i < n; i++)
    if (rowptr[i + 1] < rowptr[i]) return NULL;
  int *count = calloc((size_t)n + 1, sizeof(int));
  for (int i = 0; i < n; i++)
    for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
      const int j = col[k];
      if (j < 0 || j >= n) {
        free(count);
        return NULL;
      }
      if (j < i) continue;
      count[i]++;
      if (j != i) count[j]++;
    }
  lo_op *op = calloc(1, sizeof(lo_op));
  op->n = n;
  op->rowptr = malloc(sizeof(int) * ((size_t)n + 1));
  op->rowptr[0] = 0;
  for (int i = 0; i < n; i++) op->rowptr[i + 1] = op->rowptr[i] + count[i];
  op->nnz = op->rowptr[n];
  op->col = malloc(sizeof(int) * (size_t)(op->nnz ? op->nnz : 1));
  op->val = malloc(sizeof(cplx) * (size_t)(op->nnz ? op->nnz : 1));
  int *fill = malloc(sizeof(int) * ((size_t)n + 1));
  memcpy(fill, op->rowptr, sizeof(int) * (size_t)n);
  for (int i = 0; i < n; i++)
    for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
      const int j = col[k];
      if (j < i) continue;
      const cplx v = val[2 * (long)k] + I * val[2 * (long)k + 1];
      op->col[fill[i]] = j;
      op->val[fill[i]++] = v;
      if (j != i) {
        op->col[fill[j]] = i;
        op->val[fill[j]++] = conj(v);
      }
    }
  free(fill);
  free(count);
  return op;
}

void lo_op_free(lo_op *op) {
  if (!op) return;
  free(op->rowptr);
  free(op->col);
  free(op->val);
  free(op);
}

int lo_op_dim(const lo_op *op) { return op ? op->n : -1; }
long lo_op_nnz(const lo_op *op) { return op ? op->nnz : -1; }

void lo_op_export(const lo_op *op, int *rowptr, int *col, double *val) {
  memcpy(rowptr, op->rowptr, sizeof(int) * ((size_t)op->n + 1));
  memcpy(col, op->col, sizeof(int) * (size_t)op->nnz);
  for (long k = 0; k < op->nnz; k++) {
    val[2 * k] = creal(op->val[k]);
    val[2 * k + 1] = cimag(op->val[k]);
  }
}

/* H <- scale*H + shift*I, as SparseMatrixType::Rescale does with mkl_sparse_z_add
 * (src/mkl_sparse_matrix.cpp:73-97); a missing diagonal entry is inserted. */
void lo_op_rescale(lo_op *op, double scale, double shift) {
  const int n = op->n;
  int missing = 0;
  for (int i = 0; i < n; i++) {
    int has = 0;
    for (int k = op->rowptr[i]; k < op->rowptr[i + 1]; k++) has |= (op->col[k] == i);
    missing += !has;
  }
  if (missing) {
    const long nnz = op->nnz + missing;
    int *rp = malloc(sizeof(int) * ((size_t)n + 1));
    int *cl = malloc(sizeof(int) * (size_t)nnz);
    cplx *vl = malloc(sizeof(cplx) * (size_t)nnz);
    long t = 0;
    rp[0] = 0;
    for (int i = 0; i < n; i++) {
      int has = 0;
      for (int k = op->rowptr[i]; k < op->rowptr[i + 1]; k++) has |= (op->col[k] == i);
      int placed = has;
      for (int k = op->rowptr[i]; k < op->rowptr[i + 1]; k++) {
        if (!placed && op->col[k] > i) {
          cl[t] = i;
          vl[t++] = 0.0;
          placed = 1;
        }
        cl[t] = op->col[k];
        vl[t++] = op->val[k];
      }
      if (!placed) {
        cl[t] = i;
        vl[t++] = 0.0;
      }
      rp[i + 1] = (int)t;
    }
    free(op->rowptr);
    free(op->col);
    free(op->val);
    op->rowptr = rp;
    op->col = cl;
    op->val = vl;
    op->nnz = nnz;
  }
  for (int i = 0; i < n; i++)
    for (int k = op->rowptr[i]; k < op->rowptr[i + 1]; k++) {
      op->val[k] *= scale;
      if (op->col[k] == i) op->val[k] += shift;
    }
}

/* y <- a*A*x + b*y  (mkl_sparse_z_mv as called by src/mkl_sparse_matrix.cpp:56-60) */
static void op_mv(const lo_op *A, cplx a, const cplx *x, cplx b, cplx *y) {
  const int n = A->n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    cplx acc = 0.0;
    for (int k = A->rowptr[i]; k < A->rowptr[i + 1]; k++) acc += A->val[k] * x[A->col[k]];
    y[i] = (b == 0.0) ? a * acc : a * acc + b * y[i];
  }
}

void lo_op_mv(const lo_op *op, const double *a, const double *x, const double *b, double *y) {
  op_mv(op, a[0] + I * a[1], (const cplx *)x, b[0] + I * b[1], (cplx *)y);
}

/* linalg::vdot = cblas_zdotc: sum_i conj(x_i) y_i  (src/mkl_linear_algebra.cpp:24-30) */
static cplx vdot(int n, const cplx *x, const cplx *y) {
  cplx acc = 0.0;
  for (int i = 0; i < n; i++) acc += conj(x[i]) * y[i];
  return acc;
}

/* Moments::SetInitVectors (src/chebyshev_moments.cpp:5-22 with OP, :45-59 without):
 * T0 = OP*phi (or phi), T1 = H*T0. */
static void set_init_vectors(const lo_op *H, const lo_op *op, const cplx *phi, cplx *T0, cplx *T1) {
  const int n = H->n;
  if (op)
    op_mv(op, 1.0, phi, 0.0, T0);
  else
    memcpy(T0, phi, sizeof(cplx) * (size_t)n);
  op_mv(H, 1.0, T0, 0.0, T1);
}

/* Moments::Iterate (src/chebyshev_moments.cpp:157-162): T0 <- 2*H*T1 - T0; swap. */
static void iterate(const lo_op *H, cplx **T0, cplx **T1) {
  op_mv(H, 2.0, *T1, -1.0, *T0);
  cplx *t = *T0;
  *T0 = *T1;
  *T1 = t;
}

/* chebyshev::SpectralMoments (src/chebyshev_solver.cpp:176-199) */
int lo_moments1d(const lo_op *H, const lo_op *op, const double *states, int R, int M, double *mu_out) {
  if (!H || R <= 0 || M <= 0) return -1;
  const int n = H->n;
  cplx *mu = calloc((size_t)M, sizeof(cplx));
  cplx *a = malloc(sizeof(cplx) * (size_t)n), *b = malloc(sizeof(cplx) * (size_t)n);
  for (int r = 0; r < R; r++) {
    const cplx *phi = (const cplx *)states + (long)r * n;
    cplx *T0 = a, *T1 = b;
    set_init_vectors(H, op, phi, T0, T1);
    for (int m = 0; m < M; m++) {
      double scal = 2.0 / R;
      if (m == 0) scal *= 0.5;
      mu[m] += scal * vdot(n, phi, T0);
      iterate(H, &T0, &T1);
    }
  }
  for (int m = 0; m < M; m++) {
    mu_out[2 * m] = creal(mu[m]);
    mu_out[2 * m + 1] = cimag(mu[m]);
  }
  free(a);
  free(b);
  free(mu);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Non-orthogonal basis.  linalg::orthogonalize (src/mkl_linear_algebra.cpp:100-132) solves
 * S x = b with Eigen 3.4.0's BiCGSTAB (a third-party header library the reference includes
 * from eigen-3.4.0/, not shipped with it), tolerance 1e-4, at most 2000 iterations, and the
 * default DiagonalPreconditioner; S is Eigen::Map'd over the CSR arrays exactly as the
 * operator file stores them (SparseMatrixType::rows/cols/vals, no Hermitian expansion),
 * and solve() starts from x = 0.  bicgstab() restates that published algorithm (van der
 * Vorst's BiCGSTAB with Eigen's restart when r0 and r become orthogonal):
 *   r = b - S x, r0 = r, rho = alpha = w = 1, v = p = 0, tol2 = tol^2 |b|^2
 *   while |r|^2 > tol2 and i < maxit:
 *     rho_old = rho; rho = <r0, r>
 *     if |rho| < eps^2 |r0|^2: r = b - S x; r0 = r; rho = |r0|^2 = |r|^2; restart i once
 *     beta = (rho / rho_old) (alpha / w); p = r + beta (p - w v)
 *     y = D^-1 p; v = S y; alpha = rho / <r0, v>; s = r - alpha v
 *     z = D^-1 s; t = S z; w = <t, s> / |t|^2 (0 if |t| = 0)
 *     x += alpha y + w z; r = s - w t; i++
 * with <a, b> = sum conj(a_i) b_i, eps = DBL_EPSILON and D the diagonal of S (1 where a
 * row has no diagonal entry or a zero one).  |b| = 0 gives x = 0.
 * ------------------------------------------------------------------------- */
typedef struct {
  int n;
  const int *rp, *ci;
  const cplx *v;
  cplx *invd;
} gcsr;

static void gcsr_mv(const gcsr *S, const cplx *x, cplx *y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S->n; i++) {
    cplx acc = 0.0;
    for (int k = S->rp[i]; k < S->rp[i + 1]; k++) acc += S->v[k] * x[S->ci[k]];
    y[i] = acc;
  }
}

static double sqnorm(int n, const cplx *x) {
  double acc = 0.0;
  for (int i = 0; i < n; i++) acc += creal(x[i]) * creal(x[i]) + cimag(x[i]) * cimag(x[i]);
  return acc;
}

/* returns the iterations taken; x = S^-1 b to the tolerance */
static int bicgstab(const gcsr *S, const cplx *b, cplx *x, double tol, int maxit, cplx *work) {
  const int n = S->n;
  cplx *r = work, *r0 = work + n, *p = work + 2 * (size_t)n, *v = work + 3 * (size_t)n, *y = work + 4 * (size_t)n,
       *sv = work + 5 * (size_t)n, *z = work + 6 * (size_t)n, *t = work + 7 * (size_t)n;
  for (int i = 0; i < n; i++) x[i] = 0.0;
  for (int i = 0; i < n; i++) r[i] = b[i];  /* b - S*0 */
  memcpy(r0, r, sizeof(cplx) * (size_t)n);
  double r0_sq = sqnorm(n, r0);
  const double rhs_sq = sqnorm(n, b);
  if (rhs_sq == 0.0) return 0;
  cplx rho = 1.0, alpha = 1.0, w = 1.0;
  for (int i = 0; i < n; i++) v[i] = p[i] = 0.0;
  const double tol2 = tol * tol * rhs_sq, eps = 2.220446049250313e-16, eps2 = eps * eps;
  int it = 0, restarts = 0;
  while (sqnorm(n, r) > tol2 && it < maxit) {
    const cplx rho_old = rho;
    rho = vdot(n, r0, r);
    if (cabs(rho) < eps2 * r0_sq) {
      gcsr_mv(S, x, t);
      for (int i = 0; i < n; i++) r[i] = b[i] - t[i];
      memcpy(r0, r, sizeof(cplx) * (size_t)n);
      rho = r0_sq = sqnorm(n, r);
      if (restarts++ == 0) it = 0;
    }
    const cplx beta = (rho / rho_old) * (alpha / w);
    for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - w * v[i]);
    for (int i = 0; i < n; i++) y[i] = S->invd[i] * p[i];
    gcsr_mv(S, y, v);
    alpha = rho / vdot(n, r0, v);
    for (int i = 0; i < n; i++) sv[i] = r[i] - alpha * v[i];
    for (int i = 0; i < n; i++) z[i] = S->invd[i] * sv[i];
    gcsr_mv(S, z, t);
    const double tt = sqnorm(n, t);
    w = tt > 0.0 ? vdot(n, t, sv) / tt : 0.0;
    for (int i = 0; i < n; i++) x[i] += alpha * y[i] + w * z[i];
    for (int i = 0; i < n; i++) r[i] = sv[i] - w * t[i];
    ++it;
  }
  return it;
}

/* chebyshev::SpectralMoments_nonOrth (src/chebyshev_solver.cpp:203-229) with
 * Moments1D_nonOrth::SetInitVectors_nonOrthogonal (src/chebyshev_moments.cpp:63-124) and
 * Iterate_nonOrthogonal (:129-153):
 *   identity OP: T_0 = S^-1 phi,            T_1 = S^-1 H T_0
 *   with OP:     T_0 = OP S^-1 phi,         T_1 = S^-1 H T_0
 *   T_{m+1} = 2 S^-1 H T_m - T_{m-1};  mu_m += (2/R)(1/2)^{[m=0]} <phi|T_m>.
 * S: the stored CSR (s_rowptr, s_col, s_val of n rows).  The reference iterates after every
 * moment, so its last two solves (T_M and T_{M+1}) never reach mu; they are skipped here
 * (M solves per state instead of M + 2).  *iters: the BiCGSTAB iterations summed over all
 * solves. */
int lo_moments1d_nonorth(const lo_op *H, const lo_op *op, const int *s_rowptr, const int *s_col, const double *s_val,
                         const double *states, int R, int M, double tol, int maxit, double *mu_out, long *iters) {
  if (!H || R <= 0 || M <= 0) return -1;
  const int n = H->n;
  gcsr S = {n, s_rowptr, s_col, (const cplx *)s_val, malloc(sizeof(cplx) * (size_t)n)};
  for (int i = 0; i < n; i++) {
    S.invd[i] = 1.0;
    for (int k = s_rowptr[i]; k < s_rowptr[i + 1]; k++)
      if (s_col[k] == i) {
        if (S.v[k] != 0.0) S.invd[i] = 1.0 / S.v[k];
        break;
      }
  }
  cplx *mu = calloc((size_t)M, sizeof(cplx));
  cplx *T0 = malloc(sizeof(cplx) * (size_t)n), *T1 = malloc(sizeof(cplx) * (size_t)n);
  cplx *tmp = malloc(sizeof(cplx) * (size_t)n), *tmp2 = malloc(sizeof(cplx) * (size_t)n);
  cplx *work = malloc(sizeof(cplx) * 8 * (size_t)n);
  long its = 0;
  for (int r = 0; r < R; r++) {
    const cplx *phi = (const cplx *)states + (long)r * n;
    if (op) {
      its += bicgstab(&S, phi, tmp, tol, maxit, work);
      op_mv(op, 1.0, tmp, 0.0, T0);
    } else {
      its += bicgstab(&S, phi, T0, tol, maxit, work);
    }
    if (M > 1) {
      op_mv(H, 1.0, T0, 0.0, tmp);
      its += bicgstab(&S, tmp, T1, tol, maxit, work);
    }
    for (int m = 0; m < M; m++) {
      double scal = 2.0 / R;
      if (m == 0) scal *= 0.5;
      mu[m] += scal * vdot(n, phi, T0);
      if (m + 1 == M) break;
      if (m + 2 < M) {  /* T_{m+2} = 2 S^-1 H T_{m+1} - T_m, over T_m */
        op_mv(H, 1.0, T1, 0.0, tmp);
        its += bicgstab(&S, tmp, tmp2, tol, maxit, work);
        for (int i = 0; i < n; i++) T0[i] = 2.0 * tmp2[i] - T0[i];
      }
      cplx *t = T0;
      T0 = T1;
      T1 = t;
    }
  }
  for (int m = 0; m < M; m++) {
    mu_out[2 * m] = creal(mu[m]);
    mu_out[2 * m + 1] = cimag(mu[m]);
  }
  if (iters) *iters = its;
  free(work);
  free(tmp2);
  free(tmp);
  free(T1);
  free(T0);
  free(mu);
  free(S.invd);
  return 0;
}

/* chebyshev::besselJ (src/special_functions.cpp:3-17): libm's j0 / j1 / jn. */
static double bessel_j(int n, double x) { return n == 0 ? j0(x) : n == 1 ? j1(x) : jn(n, x); }

/* MomentsTD::Evolve (src/chebyshev_momentsTD.cpp:4-46): Phi <- exp(-i w0 dt) *
 * sum_n c_n (-i)^n J_n(x) T_n(H) Phi, x = dt * w, c_0 = 1, c_n = 2; the series stops before
 * the first n whose |J_n(x)| <= 1e-10.  T0/T1 are scratch. */
static void evolve(const lo_op *H, cplx *phi, cplx *T0, cplx *T1, double x, cplx exp0) {
  const int n = H->n;
  const double tol = 1e-10;
  memcpy(T0, phi, sizeof(cplx) * (size_t)n);
  op_mv(H, 1.0, T0, 0.0, T1);
  int k = 0;
  cplx nIp = 1.0;
  double Jn = 0.5 * bessel_j(k, x);
  double cut = 2.0 * tol;
  memset(phi, 0, sizeof(cplx) * (size_t)n);
  while (cut > tol) {
    const cplx c = nIp * 2.0 * Jn;
    for (int i = 0; i < n; i++) phi[i] += c * T0[i];
    op_mv(H, 2.0, T1, -1.0, T0);
    cplx *t = T0;
    T0 = T1;
    T1 = t;
    nIp *= -I;
    k++;
    Jn = bessel_j(k, x);
    cut = fabs(Jn);
  }
  for (int i = 0; i < n; i++) phi[i] *= exp0;
}

/* chebyshev::TimeDependentCorrelations (src/chebyshev_solver.cpp:231-275): per state,
 * PhiL = OPL Phi, PhiR = Phi; for each time step n: mu(m, n) += (2/R)(1/2)^[m=0]
 * <PhiL|T_m(H) OPR PhiR>, then both vectors evolve by dt.  mu_out: M x NT complex,
 * row-major (MomentsTD::operator(), include/chebyshev_moments.hpp:346-351).
 * w = (band_width / 2) / hbar, w0 = band_center / hbar (ChebyshevFreq / ChebyshevFreq_0,
 * include/chebyshev_moments.hpp:290-326, hbar = 0.6582119624 eV fs). */
int lo_moments_td(const lo_op *H, const lo_op *opl, const lo_op *opr, const double *states, int R, int M, int NT,
                  double dt, double band_width, double band_center, double *mu_out) {
  if (!H || R <= 0 || M <= 0 || NT <= 0) return -1;
  const int n = H->n;
  const double hbar = 0.6582119624;
  const double x = dt * (0.5 * band_width) / hbar;
  const cplx exp0 = cexp(-I * (band_center / hbar) * dt);
  cplx *mu = calloc((size_t)M * NT, sizeof(cplx));
  cplx *pl = malloc(sizeof(cplx) * (size_t)n), *pr = malloc(sizeof(cplx) * (size_t)n);
  cplx *a = malloc(sizeof(cplx) * (size_t)n), *b = malloc(sizeof(cplx) * (size_t)n);
  for (int r = 0; r < R; r++) {
    memcpy(pr, (const cplx *)states + (long)r * n, sizeof(cplx) * (size_t)n);
    if (opl)
      op_mv(opl, 1.0, pr, 0.0, pl);
    else
      memcpy(pl, pr, sizeof(cplx) * (size_t)n);
    for (int t = 0; t < NT; t++) {
      cplx *T0 = a, *T1 = b;
      set_init_vectors(H, opr, pr, T0, T1);
      for (int m = 0; m < M; m++) {
        double scal = 2.0 / R;
        if (m == 0) scal *= 0.5;
        mu[(size_t)m * NT + t] += scal * vdot(n, pl, T0);
        iterate(H, &T0, &T1);
      }
      evolve(H, pl, a, b, x, exp0);
      evolve(H, pr, a, b, x, exp0);
    }
  }
  for (size_t q = 0; q < (size_t)M * NT; q++) {
    mu_out[2 * q] = creal(mu[q]);
    mu_out[2 * q + 1] = cimag(mu[q]);
  }
  free(a);
  free(b);
  free(pl);
  free(pr);
  free(mu);
  return 0;
}

/* timeCorrelationsFromChebmom (src/timeCorrelationsFromChebmom.cpp:17-68) with
 * MomentsTD::ApplyJacksonKernel (src/chebyshev_momentsTD.cpp:135-154): Jackson factors over
 * m < T (T = min(M, ceil(pi/eta)), eta = 2 broad/1000/bw), then
 * C(t_n) = N/halfwidth sum_m delta_chebF(x, m) Re mu(m, n), x = (energy - bc)/halfwidth. */
static double delta_chebF(double x, double m);
int lo_time_correlation(const double *mu, int M, int NT, int N, double band_width, double band_center, double dt,
                        double broad_meV, double energy, double *t_out, double *c_out) {
  if (M <= 0 || NT <= 0 || broad_meV <= 0) return -1;
  const double eta = 2.0 * broad_meV / 1000 / band_width;
  int T = (int)ceil(M_PI / eta);
  if (T > M) T = M;
  const double phi = M_PI / (double)(T + 1.0);
  const double hw = band_width / 2, x = (energy - band_center) / hw;
  for (int n = 0; n < NT; n++) {
    double out = 0.0;
    for (int m = 0; m < T; m++) {
      const double g = ((T - m + 1) * cos(phi * m) + sin(phi * m) * cos(phi) / sin(phi)) * phi / M_PI;
      out += delta_chebF(x, m) * (mu[2 * ((size_t)m * NT + n)] * g);
    }
    t_out[n] = n * dt;
    c_out[n] = out * N / hw;
  }
  return T;
}

/* Vectors::IterateAll (src/chebyshev_vectors.cpp:4-21): store T_0..T_{M-1}. */
static void iterate_all(const lo_op *H, cplx *T0, cplx *T1, cplx *store, int M) {
  const int n = H->n;
  memcpy(store, T0, sizeof(cplx) * (size_t)n);
  for (int m = 1; m < M; m++) {
    memcpy(store + (long)m * n, T1, sizeof(cplx) * (size_t)n);
    iterate(H, &T0, &T1);
  }
}

/* Vectors::Multiply (src/chebyshev_vectors.cpp:24-51): store_m <- OP*store_m. */
static void multiply_all(const lo_op *op, cplx *store, int M, int n) {
  cplx *tmp = malloc(sizeof(cplx) * (size_t)n);
  for (int m = 0; m < M; m++) {
    op_mv(op, 1.0, store + (long)m * n, 0.0, tmp);
    memcpy(store + (long)m * n, tmp, sizeof(cplx) * (size_t)n);
  }
  free(tmp);
}

/* L_m = T_m(H) OPL phi, R_m = OPR T_m(H) phi  (src/chebyshev_solver.cpp:58-75,
 * src/Kubo_solver_FFT.cpp:98-113) */
static void lr_vectors(const lo_op *H, const lo_op *opl, const lo_op *opr, const cplx *phi, int M, cplx *L,
                       cplx *Rv) {
  const int n = H->n;
  cplx *a = malloc(sizeof(cplx) * (size_t)n), *b = malloc(sizeof(cplx) * (size_t)n);
  set_init_vectors(H, opl, phi, a, b);
  iterate_all(H, a, b, L, M);
  set_init_vectors(H, NULL, phi, a, b);
  iterate_all(H, a, b, Rv, M);
  if (opr) multiply_all(opr, Rv, M, n);
  free(a);
  free(b);
}

/* chebyshev::CorrelationExpansionMoments, BATCH_SIZE = M
 * (src/chebyshev_solver.cpp:26-42 table, :45-82 per state, :143-162 scaling) */
int lo_moments2d(const lo_op *H, const lo_op *opl, const lo_op *opr, const double *states, int R, int M,
                 double *mu_out) {
  if (!H || R <= 0 || M <= 0) return -1;
  const int n = H->n;
  cplx *L = malloc(sizeof(cplx) * (size_t)M * n), *Rv = malloc(sizeof(cplx) * (size_t)M * n);
  cplx *mu = calloc((size_t)M * M, sizeof(cplx));
  if (!L || !Rv || !mu) {
    free(L);
    free(Rv);
    free(mu);
    return -2;
  }
  for (int r = 0; r < R; r++) {
    const cplx *phi = (const cplx *)states + (long)r * n;
    lr_vectors(H, opl, opr, phi, M, L, Rv);
#pragma omp parallel for collapse(2) schedule(static)
    for (int m0 = 0; m0 < M; m0++)
      for (int m1 = 0; m1 < M; m1++) mu[(long)m0 * M + m1] += vdot(n, L + (long)m0 * n, Rv + (long)m1 * n);
  }
  for (int mL = 0; mL < M; mL++)
    for (int mR = mL; mR < M; mR++) {
      double scal = 4.0 / R;
      if (mL == 0) scal *= 0.5;
      if (mR == 0) scal *= 0.5;
      const cplx tmp = scal * (mu[(long)mL * M + mR] + conj(mu[(long)mR * M + mL])) / 2.0;
      mu[(long)mL * M + mR] = tmp;
      mu[(long)mR * M + mL] = conj(tmp);
    }
  for (long t = 0; t < (long)M * M; t++) {
    mu_out[2 * t] = creal(mu[t]);
    mu_out[2 * t + 1] = cimag(mu[t]);
  }
  free(L);
  free(Rv);
  free(mu);
  return 0;
}

/* Jackson damping factor g_m for a table of Mom moments
 * (src/chebyshev_moments1D.cpp:79-86, src/chebyshev_moments2D.cpp:105-116) */
static double jackson_g(int m, int Mom) {
  const double phi = M_PI / (double)(Mom + 1.0);
  return ((Mom - m + 1) * cos(phi * m) + sin(phi * m) * cos(phi) / sin(phi)) * phi / M_PI;
}

/* Truncation M -> min(M, ceil(pi/eta)), eta = 2*b/1000/BW (src/chebyshev_moments1D.cpp:70-76) */
static int jackson_cut(int M, double band_width, double broad) {
  const double eta = 2.0 * broad / 1000 / band_width;
  int maxMom = (int)ceil(M_PI / eta);
  return maxMom > M ? M : maxMom;
}

int lo_jackson1d(double *mu, int M, double band_width, double broad_meV) {
  if (broad_meV <= 0) return -1;
  const int Mt = jackson_cut(M, band_width, broad_meV);
  for (int m = 0; m < Mt; m++) {
    const double g = jackson_g(m, Mt);
    mu[2 * m] *= g;
    mu[2 * m + 1] *= g;
  }
  return Mt;
}

int lo_jackson2d(double *mu, int M0, int M1, double band_width, double b0, double b1, int *M0out, int *M1out) {
  if (b0 <= 0 || b1 <= 0) return -1;
  const int T0 = jackson_cut(M0, band_width, b0), T1 = jackson_cut(M1, band_width, b1);
  /* Moments2D::MomentNumber keeps the top-left T0 x T1 block (src/chebyshev_moments2D.cpp:4-13) */
  for (int m0 = 0; m0 < T0; m0++)
    for (int m1 = 0; m1 < T1; m1++) {
      mu[2 * ((long)m0 * T1 + m1)] = mu[2 * ((long)m0 * M1 + m1)];
      mu[2 * ((long)m0 * T1 + m1) + 1] = mu[2 * ((long)m0 * M1 + m1) + 1];
    }
  for (int m0 = 0; m0 < T0; m0++) {
    const double g0 = jackson_g(m0, T0);
    for (int m1 = 0; m1 < T1; m1++) {
      const double g = g0 * jackson_g(m1, T1);
      mu[2 * ((long)m0 * T1 + m1)] *= g;
      mu[2 * ((long)m0 * T1 + m1) + 1] *= g;
    }
  }
  *M0out = T0;
  *M1out = T1;
  return 0;
}

/* delta_chebF and DgreenR_chebF (include/chebyshev_coefficients.hpp:9-14, 25-32) */
static double delta_chebF(double x, double m) {
  const double f0 = sqrt(1.0 - x * x);
  const double fm = cos(m * acos(x));
  return fm / f0 / M_PI;
}

static cplx DgreenR_chebF(double x, double m) {
  const double f0 = sqrt(1.0 - x * x);
  const cplx fm = cpow(x - I * f0, m) * (x + I * m * f0);
  return -I * fm / f0 / f0 / f0;
}

/* src/spectralFunctionFromChebmom_FFTgrid.cpp:35-75 */
int lo_dos_fftgrid(const double *mu, int M, int N, double band_width, double band_center, double *E,
                   double *dos) {
  const double a = band_width / 2.0;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < M; i++) {
    const double x = cos(M_PI * (i + 0.5) / M);
    double out = 0.0;
    for (int m = 0; m < M; m++) out += delta_chebF(x, m) * mu[2 * m];
    out *= N / a;
    E[i] = x * a + band_center;
    dos[i] = fabs(out);
  }
  return 0;
}

/* src/spectralFunctionFromChebmom.cpp:35-72 (grid 0: num_div points
 * -1 + i*2/(num_div-1), the value as summed; the end points divide by zero) and
 * src/spectralFunctionFromChebmom_FFTgrid.cpp:35-75 (grid 1: cos(pi (i+1/2)/num_div), its
 * absolute value).  mu: the Jackson-damped moments, M of them. */
int lo_spectral_function(const double *mu, int M, int N, double band_width, double band_center, int grid,
                         int num_div, double *E, double *out) {
  if (num_div < 2 || grid < 0 || grid > 1) return -1;
  const double a = band_width / 2.0;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < num_div; i++) {
    const double x = grid == 0 ? -1.0 + i * (2 * 1.0) / (num_div - 1) : cos(M_PI * (i + 0.5) / num_div);
    double acc = 0.0;
    for (int m = 0; m < M; m++) acc += delta_chebF(x, m) * mu[2 * m];
    acc *= N / a;
    E[i] = x * a + band_center;
    out[i] = grid == 0 ? acc : fabs(acc);
  }
  return 0;
}

/* src/kuboBastinFromChebmom.cpp:35-81 (num_div = 30*M there, xbound 0.99; the
 * golden files of the reference were written with xbound 0.9) */
int lo_bastin_from_moments(const double *mu, int M0, int M1, int N, double band_width, double band_center,
                           double xbound, int num_div, double *E, double *sigma) {
  if (num_div < 2) return -1;
  const double a = band_width / 2.0;
  double *kernel = calloc((size_t)num_div, sizeof(double));
  double *en = malloc(sizeof(double) * (size_t)num_div);
  for (int i = 0; i < num_div; i++) en[i] = -xbound + i * (2 * xbound) / (num_div - 1);
#pragma omp parallel for schedule(dynamic, 8)
  for (int i = 0; i < num_div; i++) {
    const double x = en[i];
    double k = 0.0;
    for (int m0 = 0; m0 < M0; m0++) {
      const double d = delta_chebF(x, m0);
      for (int m1 = 0; m1 < M1; m1++) {
        const cplx muv = mu[2 * ((long)m0 * M1 + m1)] + I * mu[2 * ((long)m0 * M1 + m1) + 1];
        k += d * cimag(DgreenR_chebF(x, m1) * muv);
      }
    }
    kernel[i] = k * (-2.0 * N / a / a);
  }
  double acc = 0.0;
  for (int i = 0; i < num_div - 1; i++) {
    acc += kernel[i] * (en[i + 1] - en[i]);
    E[i] = en[i] * a + band_center;
    sigma[i] = acc;
  }
  free(kernel);
  free(en);
  return 0;
}

/* greenR_chebF (include/chebyshev_coefficients.hpp:16-23) */
static cplx greenR_chebF(double x, double m) {
  const double f0 = sqrt(1.0 - x * x);
  const cplx fm = cpow(x - I * f0, m);
  return -I * fm / f0;
}

/* rearrange_crescent_order of src/kuboBastinFromChebmom_FFTgrid.cpp:18-36 */
static void lo_rearrange(double *v, int n) {
  double *o = malloc(sizeof(double) * (size_t)n);
  memcpy(o, v, sizeof(double) * (size_t)n);
  for (int k = 0; k < n / 2; k++) {
    v[2 * k] = o[k];
    v[2 * k + 1] = o[n - k - 1];
  }
  for (int k = 0; k < n / 2; k++) {
    const double t = v[k];
    v[k] = v[n - k - 1];
    v[n - k - 1] = t;
  }
  free(o);
}

/* The energy sums of LinQT's post-processors on a Jackson-damped table mu[M0][M1]:
 *   variant 0 Bastin     (src/kuboBastinFromChebmom.cpp:63-81, _FFTgrid.cpp:88-106)
 *   variant 1 Greenwood  (src/kuboGreenwoodFromChebmom.cpp:61-74, _FFTgrid.cpp:62-76)
 *   variant 2 Bastin I   (src/kuboBastinIFromChebmom.cpp:63-84)
 *   variant 3 Bastin II  (src/kuboBastinIIFromChebmom.cpp:62-88)
 *   variant 4 Bastin sea (src/kuboBastinSeaFromChebmom.cpp:62-88)
 *   variant 5 Bastin surface (src/kuboBastinSurfFromChebmom.cpp:62-82)
 * grid 0: num_div points uniform in [-xbound, xbound]; grid 1: x_i = cos(pi (2i + 1/2)/num_div);
 * grid 2: grid 1 in the rearranged (ascending) order of the Bastin FFT-grid driver.
 * Writes num_div - 1 points: E = x a + c and the driver's output column. */
int lo_kubo_from_moments(int variant, int grid, const double *mu, int M0, int M1, int N, double band_width,
                         double band_center, double xbound, int num_div, double *E, double *out) {
  if (num_div < 2 || variant < 0 || variant > 5 || grid < 0 || grid > 2) return -1;
  const double a = band_width / 2.0, w = N / a / a;
  double *kernel = calloc((size_t)num_div, sizeof(double));
  double *en = malloc(sizeof(double) * (size_t)num_div);
  for (int i = 0; i < num_div; i++)
    en[i] = grid == 0 ? -xbound + i * (2 * xbound) / (num_div - 1) : cos(M_PI * (2 * i + 0.5) / num_div);
  if (grid == 2) lo_rearrange(en, num_div);
#pragma omp parallel for schedule(dynamic, 8)
  for (int i = 0; i < num_div; i++) {
    const double x = en[i];
    double k = 0.0;
    for (int m0 = 0; m0 < M0; m0++) {
      const double d0 = delta_chebF(x, m0);
      const cplx g0 = greenR_chebF(x, m0), dg0 = DgreenR_chebF(x, m0);
      for (int m1 = 0; m1 < M1; m1++) {
        const cplx muv = mu[2 * ((long)m0 * M1 + m1)] + I * mu[2 * ((long)m0 * M1 + m1) + 1];
        switch (variant) {
          case 0: k += d0 * cimag(DgreenR_chebF(x, m1) * muv); break;
          case 1:
          case 2: k += d0 * cimag(greenR_chebF(x, m1) * muv); break;
          case 3: k += -creal((g0 * DgreenR_chebF(x, m1) - dg0 * greenR_chebF(x, m1)) * muv); break;
          case 4: {
            const double dgr = creal(DgreenR_chebF(x, m1));
            k += -creal((g0 - conj(g0)) * (dgr + dgr) * muv);
            break;
          }
          default: k += d0 * delta_chebF(x, m1) * creal(muv); break;
        }
      }
    }
    const double pref[6] = {-2.0 * w, -w, -w, w / 2 / M_PI, w / 2 / M_PI, M_PI * w};
    kernel[i] = k * pref[variant];
  }
  double acc = 0.0;
  for (int i = 0; i < num_div - 1; i++) {
    const double de = en[i + 1] - en[i];
    E[i] = en[i] * a + band_center;
    switch (variant) {
      case 0: acc += kernel[i] * de; out[i] = acc; break;
      case 1: out[i] = kernel[i]; break;
      case 2: out[i] = 0.5 * (kernel[i] + kernel[i + 1]); break;
      case 3: acc += (kernel[i] + kernel[i + 1]) * de; out[i] = acc; break;
      case 4: acc += 0.5 * (kernel[i] + kernel[i + 1]) * de; out[i] = acc; break;
      default: out[i] = (kernel[i + 1] + kernel[i]) / 2.0; break;
    }
  }
  free(kernel);
  free(en);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Kubo_solver_FFT.  The reference uses FFTW backward DFTs (exponent +1,
 * unnormalised) of length nump on zero-padded inputs; here an iterative radix-2
 * transform (nump a power of two) or a direct sum.
 * ------------------------------------------------------------------------- */
typedef struct {
  int n;
  int *bitrev;
  cplx *tw; /* exp(+2 pi i k / n) */
} dft_plan;

static void dft_init(dft_plan *p, int n) {
  p->n = n;
  p->tw = malloc(sizeof(cplx) * (size_t)n);
  for (int k = 0; k < n; k++) {
    const double ang = 2.0 * M_PI * (double)k / (double)n;
    p->tw[k] = cos(ang) + I * sin(ang);
  }
  p->bitrev = NULL;
  if ((n & (n - 1)) == 0) {
    int lg = 0;
    while ((1 << lg) < n) lg++;
    p->bitrev = malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; i++) {
      int r = 0;
      for (int b = 0; b < lg; b++)
        if (i & (1 << b)) r |= 1 << (lg - 1 - b);
      p->bitrev[i] = r;
    }
  }
}

static void dft_free(dft_plan *p) {
  free(p->tw);
  free(p->bitrev);
}

/* out[k] = sum_j in[j] exp(+2 pi i j k / n) */
static void dft_backward(const dft_plan *p, const cplx *in, cplx *out) {
  const int n = p->n;
  if (p->bitrev) {
    for (int i = 0; i < n; i++) out[p->bitrev[i]] = in[i];
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1, stride = n / len;
      for (int s = 0; s < n; s += len)
        for (int j = 0; j < half; j++) {
          const cplx t = p->tw[j * stride] * out[s + j + half];
          const cplx u = out[s + j];
          out[s + j] = u + t;
          out[s + j + half] = u - t;
        }
    }
  } else {
    for (int k = 0; k < n; k++) {
      cplx acc = 0.0;
      for (int j = 0; j < n; j++) acc += in[j] * p->tw[((long)j * k) % n];
      out[k] = acc;
    }
  }
}

/* Kubo_solver_FFT::Jackson_kernel (include/Kubo_solver_FFT.hpp:99-107) */
static double fft_jackson(int m, int M) {
  return 1 / (M + 1.0) * ((M - m + 1.0) * cos(M_PI * m / (M + 1.0)) + sin(M_PI * m / (M + 1.0)) / tan(M_PI / (M + 1.0)));
}

static double re(cplx z) { return creal(z); }

/* Bastin_FFTs per-site products (src/Bastin_FFTs.cpp:20-172) and Greenwood_FFTs
 * (src/Greenwood_FFTs.cpp:15-91), summed over sites into r_data[2*nump]. */
static void fft_sites(const cplx *L, const cplx *Rv, int n, int M, int nump, int formula, cplx *r_data) {
  cplx *pf = calloc((size_t)nump, sizeof(cplx));
  for (int m = 0; m < M; m++)
    pf[m] = (double)(2 - (m == 0)) * fft_jackson(m, M) * cexp(I * (M_PI * m / (2.0 * nump)));
#pragma omp parallel
  {
    dft_plan plan;
    dft_init(&plan, nump);
    const int nseq = formula == 1 ? 8 : 4;
    cplx *in = calloc((size_t)nseq * nump, sizeof(cplx));
    cplx *out = malloc(sizeof(cplx) * (size_t)nseq * nump);
    cplx *acc = calloc((size_t)2 * nump, sizeof(cplx));
#pragma omp for schedule(static)
    for (int l = 0; l < n; l++) {
      for (int m = 0; m < M; m++) {
        const cplx bra = L[(long)m * n + l], ket = Rv[(long)m * n + l];
        in[0 * nump + m] = pf[m] * creal(bra); /* re_bras */
        in[1 * nump + m] = pf[m] * cimag(bra); /* im_bras */
        in[2 * nump + m] = pf[m] * creal(ket); /* re_kets */
        in[3 * nump + m] = pf[m] * cimag(ket); /* im_kets */
        if (nseq == 8) {
          in[4 * nump + m] = (double)m * in[0 * nump + m]; /* re_D_bras */
          in[5 * nump + m] = (double)m * in[1 * nump + m]; /* im_D_bras */
          in[6 * nump + m] = (double)m * in[2 * nump + m]; /* re_D_kets */
          in[7 * nump + m] = (double)m * in[3 * nump + m]; /* im_D_kets */
        }
      }
      for (int s = 0; s < nseq; s++) dft_backward(&plan, in + (long)s * nump, out + (long)s * nump);
      const cplx *rb = out, *ib = out + nump, *rk = out + 2 * (long)nump, *ik = out + 3 * (long)nump;
      if (formula == 1) {
        const cplx *rDb = out + 4 * (long)nump, *iDb = out + 5 * (long)nump, *rDk = out + 6 * (long)nump,
                   *iDk = out + 7 * (long)nump;
        for (int j = 0; j < nump / 2; j++) {
          acc[j] += (re(rb[j]) - I * re(ib[j])) * (rk[j] + I * ik[j]) +
                    (conj(rb[j]) - I * conj(ib[j])) * (re(rk[j]) + I * re(ik[j]));
          acc[j + nump] += (conj(rDb[j]) - I * conj(iDb[j])) * (re(rk[j]) + I * re(ik[j])) -
                           (re(rb[j]) - I * re(ib[j])) * (rDk[j] + I * iDk[j]);
        }
        for (int j = nump / 2; j < nump; j++) {
          acc[j] += (re(rb[j]) - I * re(ib[j])) * (conj(rk[j]) + I * conj(ik[j])) +
                    (rb[j] - I * ib[j]) * (re(rk[j]) + I * re(ik[j]));
          acc[j + nump] += (rDb[j] - I * iDb[j]) * (re(rk[j]) + I * re(ik[j])) -
                           (re(rb[j]) - I * re(ib[j])) * (conj(rDk[j]) + I * conj(iDk[j]));
        }
      } else {
        for (int k = 0; k < nump; k++) acc[k] += creal((re(rb[k]) - I * re(ib[k])) * (re(rk[k]) + I * re(ik[k])));
      }
    }
#pragma omp critical
    {
      for (int k = 0; k < 2 * nump; k++) r_data[k] += acc[k];
    }
    free(in);
    free(out);
    free(acc);
    dft_free(&plan);
  }
  free(pf);
}

/* Kubo_solver_FFT_postProcess::rearrange_crescent_order (src/Kubo_solver_FFT_postProcess.cpp:98-116) */
static void rearrange(double *x, int nump) {
  double *orig = malloc(sizeof(double) * (size_t)nump);
  memcpy(orig, x, sizeof(double) * (size_t)nump);
  for (int k = 0; k < nump / 2; k++) {
    x[2 * k] = orig[k];
    x[2 * k + 1] = orig[nump - k - 1];
  }
  for (int k = 0; k < nump / 2; k++) {
    const double t = x[k];
    x[k] = x[nump - k - 1];
    x[nump - k - 1] = t;
  }
  free(orig);
}

int lo_kubo_fft(const lo_op *H, const lo_op *opl, const lo_op *opr, const double *states, int R, int M, int nump,
                int formula, int N, double band_width, double band_center, double *E_out, double *sigma,
                double *integrand_out, double *final_out) {
  if (!H || R <= 0 || M <= 0 || nump < M || (formula != 0 && formula != 1)) return -1;
  const int n = H->n;
  cplx *L = malloc(sizeof(cplx) * (size_t)M * n), *Rv = malloc(sizeof(cplx) * (size_t)M * n);
  cplx *r_data = calloc((size_t)2 * nump, sizeof(cplx)), *final_data = calloc((size_t)2 * nump, sizeof(cplx));
  if (!L || !Rv || !r_data || !final_data) {
    free(L);
    free(Rv);
    free(r_data);
    free(final_data);
    return -2;
  }
  /* Kubo_solver_FFT::compute (src/Kubo_solver_FFT.cpp:56-68): running mean over states */
  for (int r = 0; r < R; r++) {
    const cplx *phi = (const cplx *)states + (long)r * n;
    lr_vectors(H, opl, opr, phi, M, L, Rv);
    memset(r_data, 0, sizeof(cplx) * 2 * (size_t)nump);
    fft_sites(L, Rv, n, M, nump, formula, r_data);
    const int cnt = r + 1;
    for (int i = 0; i < 2 * nump; i++) final_data[i] = (final_data[i] * (double)(cnt - 1) + r_data[i]) / (double)cnt;
  }
  /* post-processing (src/Kubo_solver_FFT_postProcess.cpp:8-16, 120-273, 279-397) */
  const double a = band_width / 2.0, b = band_center;
  const double omega = N / (a * a);
  double *Ek = malloc(sizeof(double) * (size_t)nump), *Er = malloc(sizeof(double) * (size_t)nump);
  double *integ = calloc((size_t)nump, sizeof(double)), *part = calloc((size_t)nump, sizeof(double));
  for (int k = 0; k < nump; k++) Ek[k] = cos(M_PI * (2 * k + 0.5) / nump);
  memcpy(Er, Ek, sizeof(double) * (size_t)nump);
  rearrange(Er, nump);
  if (formula == 1) {
    for (int k = 0; k < nump; k++) {
      integ[k] = Ek[k] * creal(final_data[k]) - (sqrt(1.0 - Ek[k] * Ek[k]) * cimag(final_data[k + nump]));
      integ[k] *= 1.0 / pow((1.0 - Ek[k] * Ek[k]), 2.0);
      integ[k] *= omega / (M_PI);
    }
    rearrange(integ, nump);
    /* integration_linqt (:36-47): left-rectangle cumulative sum, last point stays 0 */
    double acc = 0;
    for (int i = 0; i < nump - 1; i++) {
      acc += integ[i] * (Er[i + 1] - Er[i]);
      part[i] = acc;
    }
  } else {
    for (int k = 0; k < nump; k++)
      part[k] = 2.0 * omega * creal(final_data[k]) / (1.0 - Ek[k] * Ek[k]) / (2 * M_PI);
    rearrange(part, nump);
  }
  for (int e = 0; e < nump; e++) {
    E_out[e] = a * Er[e] - b;
    sigma[e] = part[e];
    if (integrand_out) integrand_out[e] = integ[e];
  }
  if (final_out)
    for (int i = 0; i < 2 * nump; i++) {
      final_out[2 * i] = creal(final_data[i]);
      final_out[2 * i + 1] = cimag(final_data[i]);
    }
  free(Ek);
  free(Er);
  free(integ);
  free(part);
  free(L);
  free(Rv);
  free(r_data);
  free(final_data);
  return 0;
}
