/*
 * linqt_oracle.h -- CPU restatement of LinQT's Chebyshev-moment hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA path in
 * linqt_b200/ is compared against; only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load it.  It is never the product path.
 *
 * Pinned against: the golden tables shipped with the reference
 * (the .chebmom2D and JACKSON.dat files under examples/utilities/wannier2sparse/linear_chain),
 * and against the reference's own sources compiled under oracle/_ref.
 *
 * Conventions: complex numbers are interleaved (re, im) doubles; operators are
 * square CSR matrices given the way LinQT stores them (0-based, Hermitian, only
 * entries with col >= row are used, include/sparse_matrix.hpp:52-54); states are
 * R consecutive length-N complex vectors.
 */
#ifndef LINQT_ORACLE_H
#define LINQT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lo_op lo_op;

/* Build a Hermitian operator from an upper-stored CSR (strictly lower entries
 * dropped, lower triangle = conj(upper)).  Returns NULL on invalid input. */
lo_op *lo_op_from_upper(int n, const int *rowptr, const int *col, const double *val);
void lo_op_free(lo_op *op);
int lo_op_dim(const lo_op *op);
long lo_op_nnz(const lo_op *op); /* Hermitian-expanded non-zeros */
/* op <- scale*op + shift*I  (src/mkl_sparse_matrix.cpp:73-97) */
void lo_op_rescale(lo_op *op, double scale, double shift);
/* y <- a*op*x + b*y for one vector  (src/mkl_sparse_matrix.cpp:56-60) */
void lo_op_mv(const lo_op *op, const double *a, const double *x, const double *b, double *y);
/* Export the expanded CSR (arrays sized n+1, nnz, 2*nnz) */
void lo_op_export(const lo_op *op, int *rowptr, int *col, double *val);

/* mu[2*M] = chebyshev::SpectralMoments (src/chebyshev_solver.cpp:176-199); op==NULL is the identity */
int lo_moments1d(const lo_op *H, const lo_op *op, const double *states, int R, int M, double *mu);
int lo_moments_td(const lo_op *H, const lo_op *opl, const lo_op *opr, const double *states, int R, int M, int NT,
                  double dt, double band_width, double band_center, double *mu_out);
int lo_time_correlation(const double *mu, int M, int NT, int N, double band_width, double band_center, double dt,
                        double broad_meV, double energy, double *t_out, double *c_out);

/* mu[2*M*M] = chebyshev::CorrelationExpansionMoments with BATCH_SIZE = M
 * (src/chebyshev_solver.cpp:45-82, 86-172), row-major mu(mL, mR) */
int lo_moments2d(const lo_op *H, const lo_op *opl, const lo_op *opr, const double *states, int R, int M,
                 double *mu);

/* Jackson kernel with truncation; returns the truncated moment count
 * (src/chebyshev_moments1D.cpp:68-87) */
int lo_jackson1d(double *mu, int M, double band_width, double broad_meV);
/* 2D variant, compacts mu to M0'xM1' row-major (src/chebyshev_moments2D.cpp:87-117) */
int lo_jackson2d(double *mu, int M0, int M1, double band_width, double b0, double b1, int *M0out, int *M1out);

/* DOS on the Chebyshev grid E_i = cos(pi(i+1/2)/M)  (src/spectralFunctionFromChebmom_FFTgrid.cpp:35-75).
 * E[M] (physical energies), dos[M] = |N/a sum_m delta(E_i,m) Re mu_m| */
/* chebyshev::SpectralMoments_nonOrth (src/chebyshev_solver.cpp:203-229): 1D moments in a
 * non-orthogonal basis, S^-1 applied by BiCGSTAB (tolerance tol, at most maxit iterations,
 * Jacobi preconditioner, x0 = 0) on the stored CSR of S (no Hermitian expansion).  op = NULL
 * is the identity.  *iters: the BiCGSTAB iterations summed over all solves. */
int lo_moments1d_nonorth(const lo_op *H, const lo_op *op, const int *s_rowptr, const int *s_col, const double *s_val,
                         const double *states, int R, int M, double tol, int maxit, double *mu_out, long *iters);
int lo_dos_fftgrid(const double *mu, int M, int N, double band_width, double band_center, double *E, double *dos);
/* spectralFunctionFromChebmom (grid 0: num_div uniform points in [-1, 1], raw sums) and
 * spectralFunctionFromChebmom_FFTgrid (grid 1: cos(pi (i+1/2)/num_div), absolute values)
 * on Jackson-damped moments mu[M]: E[num_div], out[num_div]. */
int lo_spectral_function(const double *mu, int M, int N, double band_width, double band_center, int grid,
                         int num_div, double *E, double *out);

/* Kubo-Bastin sigma(E) from a Jackson-damped 2D table (src/kuboBastinFromChebmom.cpp:35-81).
 * num_div energies in [-xbound, xbound]; writes num_div-1 points E[i], sigma[i]. */
int lo_kubo_from_moments(int variant, int grid, const double *mu, int M0, int M1, int N, double band_width,
                         double band_center, double xbound, int num_div, double *E, double *out);
int lo_bastin_from_moments(const double *mu, int M0, int M1, int N, double band_width, double band_center,
                           double xbound, int num_div, double *E, double *sigma);

/* Kubo_solver_FFT::compute with one section (src/Kubo_solver_FFT.cpp:12-136,
 * src/Bastin_FFTs.cpp:6-173, src/Greenwood_FFTs.cpp:6-91,
 * src/Kubo_solver_FFT_postProcess.cpp:8-397).  formula 0 = Greenwood, 1 = Bastin.
 * Outputs, each of length nump and in ascending energy: E (a*E-b as the reference
 * prints it), sigma, integrand (Bastin only; may be NULL).  final_data (may be NULL)
 * receives the 2*nump complex averages r_data that the post-processing consumes. */
int lo_kubo_fft(const lo_op *H, const lo_op *opl, const lo_op *opr, const double *states, int R, int M, int nump,
                int formula, int N, double band_width, double band_center, double *E, double *sigma,
                double *integrand, double *final_data);

#ifdef __cplusplus
}
#endif

#endif
