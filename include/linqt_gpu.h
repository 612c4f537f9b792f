/*
 * linqt_gpu.h -- C ABI of the B200 Chebyshev-moment engine (liblinqt_gpu.so).
 *
 * The library computes LinQT's kernel-polynomial hot path on one NVIDIA B200
 * (sm_100a): the Chebyshev recursion T_{n+1} = 2 H T_n - T_{n-1} on a rescaled
 * sparse complex Hamiltonian, the 1D moments mu_n = <r|T_n(H)|r>, the 2D
 * Kubo-Bastin moments mu_nm = <r|V T_m(H) V T_n(H)|r>, the FFT-based
 * Bastin/Greenwood reconstruction of Kubo_solver_FFT, and the energy-grid
 * reconstructions of the *FromChebmom post-processors.
 *
 * Conventions
 *   - Complex numbers are interleaved (re, im) pairs of double.
 *   - Operators are square CSR matrices, 0-based, int32 indices.  With
 *     LINQT_STORAGE_HERMITIAN_UPPER (LinQT's convention, include/sparse_matrix.hpp:52-54)
 *     only entries with col >= row are read, the diagonal counts once and the
 *     lower triangle is the conjugate of the upper one.
 *   - States are R consecutive length-N vectors (the `vector` state-file layout,
 *     include/quantum_states.hpp:155-183).
 *   - Every function returns LINQT_OK (0) or a negative LINQT_ERR_* code; the
 *     message of the last error of the calling thread is linqt_last_error().
 *     No function aborts or throws across the ABI.
 *   - Host-pointer entry points copy inputs to the device and results back and
 *     return when the results are on the host.  *_dev entry points take device
 *     pointers and enqueue work on the session's stream without synchronising.
 *   - A session (NULL = the calling thread's default session on the current
 *     device) owns a CUDA stream and a cache of device workspaces; one session
 *     must not be used by two host threads at once.
 */
#ifndef LINQT_GPU_H
#define LINQT_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LINQT_ABI_VERSION 3

enum {
  LINQT_OK = 0,
  LINQT_ERR_INVALID = -1,     /* bad argument (size, pointer, CSR structure) */
  LINQT_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  LINQT_ERR_NOMEM = -3,       /* device allocation failed or exceeds the session budget */
  LINQT_ERR_UNSUPPORTED = -4, /* option combination not implemented */
  LINQT_ERR_INTERNAL = -5,    /* unexpected internal failure */
  LINQT_ERR_TIMEOUT = -6,     /* a bounded device wait expired */
  LINQT_ERR_CANCELLED = -7    /* request cancelled (serving) */
};

enum { LINQT_STORAGE_HERMITIAN_UPPER = 0, LINQT_STORAGE_GENERAL = 1 };

enum {
  LINQT_PREC_FP64 = 0,       /* FP64 recursion, FP64 moment contraction */
  LINQT_PREC_MIXED = 1,      /* FP32 Chebyshev vectors (FP64 operators and accumulation in the recursion),
                                moment contraction on the INT8 tensor cores from 4-digit (28-bit) splits
                                of the FP32 blocks with exact INT32 accumulation, FP64 across chunks */
  LINQT_PREC_FP32 = 2,       /* FP32 vectors, FP64 MMA contraction of the FP32 blocks (diagnostic) */
  LINQT_PREC_MIXED_TF32 = 3, /* FP32 vectors, 3xTF32 tensor-core contraction with FP32 accumulation over
                                2048-float chunks (the split-precision form; its truncating FP32
                                accumulation costs about 4e-5 of max|mu|) */
  LINQT_PREC_MIXED_FAST = 4  /* as LINQT_PREC_MIXED with 3-digit (21-bit) splits: 6 instead of 10 INT8
                                products, ~1e-7 of max|mu| */
};

enum { LINQT_KUBO_GREENWOOD = 0, LINQT_KUBO_BASTIN = 1 }; /* chebyshev::formula, include/Kubo_solver_FFT.hpp:17-21 */

enum { LINQT_FORMAT_CSR = 0, LINQT_FORMAT_SELL = 1, LINQT_FORMAT_AUTO = 2, LINQT_FORMAT_LOCAL = 3 };

typedef struct linqt_op linqt_op;
typedef struct linqt_session linqt_session;

/* Solver options; zero-initialised = defaults (FP64, CSR, automatic tiling). */
typedef struct linqt_opts {
  int precision;    /* LINQT_PREC_* */
  int format;       /* sparse layout of H in the persistent recursions: LINQT_FORMAT_CSR (default),
                       LINQT_FORMAT_SELL (SELL-C-sigma, C = 32, sigma = 8C), LINQT_FORMAT_LOCAL
                       (the CSR rows copied in a locality order found by recursive bisection of the
                       operator's graph and visited in that order, see linqt_locality_order:
                       neighbour rows are read close together in time, for lattices such as 3D ones
                       whose neighbours lie far apart in the row numbering) or LINQT_FORMAT_AUTO
                       (autotuned among CSR with and without its shared-memory row cache and SELL
                       with C = 8, 32, plus the CSR rows and SELL-32 in the locality order when a
                       block exceeds 64 MB (linqt_op_tuned reports the choices), times the thread
                       shapes of the block (threads per row min(R, 32) >> s, s = 0..3), and for 1D
                       moments without a fixed block_width the block width (R, R/2, R/4, R/8);
                       cached per operator, width and precision).  The layout changes only the
                       order of the per-block dot-product sums. */
  int block_width;  /* vector columns per recursion block (0 = all R, or the autotuned chunk) */
  int doubling;     /* 1D: 0 = doubling identities when the operator is the identity, 1 = force them, 2 = direct <r|T_n r> */
  int use_graphs;   /* 1: *_dev solves replay an instantiated CUDA graph from the second call with the same
                       pointers, sizes and operators on (first call eager, second captured); workspace
                       reallocations drop the session's graphs; not for sessions on the legacy stream */
  int step_launches; /* 1 = one kernel launch per recursion step instead of one persistent cooperative launch */
  int realisations; /* linqt_moments1d_realisations: 0 = autotuned (short timed trials of both, cached per
                       operator pattern, S, R/S and precision), 1 = stacked in one launch, 2 = one solve each */
  int operator_precision; /* values of H in the 1D recursions (linqt_moments1d[_dev],
                       linqt_moments1d_realisations[_dev]): 0 = complex128 (default), 1 = complex64 (each
                       value rounded once to FP32, products accumulated in FP64; every layout, persistent
                       recursion); other solvers accept 0 only */
  int thread_shape; /* 1D moments (linqt_moments1d[_dev]) in one persistent launch: 0 = the format's
                       choice (shape 0, or autotuned with LINQT_FORMAT_AUTO); s + 1 = thread shape s,
                       for tests and experiments (shape s of a block of R columns: min(R, 32) >> s
                       threads per row, at most 8 columns per thread; an invalid s is
                       LINQT_ERR_INVALID) */
  int reserved[7];
} linqt_opts;

/* ---- library / sessions ------------------------------------------------ */
int linqt_abi_version(void);
const char *linqt_last_error(void);
int linqt_session_create(int device, linqt_session **out);
int linqt_session_destroy(linqt_session *s);
/* Run the session's work on an externally owned stream (e.g. torch's current stream). */
int linqt_session_set_stream(linqt_session *s, void *cuda_stream);
int linqt_session_get_stream(linqt_session *s, void **cuda_stream);
/* Wait for the session's work; reports LINQT_ERR_TIMEOUT if a persistent recursion
 * kernel's bounded grid-barrier wait gave up since the last check. */
int linqt_session_synchronize(linqt_session *s);
/* Release cached device workspaces. */
int linqt_session_trim(linqt_session *s);
/* Cumulative device time (ms, CUDA events on the session stream) spent in each
 * phase since the last reset: [0] recursion, [1] moment contraction, [2] FFT
 * reconstruction, [3] other; launches[0..3] the kernel launches per phase. */
int linqt_session_phase_times(linqt_session *s, double ms[4], long launches[4], int reset);
int linqt_session_enable_timing(linqt_session *s, int on);
/* Run this session's persistent recursion kernels with at most `share` (0 < share <= 1) of the
 * device's co-resident CTAs, launched on the session's own stream.  By default (share = 1)
 * every persistent kernel of every session takes the whole device, one at a time (they queue
 * on a device-wide cooperative lane, since two full-device grids could not be resident
 * together).  Sessions whose shares add up to at most 1 can run their recursions at the
 * same time; a grid that still does not become resident in time ends its solve with
 * LINQT_ERR_TIMEOUT instead of waiting (the server retries such a request with share 1).
 * Results depend on the share only through the order of the partial sums (last digits). */
int linqt_session_set_sm_share(linqt_session *s, double share);
/* Fault injection for tests of the timeout path (no counterpart in the reference).  From the
 * next solve on, the grid barriers of the session's persistent kernels wait for
 * extra_arrivals CTAs that were never launched and give up after spin_limit polls (0: the
 * normal limit of 2^24); the kernels then return early and the solve reports
 * LINQT_ERR_TIMEOUT.  (0, 0) restores normal barriers.  No other session is affected. */
int linqt_session_inject_barrier_timeout(linqt_session *s, int extra_arrivals, long long spin_limit);
/* Instantiated CUDA graphs held by the session (opts.use_graphs) and solves launched from them. */
int linqt_session_graph_stats(linqt_session *s, int *graphs, long *replays);

/* ---- operators: SparseMatrixType (include/sparse_matrix.hpp:45-88) ------ */
/* ConvertFromCSR (src/mkl_sparse_matrix.cpp:39-54) + BuildOPFromCSRFile (include/sparse_matrix.hpp:100-108) */
int linqt_csr_create(linqt_session *s, int n, const int *rowptr, const int *col, const double *val, int storage,
                     linqt_op **out);
int linqt_op_destroy(linqt_op *op);
/* dimension and Hermitian-expanded non-zeros (diagonal included) */
int linqt_op_info(const linqt_op *op, int *n, long *nnz);
/* The autotuner's cached decisions for this operator (LINQT_FORMAT_AUTO and
 * opts.realisations = 0), as text: one "key choice" line per tuned case, the key naming the
 * recursion, block width, precision and second operator, the choice a layout and thread shape
 * ("csr", "csr_nocache", "sell<C>", "sell<C>_local"; "shape <s>"), a block width or a
 * realisations mode.  Writes at most cap bytes including the terminating NUL; *len = the full
 * length without it (call with cap = 0 to size the buffer).  No LinQT counterpart. */
int linqt_op_tuned(const linqt_op *op, char *buf, long cap, long *len);
/* H <- a*H + b*I  -- SparseMatrixType::Rescale (src/mkl_sparse_matrix.cpp:73-97) */
int linqt_op_rescale(linqt_op *op, const double a[2], const double b[2]);
/* y <- a*op*x + b*y for ncols column-major vectors of length n (ld = n):
 * SparseMatrixType::Multiply (src/mkl_sparse_matrix.cpp:56-69) for ncols = 1,
 * SparseMatrixType::BatchMultiply (src/mkl_sparse_matrix.cpp:102-106) for ncols > 1.  Host pointers. */
int linqt_op_multiply(linqt_session *s, const linqt_op *op, const double a[2], const double *x, const double b[2],
                      double *y, int ncols);
/* Gershgorin bounds of the Hermitian operator in FP64 on the device (replaces
 * utility::SpectralBounds, src/chebyshev_solver.cpp:8-23, which reads ./BOUNDS). */
int linqt_spectral_bounds(linqt_session *s, const linqt_op *op, double *lo, double *hi);

/* ---- states -------------------------------------------------------------- */
/* R random-phase states r_i = exp(i phi_i)/sqrt(N), phi = 2 pi u, written R x N
 * (state-major, interleaved complex) to device memory.  u comes from Philox4x32-10 with
 * key = seed and counter = (index lo, index hi, 0, 0), index = r*N + i; u = (x >> 11) 2^-53
 * with x = (w0 << 32) | w1.  Replaces the phase filler qstates::FillWithRandomPhase
 * (include/quantum_states.hpp:231-252), which LinQT declares but never calls. */
int linqt_random_phase_states_dev(linqt_session *s, int N, int R, unsigned long long seed, double *states_dev);

/* ---- moment solvers ------------------------------------------------------ */
/* chebyshev::SpectralMoments (src/chebyshev_solver.cpp:176-199): mu[2*M] =
 * sum_r (2/R)(1/2)^{[m=0]} <r|T_m(H) OP|r>.  op = NULL is the identity. */
int linqt_moments1d(linqt_session *s, const linqt_op *H, const linqt_op *op, const double *states, int R, int M,
                    const linqt_opts *opts, double *mu);
int linqt_moments1d_dev(linqt_session *s, const linqt_op *H, const linqt_op *op, const double *states_dev, int R,
                        int M, const linqt_opts *opts, double *mu_dev);

/* chebyshev::SpectralMoments_nonOrth (src/chebyshev_solver.cpp:203-229) with
 * Moments1D_nonOrth::SetInitVectors_nonOrthogonal / Iterate_nonOrthogonal
 * (src/chebyshev_moments.cpp:63-153): 1D moments in a non-orthogonal basis with overlap
 * matrix S, mu[2*M] = sum_r (2/R)(1/2)^{[m=0]} <r|T_m> with
 *   T_0 = S^-1 r (op = NULL) or op S^-1 r,  T_1 = S^-1 H T_0,  T_{m+1} = 2 S^-1 H T_m - T_{m-1}.
 * Each S^-1 is a BiCGSTAB solve as linalg::orthogonalize (src/mkl_linear_algebra.cpp:100-132)
 * runs it with Eigen 3.4: Jacobi preconditioner, x0 = 0, stop when |r| <= tol |b| or after
 * maxit iterations (the reference: tol = 1e-4, maxit = 2000).  S is used as its handle holds
 * it: the reference hands the solver the CSR arrays as the file stores them (the upper
 * triangle), so create S with LINQT_STORAGE_GENERAL from those arrays to reproduce it.
 * FP64 only.  iterations (may be NULL) gets the BiCGSTAB iterations summed over all solves
 * (the _dev form synchronises the session stream when it is given).  The reference solves
 * twice more per state after the last moment it uses; those solves do not reach mu and are
 * not run. */
int linqt_moments1d_nonorth(linqt_session *s, const linqt_op *H, const linqt_op *op, const linqt_op *S,
                            const double *states, int R, int M, double tol, int maxit, const linqt_opts *opts,
                            double *mu, long *iterations);
int linqt_moments1d_nonorth_dev(linqt_session *s, const linqt_op *H, const linqt_op *op, const linqt_op *S,
                                const double *states_dev, int R, int M, double tol, int maxit,
                                const linqt_opts *opts, double *mu_dev, long *iterations);

/* Disorder realisations batched in one recursion (no reference counterpart: LinQT runs
 * one Hamiltonian per process).  H[0..S) share one sparsity pattern (e.g. Anderson disorder
 * seeds); states are R x N with R = S * Rs, the Rs states of realisation r in rows
 * [r Rs, (r+1) Rs).  All run as one R-wide block in one persistent launch, the grid split into
 * S groups of CTAs, each reading its realisation's values and columns.  mu[2*S*M]: the
 * SpectralMoments of each realisation (identity operator) with its Rs states.  Rs a power of
 * two <= 256. */
int linqt_moments1d_realisations(linqt_session *s, const linqt_op *const *H, int S, const double *states, int R,
                                 int M, const linqt_opts *opts, double *mu);
int linqt_moments1d_realisations_dev(linqt_session *s, const linqt_op *const *H, int S, const double *states_dev,
                                     int R, int M, const linqt_opts *opts, double *mu_dev);

/* chebyshev::TimeDependentCorrelations (src/chebyshev_solver.cpp:231-275) with
 * MomentsTD::Evolve (src/chebyshev_momentsTD.cpp:4-46): for each state, PhiL = OPL phi and
 * PhiR = phi; at time step n (t = n dt, fs) mu[m*NT + n] += (2/R)(1/2)^{[m=0]}
 * <PhiL|T_m(H) OPR PhiR>, then PhiL and PhiR evolve by exp(-i H dt / hbar), hbar =
 * 0.6582119624 eV fs, as the series sum_k (2 - [k=0]) (-i)^k J_k(dt w) T_k(H), w =
 * band_width / 2 / hbar, times exp(-i band_center dt / hbar), truncated before the first
 * |J_k| <= 1e-10.  H must already be rescaled with band_width / band_center (eV).
 * mu: 2*M*NT doubles (MomentsTD layout).  FP64 only.  opl/opr = NULL are identities. */
int linqt_moments_td(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                     const double *states, int R, int M, int NT, double dt, double band_width, double band_center,
                     const linqt_opts *opts, double *mu);
int linqt_moments_td_dev(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                         const double *states_dev, int R, int M, int NT, double dt, double band_width,
                         double band_center, const linqt_opts *opts, double *mu_dev);

/* timeCorrelationsFromChebmom (src/timeCorrelationsFromChebmom.cpp:17-68) with
 * MomentsTD::ApplyJacksonKernel (src/chebyshev_momentsTD.cpp:135-154): the Jackson kernel over
 * m (broad_meV), then corr[n] = N/(band_width/2) sum_m delta_chebF(x, m) Re mu(m, n) at the
 * energy x = (energy - band_center)/(band_width/2), t[n] = n dt.  mu: M x NT (MomentsTD
 * layout); M_used (may be NULL) gets the moments kept. */
int linqt_time_correlation_from_moments(linqt_session *s, const double *mu, int M, int NT, int N, double band_width,
                                        double band_center, double dt, double broad_meV, double energy, double *t,
                                        double *corr, int *M_used);

/* chebyshev::CorrelationExpansionMoments (src/chebyshev_solver.cpp:86-172) with the
 * default BATCH_SIZE: mu[2*M*M] row-major mu(mL, mR), symmetrised and scaled by
 * (4/R)(1/2)^{[mL=0]}(1/2)^{[mR=0]}.  opl/opr = NULL are identities. */
int linqt_moments2d(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                    const double *states, int R, int M, const linqt_opts *opts, double *mu);
int linqt_moments2d_dev(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                        const double *states_dev, int R, int M, const linqt_opts *opts, double *mu_dev);

/* chebyshev::Kubo_solver_FFT::compute with one section (src/Kubo_solver_FFT.cpp:12-136,
 * src/Bastin_FFTs.cpp:6-173, src/Greenwood_FFTs.cpp:6-91) and its post-processing
 * (src/Kubo_solver_FFT_postProcess.cpp:120-397).  nump >= M.  Outputs of length nump,
 * ascending energy: E (printed as a*E - b by the reference), sigma, integrand (Bastin;
 * may be NULL).  band_width/band_center are the rescaling of H (a = band_width/2). */
int linqt_kubo_fft(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                   const double *states, int R, int M, int nump, int formula, double band_width, double band_center,
                   const linqt_opts *opts, double *E, double *sigma, double *integrand);
int linqt_kubo_fft_dev(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                       const double *states_dev, int R, int M, int nump, int formula, double band_width,
                       double band_center, const linqt_opts *opts, double *out_dev /* 3*nump: E, sigma, integrand */);

/* One Kubo-Bastin solve: the L/R Chebyshev blocks (L_m = T_m(H) OPL r, R_m = OPR T_m(H) r)
 * are computed once and feed both the 2D moment table of linqt_moments2d (mu, may be NULL)
 * and the FFT Bastin reconstruction of linqt_kubo_fft with formula LINQT_KUBO_BASTIN
 * (E/sigma/integrand, may be NULL).  The reference computes the same two results with two
 * separate solvers, each running its own recursion: chebyshev::CorrelationExpansionMoments
 * (src/chebyshev_solver.cpp:86-172) and Kubo_solver_FFT::compute (src/Kubo_solver_FFT.cpp:12-72). */
int linqt_kubo_bastin(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                      const double *states, int R, int M, int nump, double band_width, double band_center,
                      const linqt_opts *opts, double *mu, double *E, double *sigma, double *integrand);
int linqt_kubo_bastin_dev(linqt_session *s, const linqt_op *H, const linqt_op *opl, const linqt_op *opr,
                          const double *states_dev, int R, int M, int nump, double band_width, double band_center,
                          const linqt_opts *opts, double *mu_dev, double *out_dev /* 3*nump or NULL */);

/* ---- 1D moments without device allocation ------------------------------- */
/* No counterpart in the reference: LinQT allocates host vectors per call and has no
 * notion of device memory.
 *
 * For callers that must not call cudaMalloc or cudaFree while they run.  The regular
 * entry points draw on a per-session workspace cache, and a cache miss or resize calls
 * cudaMalloc/cudaFree; cudaFree synchronises the whole device.  That does not suit a
 * serving loop with a latency bound, a thread sharing the GPU with a framework whose
 * caching allocator owns the device memory, or code that may not call the CUDA
 * allocation API at all.
 *
 * Computes the same result as linqt_moments1d_dev(NULL, H, NULL, ...) with default
 * options: FP64, identity operator, mu_dev[2*M] from the R states at states_dev (R x N
 * complex doubles).  Everything is enqueued on cuda_stream (NULL = the legacy default
 * stream) and the call returns without synchronising.  Scratch lives in one
 * statically sized __device__ array of LINQT_NOALLOC_SCRATCH_BYTES that every GPU
 * loading the library holds until exit.
 *
 * Limits:
 *   - 2 Chebyshev blocks of N x Rc complex doubles (Rc = min(256, next power of two
 *     >= R); R > 256 runs in chunks of 256 states) plus reduction buffers must fit in
 *     that array; a larger solve is rejected with LINQT_ERR_INVALID and a message
 *     giving the size it needs.
 *   - cuda_stream must belong to H's device (LINQT_ERR_INVALID otherwise).
 *   - The first call on a device resolves the array's device address
 *     (cudaGetSymbolAddress) and keeps it for the life of the process; make that first
 *     call before any stream capture.  The kept address does not survive a
 *     cudaDeviceReset or a new primary context on that device: do not call this entry
 *     point after either.
 *   - All calls share the one array, which keeps the last call's contents.  Calls
 *     that overlap on the GPU (two streams, or two host threads) race on it and must
 *     be serialised by the caller. */
#define LINQT_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int linqt_moments1d_noalloc(const linqt_op *H, const double *states_dev, int R, int M, double *mu_dev,
                            void *cuda_stream);

/* ---- reconstructions (FP64 on the device) ------------------------------- */
/* Moments1D::ApplyJacksonKernel (src/chebyshev_moments1D.cpp:68-87) followed by the DOS of
 * spectralFunctionFromChebmom_FFTgrid (src/spectralFunctionFromChebmom_FFTgrid.cpp:35-75).
 * mu[2*M] in; E, dos of length *num_out (= truncated M) out. */
int linqt_dos_from_moments(linqt_session *s, const double *mu, int M, int N, double band_width, double band_center,
                           double broad_meV, double *E, double *dos, int *num_out);
/* Moments1D::ApplyJacksonKernel (src/chebyshev_moments1D.cpp:68-87) followed by the spectral
 * function N/a sum_m delta_chebF(x_i, m) Re mu_m of
 *   grid = LINQT_GRID_UNIFORM:   spectralFunctionFromChebmom (src/spectralFunctionFromChebmom.cpp:35-72):
 *                                x_i = -1 + i 2/(num_div - 1), the sum as it is; num_div <= 0 means 30*M'.
 *                                The end points x = +-1 divide by zero: non-finite, as in the reference;
 *   grid = LINQT_GRID_CHEBYSHEV: spectralFunctionFromChebmom_FFTgrid (as linqt_dos_from_moments):
 *                                x_i = cos(pi (i + 1/2)/num_div), its absolute value; num_div <= 0 means M'.
 * M' = the moments kept by the Jackson kernel.  E = x a + c.  *num_out = num_div points written. */
int linqt_spectral_function_from_moments(linqt_session *s, const double *mu, int M, int N, double band_width,
                                         double band_center, double broad_meV, int grid, int num_div, double *E,
                                         double *out, int *num_out);
/* Moments2D::ApplyJacksonKernel (src/chebyshev_moments2D.cpp:87-117) followed by
 * kuboBastinFromChebmom (src/kuboBastinFromChebmom.cpp:35-81): num_div energies in
 * [-xbound, xbound] (num_div <= 0 means 30*M'), *num_out = num_div-1 points written. */
int linqt_bastin_from_moments(linqt_session *s, const double *mu, int M0, int M1, int N, double band_width,
                              double band_center, double broad_meV, double xbound, int num_div, double *E,
                              double *sigma, int *num_out);
/* LinQT's energy-sum post-processors on a 2D table: Moments2D::ApplyJacksonKernel(broad,
 * broad) and then, for variant
 *   LINQT_SUM_BASTIN      kuboBastinFromChebmom{,_FFTgrid}   (running left-rectangle integral)
 *   LINQT_SUM_GREENWOOD   kuboGreenwoodFromChebmom{,_FFTgrid} (the kernel itself)
 *   LINQT_SUM_BASTIN_I    kuboBastinIFromChebmom             (mean of neighbouring points)
 *   LINQT_SUM_BASTIN_II   kuboBastinIIFromChebmom            (running sum of (k_i + k_{i+1}) dE)
 *   LINQT_SUM_BASTIN_SEA  kuboBastinSeaFromChebmom           (running trapezoid integral)
 *   LINQT_SUM_BASTIN_SURF kuboBastinSurfFromChebmom          (mean of neighbouring points)
 * on grid LINQT_GRID_UNIFORM (num_div points in [-xbound, xbound]; num_div <= 0: 30*M'),
 * LINQT_GRID_CHEBYSHEV (x_i = cos(pi (2i + 1/2)/num_div), the _FFTgrid Greenwood order;
 * num_div <= 0: M') or LINQT_GRID_CHEBYSHEV_ASCENDING (the same points in the ascending order
 * of the _FFTgrid Bastin driver).  M' = max of the truncated moment counts.  Writes
 * *num_out = num_div - 1 points: E = x a + c and the driver's second column.  The drivers
 * other than kuboBastinFromChebmom use xbound = 1, where the first point divides by zero;
 * the same non-finite values result here.  Files src/kubo*FromChebmom*.cpp:33-90. */
enum {
  LINQT_SUM_BASTIN = 0,
  LINQT_SUM_GREENWOOD = 1,
  LINQT_SUM_BASTIN_I = 2,
  LINQT_SUM_BASTIN_II = 3,
  LINQT_SUM_BASTIN_SEA = 4,
  LINQT_SUM_BASTIN_SURF = 5
};
enum { LINQT_GRID_UNIFORM = 0, LINQT_GRID_CHEBYSHEV = 1, LINQT_GRID_CHEBYSHEV_ASCENDING = 2 };
int linqt_kubo_from_moments(linqt_session *s, const double *mu, int M0, int M1, int N, double band_width,
                            double band_center, double broad_meV, int variant, int grid, double xbound, int num_div,
                            double *E, double *out, int *num_out);
/* Jackson kernels alone (in place on host arrays; returns the truncated sizes). */
int linqt_jackson1d(double *mu, int M, double band_width, double broad_meV, int *M_out);
int linqt_jackson2d(double *mu, int M0, int M1, double band_width, double b0, double b1, int *M0_out, int *M1_out);

/* Locality order of the rows of a CSR pattern (host only; no LinQT counterpart: it is the
 * traversal order behind LINQT_FORMAT_LOCAL).  The row graph is ordered breadth-first
 * from a pseudo-peripheral row and cut into halves, recursively, until the parts have at most
 * part_rows rows (>= 1); order[pos] = row, a permutation of 0..n-1.  The pattern must be
 * structurally symmetric (a Hermitian operator's expanded rows are) with columns in [0, n). */
int linqt_locality_order(int n, const int *rowptr, const int *col, int part_rows, int *order);

/* ---- serving (continuous batching of DOS / Kubo-Bastin solves) ----------- */
typedef struct linqt_server linqt_server;
enum { LINQT_REQ_DOS = 0, LINQT_REQ_KUBO_BASTIN = 1 };
typedef struct linqt_request {
  int kind;              /* LINQT_REQ_* */
  const linqt_op *H;     /* rescaled Hamiltonian (device resident) */
  const linqt_op *op;    /* DOS: optional operator; Kubo: velocity used on both sides */
  const double *states;  /* host, R x N (copied at submit); NULL: random phases from seed, made on the device */
  int R, M;
  int precision;         /* LINQT_PREC_* */
  double *mu_out;        /* host result buffer: 2*M (DOS) or 2*M*M (Kubo) */
  unsigned long long seed; /* states == NULL: as linqt_random_phase_states_dev(N = H's dimension, R, seed) */
  /* Kubo-Bastin: sigma_xx(E) from the same recursion (linqt_kubo_bastin) when sigma_out != NULL:
   * 3*nump doubles (E, sigma, integrand), nump >= M; band_width / band_center are H's rescaling */
  double *sigma_out;
  int nump;
  double band_width, band_center;
} linqt_request;
int linqt_server_create(int device, size_t hbm_budget_bytes, int max_active, linqt_server **out);
int linqt_server_submit(linqt_server *srv, const linqt_request *req, long *ticket);
/* status: 0 pending, 1 running, 2 done, <0 error code; latency in ms once done */
int linqt_server_poll(linqt_server *srv, long ticket, int *status, double *latency_ms);
int linqt_server_wait_all(linqt_server *srv);
/* Withdraw a request that has not started: its status becomes LINQT_ERR_CANCELLED and mu_out is
 * not written.  LINQT_ERR_INVALID (and nothing changes) once it runs or has finished. */
int linqt_server_cancel(linqt_server *srv, long ticket);
/* forget a finished request (its ticket becomes unknown); LINQT_ERR_INVALID while it is queued or running */
int linqt_server_release(linqt_server *srv, long ticket);
/* timeouts_retried: requests whose side-by-side persistent recursion did not become
 * co-resident in time and were re-run on the device-wide cooperative lane (see
 * linqt_session_set_sm_share); nomem_retried (may be NULL): requests whose workspaces did not
 * fit next to the running ones and were re-run alone. */
int linqt_server_stats(linqt_server *srv, long *timeouts_retried, long *nomem_retried);
int linqt_server_destroy(linqt_server *srv);

/* ---- operator builder: utilities/wannier2sparse -------------------------- */
/* A Wannier90 tight-binding model, read like tbmodel::readOrbitalPositions / readUnitCell /
 * readWannierModel (utilities/wannier2sparse/src/tbmodel.cpp:5-22, wannier_parser.cpp:45-117):
 * LABEL.xyz (orbital count, then "label x y z" per orbital; spin-down orbitals in the second
 * half), LABEL.uc (3 lattice vectors), LABEL_hr.dat (Wannier90 hoppings).  A LABEL.stdis
 * static-disorder file is rejected with LINQT_ERR_UNSUPPORTED (the reference draws it from
 * std::random_device). */
typedef struct linqt_tbmodel linqt_tbmodel;
int linqt_tbmodel_load(const char *label, linqt_tbmodel **out);
int linqt_tbmodel_destroy(linqt_tbmodel *m);
int linqt_tbmodel_info(const linqt_tbmodel *m, int *num_orbitals, long *num_hoppings);
/* The CSR file hopping_list::save_hopping_list_as_csr writes for
 * tbmodel::WannierOperator(op).wrap_in_supercell(cell_dim) (src/main.cpp:46-53,
 * hopping_list.cpp:158-285): the upper triangle (col >= row) of the operator on a supercell
 * of cell_dim[0] x cell_dim[1] x cell_dim[2] unit cells, rows sorted by column, entries of
 * equal (row, col) summed, 0-based int32 indices.  op: "HAM", one of VX VY VZ, V{X,Y,Z}S{X,Y,Z},
 * SX SY SZ, TX TY TZ (include/operator_utils.hpp:31-35), or NAME with a spinorial NAME.OP file
 * in the working directory (tbmodel.cpp:331-354).  Built on the session's device.
 *   linqt_supercell_csr:     host arrays; rowptr == NULL asks for *n and *nnz only;
 *                            capacity = room in col and val (entries)
 *   linqt_supercell_csr_dev: device arrays (rowptr_dev of *n + 1 entries, from a size query),
 *                            filled on the session stream
 *   linqt_supercell_write_csr: the text file itself (same bytes as the reference writes)
 *   linqt_supercell_operator:  a device operator with the file's (Hermitian-upper) meaning */
int linqt_supercell_csr(linqt_session *s, linqt_tbmodel *m, const char *op, const int cell_dim[3], int *n, long *nnz,
                        int *rowptr, int *col, double *val, long capacity);
int linqt_supercell_csr_dev(linqt_session *s, linqt_tbmodel *m, const char *op, const int cell_dim[3], int *n,
                            long *nnz, int *rowptr_dev, int *col_dev, double *val_dev, long capacity);
int linqt_supercell_write_csr(linqt_session *s, linqt_tbmodel *m, const char *op, const int cell_dim[3],
                              const char *path);
int linqt_supercell_operator(linqt_session *s, linqt_tbmodel *m, const char *op, const int cell_dim[3],
                             linqt_op **out);

#ifdef __cplusplus
}
#endif

#endif
