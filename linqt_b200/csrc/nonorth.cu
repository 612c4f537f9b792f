// 1D Chebyshev moments in a non-orthogonal basis: chebyshev::SpectralMoments_nonOrth
// (src/chebyshev_solver.cpp:203-229) with Moments1D_nonOrth::SetInitVectors_nonOrthogonal /
// Iterate_nonOrthogonal (src/chebyshev_moments.cpp:63-153).
//
// With an overlap matrix S the recursion runs on S^-1 H:
//   T_0 = S^-1 phi (or OP S^-1 phi),  T_1 = S^-1 H T_0,  T_{m+1} = 2 S^-1 H T_m - T_{m-1},
//   mu_m += (2/R)(1/2)^{[m=0]} <phi|T_m>,
// and every S^-1 is a BiCGSTAB solve (linalg::orthogonalize, src/mkl_linear_algebra.cpp:100-132,
// which calls Eigen 3.4's BiCGSTAB: tolerance 1e-4, at most 2000 iterations, diagonal
// preconditioner, x0 = 0, on the CSR arrays of S exactly as stored).  The solver here follows
// that algorithm step by step (see k_nonorth_1d), so its iterates and its stopping point are
// the reference's up to rounding.
//
// One cooperative launch runs a whole recursion for a block of up to 32 states: the H
// products, the BiCGSTAB iterations and the dot products, with grid barriers between the
// phases (4 per BiCGSTAB iteration).  Each state (block column) has its own solver scalars;
// a column whose solve has converged stops updating while the others go on, exactly as the
// reference's one-state-at-a-time solves would.  The scalars come from grid-wide sums that
// every CTA forms itself in the same fixed order, so all CTAs take the same decisions.
#include <algorithm>
#include <complex>

#include "grid_sync.cuh"
#include "internal.cuh"

namespace linqt {

namespace {

constexpr int kT = 256;       // threads per CTA (the cooperative lane launches 256-thread CTAs)
constexpr int kMaxCols = 32;  // states per launch

struct Csr {
  const int *rp, *ci;
  const double2 *v;
};

struct NonOrthArgs {
  int n, Rb, M, maxit;
  double tol;
  Csr H, S, OP;          // OP.rp == nullptr: identity
  const double2 *invd;   // [n]: 1 / S_ii (1 where the diagonal entry is missing or zero)
  const double2 *phi;    // n x Rb block of the states
  double2 *T0, *T1, *B, *X, *R, *R0, *P, *V, *Sv, *Tv;  // n x Rb blocks
  double2 *part;         // [3][grid][Rb] per-CTA partial sums
  double2 *dots;         // [M][Rb]: <phi|T_m> per column
  long long *iters;      // [Rb]: BiCGSTAB iterations summed over the solves
  GridBarrier *bar;
};

// Solver scalars of one column (identical in every CTA).
struct Col {
  double2 rho, rho_old, rho_next, alpha, w;
  double r0sq, tol2, rr;
  int it, restarts, active, restart;
  long long total_it;
};

// Complex products and differences rounded the same way wherever they are formed (no FMA
// contraction), so that a value one CTA recomputes from a neighbour's data equals the value
// the owner stores: y = D^-1 p, z = D^-1 s and s = r - alpha v.
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 csub_rn(double2 a, double2 b) {
  return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// sum_k A_ik x_k for column c of a block of Rb columns
__device__ __forceinline__ double2 gather(const Csr &A, int i, int c, int Rb, const double2 *x) {
  double2 acc = make_double2(0, 0);
  for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) acc = cfma(A.v[k], x[(size_t)A.ci[k] * Rb + c], acc);
  return acc;
}

// Per-CTA sums of nv values per column (thread t serves column t % Rb), written to
// part[(q * grid + cta) * Rb + c] in a fixed order.
__device__ void cta_partials(const double2 *vals, int nv, double2 *part, int Rb) {
  __shared__ double2 sh[kT];
  for (int q = 0; q < nv; ++q) {
    sh[threadIdx.x] = vals[q];
    __syncthreads();
    if ((int)threadIdx.x < Rb) {
      double2 a = make_double2(0, 0);
      for (int k = threadIdx.x; k < kT; k += Rb) a = cadd(a, sh[k]);
      part[((size_t)q * gridDim.x + blockIdx.x) * Rb + threadIdx.x] = a;
    }
    __syncthreads();
  }
}

// After the grid barrier: the grid-wide totals tot[q * Rb + c] (shared memory), summed by
// every CTA in the same order (kT / Rb threads per column, then a fixed tree).
__device__ void grid_totals(const double2 *part, int nv, int Rb, double2 *tot) {
  __shared__ double2 sh[kT];
  const int per = kT / Rb, c = threadIdx.x % Rb, j = threadIdx.x / Rb;
  for (int q = 0; q < nv; ++q) {
    double2 a = make_double2(0, 0);
    for (int b = j; b < (int)gridDim.x; b += per) a = cadd(a, __ldcg(part + ((size_t)q * gridDim.x + b) * Rb + c));
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int s = per / 2; s > 0; s >>= 1) {
      if (j < s) sh[threadIdx.x] = cadd(sh[threadIdx.x], sh[threadIdx.x + s * Rb]);
      __syncthreads();
    }
    if (j == 0) tot[q * Rb + c] = sh[c];
    __syncthreads();
  }
}

// partial sums -> barrier -> totals; false if the barrier gave up
__device__ bool reduce(const NonOrthArgs &a, const double2 *vals, int nv, double2 *tot) {
  cta_partials(vals, nv, a.part, a.Rb);
  if (!grid_barrier(a.bar, gridDim.x)) return false;
  grid_totals(a.part, nv, a.Rb, tot);
  return true;
}

#define LQ_ELEMS for (long e = (long)blockIdx.x * kT + threadIdx.x; e < ne; e += stride)

// x = S^-1 b by BiCGSTAB (Eigen 3.4's algorithm, see the file comment), all columns at once.
// `extra` (this thread's partial of another column sum) rides on the first reduction; its
// totals go to dots[m_dot] when m_dot >= 0.  Returns false if a barrier gave up.
__device__ bool bicgstab(const NonOrthArgs &a, const double2 *b, double2 *x, Col *col, double2 *tot, double2 extra,
                         int m_dot) {
  const int Rb = a.Rb, c = threadIdx.x % Rb;
  const long ne = (long)a.n * Rb, stride = (long)gridDim.x * kT;
  const double eps = 2.220446049250313e-16, eps2 = eps * eps;
  {
    double2 q[3] = {make_double2(0, 0), make_double2(0, 0), extra};
    LQ_ELEMS {
      const double2 bv = b[e];
      x[e] = make_double2(0, 0);  // x0 = 0, so r = b - S x0 = b
      a.R[e] = bv;
      a.R0[e] = bv;
      a.P[e] = make_double2(0, 0);
      a.V[e] = make_double2(0, 0);
      q[0].x += cabs2(bv);
      q[1] = cfma_conj(bv, bv, q[1]);
    }
    if (!reduce(a, q, 3, tot)) return false;
  }
  if ((int)threadIdx.x < Rb) {
    Col &s = col[threadIdx.x];
    const double rhs = tot[threadIdx.x].x;
    s.r0sq = s.rr = rhs;
    s.tol2 = a.tol * a.tol * rhs;
    s.rho = s.alpha = s.w = make_double2(1, 0);
    s.rho_next = tot[Rb + threadIdx.x];
    s.it = s.restarts = 0;
    s.active = rhs != 0.0;  // |b| = 0: x = 0, no iteration
    if (m_dot >= 0 && blockIdx.x == 0) a.dots[(size_t)m_dot * Rb + threadIdx.x] = tot[2 * Rb + threadIdx.x];
  }
  __shared__ int any_active, any_restart;
  for (;;) {
    if (threadIdx.x == 0) any_active = any_restart = 0;
    __syncthreads();
    if ((int)threadIdx.x < Rb) {
      Col &s = col[threadIdx.x];
      s.active = s.active && s.rr > s.tol2 && s.it < a.maxit;
      s.restart = 0;
      if (s.active) {
        atomicOr(&any_active, 1);
        s.rho_old = s.rho;
        s.rho = s.rho_next;  // <r0, r>
        if (sqrt(cabs2(s.rho)) < eps2 * s.r0sq) {
          s.restart = 1;
          atomicOr(&any_restart, 1);
        }
      }
    }
    __syncthreads();
    if (!any_active) break;
    if (any_restart) {
      // r0 became orthogonal to r: r = b - S x, r0 = r, rho = |r0|^2 = |r|^2
      double2 q = make_double2(0, 0);
      if (col[c].restart) {
        LQ_ELEMS {
          const int i = (int)(e / Rb);
          const double2 r = csub(b[e], gather(a.S, i, c, Rb, x));
          a.R[e] = r;
          a.R0[e] = r;
          q.x += cabs2(r);
        }
      }
      if (!reduce(a, &q, 1, tot)) return false;
      if ((int)threadIdx.x < Rb && col[threadIdx.x].restart) {
        Col &s = col[threadIdx.x];
        s.r0sq = tot[threadIdx.x].x;
        s.rho = make_double2(s.r0sq, 0);
        if (s.restarts++ == 0) s.it = 0;
      }
      __syncthreads();
    }
    // beta = (rho / rho_old) (alpha / w); p = r + beta (p - w v)
    const Col &s = col[c];
    if (s.active) {
      const double2 beta = cmul(cdiv(s.rho, s.rho_old), cdiv(s.alpha, s.w));
      LQ_ELEMS { a.P[e] = cadd(a.R[e], cmul(beta, csub(a.P[e], cmul(s.w, a.V[e])))); }
    }
    if (!grid_barrier(a.bar, gridDim.x)) return false;
    // v = S D^-1 p; <r0, v>
    {
      double2 q = make_double2(0, 0);
      if (s.active) {
        LQ_ELEMS {
          const int i = (int)(e / Rb);
          double2 acc = make_double2(0, 0);
          for (int k = a.S.rp[i]; k < a.S.rp[i + 1]; ++k) {
            const int j = a.S.ci[k];
            acc = cfma(a.S.v[k], cmul_rn(a.invd[j], a.P[(size_t)j * Rb + c]), acc);
          }
          a.V[e] = acc;
          q = cfma_conj(a.R0[e], acc, q);
        }
      }
      if (!reduce(a, &q, 1, tot)) return false;
      if ((int)threadIdx.x < Rb && col[threadIdx.x].active)
        col[threadIdx.x].alpha = cdiv(col[threadIdx.x].rho, tot[threadIdx.x]);
      __syncthreads();
    }
    // s = r - alpha v (formed by the owner and, identically, by every row that gathers it);
    // t = S D^-1 s; |t|^2, <t, s>
    {
      double2 q[2] = {make_double2(0, 0), make_double2(0, 0)};
      if (s.active) {
        const double2 al = s.alpha;
        LQ_ELEMS {
          const int i = (int)(e / Rb);
          const double2 sv = csub_rn(a.R[e], cmul_rn(al, a.V[e]));
          double2 acc = make_double2(0, 0);
          for (int k = a.S.rp[i]; k < a.S.rp[i + 1]; ++k) {
            const size_t jj = (size_t)a.S.ci[k] * Rb + c;
            const double2 sj = csub_rn(a.R[jj], cmul_rn(al, a.V[jj]));
            acc = cfma(a.S.v[k], cmul_rn(a.invd[a.S.ci[k]], sj), acc);
          }
          a.Sv[e] = sv;
          a.Tv[e] = acc;
          q[0].x += cabs2(acc);
          q[1] = cfma_conj(acc, sv, q[1]);
        }
      }
      if (!reduce(a, q, 2, tot)) return false;
      if ((int)threadIdx.x < Rb && col[threadIdx.x].active) {
        const double tt = tot[threadIdx.x].x;
        col[threadIdx.x].w = tt > 0.0 ? cscale(tot[Rb + threadIdx.x], 1.0 / tt) : make_double2(0, 0);
      }
      __syncthreads();
    }
    // x += alpha D^-1 p + w D^-1 s; r = s - w t; |r|^2, <r0, r>
    {
      double2 q[2] = {make_double2(0, 0), make_double2(0, 0)};
      if (s.active) {
        const double2 al = s.alpha, om = s.w;
        LQ_ELEMS {
          const int i = (int)(e / Rb);
          const double2 y = cmul_rn(a.invd[i], a.P[e]), z = cmul_rn(a.invd[i], a.Sv[e]);
          x[e] = cadd(x[e], cadd(cmul(al, y), cmul(om, z)));
          const double2 r = csub(a.Sv[e], cmul(om, a.Tv[e]));
          a.R[e] = r;
          q[0].x += cabs2(r);
          q[1] = cfma_conj(a.R0[e], r, q[1]);
        }
      }
      if (!reduce(a, q, 2, tot)) return false;
      if ((int)threadIdx.x < Rb && col[threadIdx.x].active) {
        Col &t = col[threadIdx.x];
        t.rr = tot[threadIdx.x].x;
        t.rho_next = tot[Rb + threadIdx.x];
        t.it++;
        t.total_it++;
      }
      __syncthreads();
    }
  }
  __syncthreads();
  return true;
}

__global__ void __launch_bounds__(kT) k_nonorth_1d(NonOrthArgs a) {
  __shared__ Col col[kMaxCols];
  __shared__ double2 tot[3 * kMaxCols];
  const int Rb = a.Rb, c = threadIdx.x % Rb;
  const long ne = (long)a.n * Rb, stride = (long)gridDim.x * kT;
  if ((int)threadIdx.x < Rb) col[threadIdx.x].total_it = 0;
  __syncthreads();
  double2 *T0 = a.T0, *T1 = a.T1;
  // T_0 = S^-1 phi, or OP S^-1 phi
  if (a.OP.rp) {
    if (!bicgstab(a, a.phi, a.X, col, tot, make_double2(0, 0), -1)) return;
    LQ_ELEMS { T0[e] = gather(a.OP, (int)(e / Rb), c, Rb, a.X); }
    if (!grid_barrier(a.bar, gridDim.x)) return;
  } else {
    if (!bicgstab(a, a.phi, T0, col, tot, make_double2(0, 0), -1)) return;
  }
  // moment m: T0 = T_{m-1}, T1 = T_m for m >= 1 (T0 = T_0 at m = 0)
  for (int m = 0; m < a.M; ++m) {
    const double2 *Tm = m == 0 ? T0 : T1;
    double2 dq = make_double2(0, 0);
    if (m + 1 == a.M) {  // the last moment: its dot product only
      LQ_ELEMS { dq = cfma_conj(a.phi[e], Tm[e], dq); }
      if (!reduce(a, &dq, 1, tot)) return;
      if (blockIdx.x == 0 && (int)threadIdx.x < Rb) a.dots[(size_t)m * Rb + threadIdx.x] = tot[threadIdx.x];
      break;
    }
    // B = H T_m (and <phi|T_m>, reduced with the solve's first sums)
    LQ_ELEMS {
      a.B[e] = gather(a.H, (int)(e / Rb), c, Rb, Tm);
      dq = cfma_conj(a.phi[e], Tm[e], dq);
    }
    if (!grid_barrier(a.bar, gridDim.x)) return;
    if (m == 0) {  // T_1 = S^-1 H T_0
      if (!bicgstab(a, a.B, T1, col, tot, dq, 0)) return;
      continue;
    }
    // T_{m+1} = 2 S^-1 H T_m - T_{m-1}, written over T_{m-1}
    if (!bicgstab(a, a.B, a.X, col, tot, dq, m)) return;
    LQ_ELEMS { T0[e] = make_double2(2 * a.X[e].x - T0[e].x, 2 * a.X[e].y - T0[e].y); }
    double2 *t = T0;
    T0 = T1;
    T1 = t;
    if (!grid_barrier(a.bar, gridDim.x)) return;
  }
  if (blockIdx.x == 0 && (int)threadIdx.x < Rb) a.iters[threadIdx.x] = col[threadIdx.x].total_it;
}

#undef LQ_ELEMS

// mu[m] (+)= sum_{c < w} (2/R)(1/2)^{[m=0]} dots[m][c]  (fixed order)
__global__ void k_nonorth_mu(const double2 *__restrict__ dots, int M, int Rb, int w, int R, int accumulate,
                             double2 *__restrict__ mu) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    double2 acc = make_double2(0, 0);
    for (int c = 0; c < w; ++c) acc = cadd(acc, dots[(size_t)m * Rb + c]);
    const double scal = (m == 0 ? 0.5 : 1.0) * 2.0 / R;
    const double2 v = cscale(acc, scal);
    mu[m] = accumulate ? cadd(mu[m], v) : v;
  }
}

}  // namespace

void moments1d_nonorth_dev(Session *s, const DeviceOp &H, const DeviceOp *op, const DeviceOp &S,
                           const double2 *states, int R, int M, double tol, int maxit, double2 *mu,
                           long long *iterations) {
  LQ_REQUIRE(R > 0 && M > 0, "moments1d_nonorth: R and M must be positive");
  LQ_REQUIRE(tol > 0 && maxit > 0, "moments1d_nonorth: tolerance and iteration limit must be positive");
  LQ_REQUIRE(S.n == H.n && (!op || op->n == H.n), "moments1d_nonorth: operator dimension mismatch");
  const int N = H.n;
  int Rb = 1;
  while (Rb < R && Rb < kMaxCols) Rb <<= 1;
  // D^-1 of the preconditioner from S as the handle holds it (the first diagonal entry of a
  // row; 1 where it is missing or zero), divided on the host like Eigen's Scalar(1) / value
  std::vector<double2> invd(N, make_double2(1, 0));
  for (int i = 0; i < N; ++i)
    for (int k = S.rowptr[i]; k < S.rowptr[i + 1]; ++k)
      if (S.col[k] == i) {
        const std::complex<double> v(S.val[k].x, S.val[k].y);
        if (v != 0.0) {
          const std::complex<double> r = 1.0 / v;
          invd[i] = make_double2(r.real(), r.imag());
        }
        break;
      }
  const size_t blk = sizeof(double2) * (size_t)N * Rb;
  double2 *d_invd = (double2 *)s->get("no_invd", sizeof(double2) * (size_t)N);
  LQ_CUDA(cudaMemcpyAsync(d_invd, invd.data(), sizeof(double2) * N, cudaMemcpyHostToDevice, s->stream));
  char *W = (char *)s->get("no_blocks", 11 * blk);
  const void *f = (const void *)k_nonorth_1d;
  double2 *dots = (double2 *)s->get("no_dots", sizeof(double2) * (size_t)M * Rb);
  long long *its = (long long *)s->get("no_iters", sizeof(long long) * kMaxCols);
  std::vector<long long> h_its(kMaxCols);
  long long total_its = 0;
  PhaseScope ph(s, PH_RECURSION);
  for (int c0 = 0; c0 < R; c0 += Rb) {
    const int w = std::min(Rb, R - c0);
    NonOrthArgs a;
    a.n = N;
    a.Rb = Rb;
    a.M = M;
    a.maxit = maxit;
    a.tol = tol;
    a.H = Csr{H.d_rowptr, H.d_col, H.d_val64};
    a.S = Csr{S.d_rowptr, S.d_col, S.d_val64};
    a.OP = op ? Csr{op->d_rowptr, op->d_col, op->d_val64} : Csr{nullptr, nullptr, nullptr};
    a.invd = d_invd;
    double2 *b = (double2 *)W;
    a.phi = b;
    a.T0 = b + 1 * (size_t)N * Rb;
    a.T1 = b + 2 * (size_t)N * Rb;
    a.B = b + 3 * (size_t)N * Rb;
    a.X = b + 4 * (size_t)N * Rb;
    a.R = b + 5 * (size_t)N * Rb;
    a.R0 = b + 6 * (size_t)N * Rb;
    a.P = b + 7 * (size_t)N * Rb;
    a.V = b + 8 * (size_t)N * Rb;
    a.Sv = b + 9 * (size_t)N * Rb;
    a.Tv = b + 10 * (size_t)N * Rb;
    a.dots = dots;
    a.iters = its;
    states_to_block_stream(s->stream, s->sm_count, states + (size_t)c0 * N, (void *)a.phi, N, w, Rb);
    a.bar = barrier_for(s);
    // the grid (and its share of the device) is sized per launch
    const int grid = coop_grid(s, f, ((long)N * Rb + kT - 1) / kT, 0);
    a.part = (double2 *)s->get("no_part", sizeof(double2) * 3 * (size_t)grid * Rb);
    void *args[] = {&a};
    coop_launch(s, f, grid, args, 0);
    k_nonorth_mu<<<(M + 255) / 256, 256, 0, s->stream>>>(dots, M, Rb, w, R, c0 > 0, mu);
    LQ_LAUNCHED();
    ph.launches(3);
    if (iterations) {
      LQ_CUDA(cudaMemcpyAsync(h_its.data(), its, sizeof(long long) * kMaxCols, cudaMemcpyDeviceToHost, s->stream));
      LQ_CUDA(cudaStreamSynchronize(s->stream));
      for (int k = 0; k < w; ++k) total_its += h_its[k];
    }
  }
  if (iterations) *iterations = total_its;
}

}  // namespace linqt
