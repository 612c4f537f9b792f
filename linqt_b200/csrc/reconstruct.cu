// FP64 post-processing on the device: Jackson damping, the DOS on the Chebyshev
// grid, the Kubo-Bastin energy sum, and Gershgorin spectral bounds.
#include <cmath>

#include "internal.cuh"

namespace linqt {

namespace {

// Jackson factor g_m for a table of Mom moments
// (src/chebyshev_moments1D.cpp:79-86, src/chebyshev_moments2D.cpp:105-116)
__device__ __host__ inline double jackson_g(int m, int Mom) {
  const double phi = M_PI / (double)(Mom + 1.0);
  return ((Mom - m + 1) * cos(phi * m) + sin(phi * m) * cos(phi) / sin(phi)) * phi / M_PI;
}

// out[M0t x M1t] = mu[:M0t, :M1t] * g0 * g1  (truncation keeps the top-left block,
// src/chebyshev_moments2D.cpp:4-13)
__global__ void k_jackson2d(const double2 *__restrict__ mu, int M1, int M0t, int M1t, double2 *__restrict__ out) {
  const long tot = (long)M0t * M1t;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t / M1t), j = (int)(t % M1t);
    out[t] = cscale(mu[(size_t)i * M1 + j], jackson_g(i, M0t) * jackson_g(j, M1t));
  }
}

// DOS on E_i = cos(pi (i+1/2)/M): |N/a sum_m delta(E_i, m) Re mu_m|
// (src/spectralFunctionFromChebmom_FFTgrid.cpp:40-75, delta_chebF of
// include/chebyshev_coefficients.hpp:9-14).  One block per energy.
__global__ void k_dos(const double2 *__restrict__ mu, int M, double N, double a, double bc, double *__restrict__ E,
                      double *__restrict__ dos) {
  const int i = blockIdx.x;
  const double x = cos(M_PI * (i + 0.5) / M);
  const double f0 = sqrt(1.0 - x * x), th = acos(x);
  double acc = 0.0;
  for (int m = threadIdx.x; m < M; m += blockDim.x) acc += cos(m * th) / f0 / M_PI * mu[m].x;
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    E[i] = x * a + bc;
    dos[i] = fabs(sh[0] * N / a);
  }
}

// Table conj(DgreenR_chebF(E_i, m)) for the Bastin sum (include/chebyshev_coefficients.hpp:25-32):
// DG(x, m) = -i (x - i f0)^m (x + i m f0) / f0^3 with (x - i f0)^m = exp(-i m acos x).
__global__ void k_dgreen_table(int num_div, int M1, double xbound, double2 *__restrict__ tab) {
  const long tot = (long)num_div * M1;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t / M1), m = (int)(t % M1);
    const double x = -xbound + i * (2 * xbound) / (num_div - 1);
    const double f0 = sqrt(1.0 - x * x), th = acos(x);
    double sn, cs;
    sincos(m * th, &sn, &cs);
    const double2 p = make_double2(cs, -sn);            // (x - i f0)^m
    const double2 q = cmul(p, make_double2(x, m * f0));  // * (x + i m f0)
    const double inv = 1.0 / (f0 * f0 * f0);
    const double2 dg = make_double2(q.y * inv, -q.x * inv);  // -i * q / f0^3
    tab[t] = cconj(dg);
  }
}

// kernel_i = -2N/a^2 sum_m0 delta(E_i, m0) Im(Y(i, m0)),  Y(i, m0) = sum_m1 DG(E_i,m1) mu(m0,m1)
// (src/kuboBastinFromChebmom.cpp:63-72).  One warp per energy.
__global__ void k_bastin_kernel(const double2 *__restrict__ Y, int num_div, int M0, double pref, double xbound,
                                double *__restrict__ kern) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
  if (w >= num_div) return;
  const double x = -xbound + w * (2 * xbound) / (num_div - 1);
  const double f0 = sqrt(1.0 - x * x), th = acos(x);
  double acc = 0.0;
  for (int m0 = l; m0 < M0; m0 += 32) acc += cos(m0 * th) / f0 / M_PI * Y[(size_t)w * M0 + m0].y;
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (l == 0) kern[w] = acc * pref;
}

// left-rectangle cumulative integral (src/kuboBastinFromChebmom.cpp:74-81); single thread,
// fixed order, FP64
__global__ void k_bastin_integrate(const double *__restrict__ kern, int num_div, double xbound, double a, double bc,
                                   double *__restrict__ E, double *__restrict__ sigma) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double acc = 0.0;
  for (int i = 0; i < num_div - 1; ++i) {
    const double e0 = -xbound + i * (2 * xbound) / (num_div - 1);
    const double e1 = -xbound + (i + 1) * (2 * xbound) / (num_div - 1);
    acc += kern[i] * (e1 - e0);
    E[i] = e0 * a + bc;
    sigma[i] = acc;
  }
}

// Gershgorin: per-block min(center - radius), max(center + radius)
__global__ void k_gershgorin(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                             const double2 *__restrict__ v, double2 *__restrict__ part) {
  double lo = INFINITY, hi = -INFINITY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double c = 0.0, r = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      if (ci[k] == i)
        c += v[k].x;
      else
        r += hypot(v[k].x, v[k].y);
    }
    lo = fmin(lo, c - r);
    hi = fmax(hi, c + r);
  }
  __shared__ double sl[256], sh[256];
  sl[threadIdx.x] = lo;
  sh[threadIdx.x] = hi;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sl[threadIdx.x] = fmin(sl[threadIdx.x], sl[threadIdx.x + o]);
      sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = make_double2(sl[0], sh[0]);
}

__global__ void k_minmax(const double2 *__restrict__ part, int nb, double2 *__restrict__ out) {
  if (threadIdx.x || blockIdx.x) return;
  double lo = INFINITY, hi = -INFINITY;
  for (int b = 0; b < nb; ++b) {
    lo = fmin(lo, part[b].x);
    hi = fmax(hi, part[b].y);
  }
  *out = make_double2(lo, hi);
}

}  // namespace

int jackson_cut(int M, double band_width, double broad) {
  const double eta = 2.0 * broad / 1000 / band_width;
  const int maxMom = (int)ceil(M_PI / eta);
  return maxMom > M ? M : maxMom;
}

double jackson_factor(int m, int Mom) { return jackson_g(m, Mom); }

void jackson2d_dev(Session *s, const double2 *mu, int M0, int M1, int M0t, int M1t, double2 *out) {
  (void)M0;
  const long tot = (long)M0t * M1t;
  const int g = (int)std::max(1L, std::min((tot + 255) / 256, (long)s->sm_count * 8));
  k_jackson2d<<<g, 256, 0, s->stream>>>(mu, M1, M0t, M1t, out);
  LQ_LAUNCHED();
}

void dos_grid(Session *s, const double2 *mu, int M, int N, double band_width, double band_center, double *E,
              double *dos) {
  k_dos<<<M, 256, 0, s->stream>>>(mu, M, (double)N, band_width / 2.0, band_center, E, dos);
  LQ_LAUNCHED();
}

void bastin_grid(Session *s, const double2 *mu, int M0, int M1, int N, double band_width, double band_center,
                 double xbound, int num_div, double *E, double *sigma) {
  double2 *tab = (double2 *)s->get("bastin_dg", sizeof(double2) * (size_t)num_div * M1);
  double2 *Y = (double2 *)s->get("bastin_y", sizeof(double2) * (size_t)num_div * M0);
  double *kern = (double *)s->get("bastin_kern", sizeof(double) * (size_t)num_div);
  const long tot = (long)num_div * M1;
  const int g = (int)std::max(1L, std::min((tot + 255) / 256, (long)s->sm_count * 16));
  k_dgreen_table<<<g, 256, 0, s->stream>>>(num_div, M1, xbound, tab);
  LQ_LAUNCHED();
  // Y(i, m0) = sum_m1 conj(tab(i, m1)) mu(m0, m1) = sum_m1 DG(E_i, m1) mu(m0, m1)
  zgemm_cn(s, tab, num_div, mu, M0, M1, Y, false);
  const double a = band_width / 2.0;
  const double pref = -2.0 * N / a / a;
  k_bastin_kernel<<<(num_div * 32 + 255) / 256, 256, 0, s->stream>>>(Y, num_div, M0, pref, xbound, kern);
  LQ_LAUNCHED();
  k_bastin_integrate<<<1, 32, 0, s->stream>>>(kern, num_div, xbound, a, band_center, E, sigma);
  LQ_LAUNCHED();
}

void gershgorin(Session *s, const DeviceOp &A, double *lo, double *hi) {
  const int nb = (int)std::max(1L, std::min(((long)A.n + 255) / 256, (long)s->sm_count * 4));
  double2 *part = (double2 *)s->get("gersh_part", sizeof(double2) * (nb + 1));
  k_gershgorin<<<nb, 256, 0, s->stream>>>(A.n, A.d_rowptr, A.d_col, A.d_val64, part);
  LQ_LAUNCHED();
  k_minmax<<<1, 1, 0, s->stream>>>(part, nb, part + nb);
  LQ_LAUNCHED();
  double2 h;
  LQ_CUDA(cudaMemcpyAsync(&h, part + nb, sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
  LQ_CUDA(cudaStreamSynchronize(s->stream));
  *lo = h.x;
  *hi = h.y;
}

}  // namespace linqt
