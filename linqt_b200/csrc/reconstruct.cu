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

// The spectral function N/a sum_m delta(E_i, m) Re mu_m (delta_chebF of
// include/chebyshev_coefficients.hpp:9-14) on num_div energies, one block per energy:
//   grid 0: x_i = -1 + i 2/(num_div - 1), the sum as it is (src/spectralFunctionFromChebmom.cpp:35-72;
//           the end points divide by zero and come out non-finite there and here);
//   grid 1: x_i = cos(pi (i+1/2)/num_div), its absolute value
//           (src/spectralFunctionFromChebmom_FFTgrid.cpp:35-75).
__global__ void k_dos(const double2 *__restrict__ mu, int M, double N, double a, double bc, int grid, int num_div,
                      double *__restrict__ E, double *__restrict__ dos) {
  const int i = blockIdx.x;
  const double x = grid == 0 ? -1.0 + i * (2 * 1.0) / (num_div - 1) : cos(M_PI * (i + 0.5) / num_div);
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
    const double v = sh[0] * N / a;
    dos[i] = grid == 0 ? v : fabs(v);
  }
}

// ---------------------------------------------------------------------------
// The energy sums of LinQT's post-processors (kuboBastinFromChebmom{,_FFTgrid},
// kuboGreenwoodFromChebmom{,_FFTgrid}, kuboBastin{I,II,Sea,Surf}FromChebmom) on a
// Jackson-damped table mu[M0][M1]:  kernel(x) = pref * sum_{m0,m1} f(x, m0, m1, mu).
// Each is evaluated as Y(i, m0) = sum_m1 B(x_i, m1) mu(m0, m1) (an FP64 GEMM against a
// coefficient table) and a per-energy sum over m0 with the left coefficient.  The
// coefficient functions are those of include/chebyshev_coefficients.hpp:9-32:
//   delta(x, m)  = cos(m acos x) / f0 / pi,            f0 = sqrt(1 - x^2)
//   G(x, m)      = -i (x - i f0)^m / f0,                (x - i f0)^m = exp(-i m acos x)
//   DG(x, m)     = -i (x - i f0)^m (x + i m f0) / f0^3
// ---------------------------------------------------------------------------
enum CoefKind { COEF_DELTA = 0, COEF_G = 1, COEF_DG = 2, COEF_REDG2 = 3 };

// energy i of the grid: 0 uniform in [-xbound, xbound]; 1 cos(pi (2i + 1/2)/n); 2 grid 1 in
// the ascending order of rearrange_crescent_order (src/kuboBastinFromChebmom_FFTgrid.cpp:18-36)
__device__ __host__ inline double grid_energy(int grid, int i, int n, double xbound) {
  if (grid == 0) return -xbound + i * (2 * xbound) / (n - 1);
  if (grid == 2) i = rearranged_source(i, n);
  return cos(M_PI * (2 * i + 0.5) / n);
}

__device__ inline double2 coef(int kind, double x, int m) {
  const double f0 = sqrt(1.0 - x * x), th = acos(x);
  double sn, cs;
  sincos(m * th, &sn, &cs);
  if (kind == COEF_DELTA) return make_double2(cs / f0 / M_PI, 0.0);
  const double2 p = make_double2(cs, -sn);  // (x - i f0)^m
  if (kind == COEF_G) return make_double2(p.y / f0, -p.x / f0);  // -i p / f0
  const double2 q = cmul(p, make_double2(x, m * f0));             // * (x + i m f0)
  const double inv = 1.0 / (f0 * f0 * f0);
  const double2 dg = make_double2(q.y * inv, -q.x * inv);          // -i q / f0^3
  if (kind == COEF_DG) return dg;
  return make_double2(dg.x + dg.x, 0.0);                           // Re DG + conj(Re DG)
}

// tab(i, m) = conj(B(x_i, m)): zgemm_cn conjugates its first operand
__global__ void k_coef_table(int kind, int grid, int num_div, int M1, double xbound, double2 *__restrict__ tab) {
  const long tot = (long)num_div * M1;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t / M1), m = (int)(t % M1);
    tab[t] = cconj(coef(kind, grid_energy(grid, i, num_div, xbound), m));
  }
}

// kernel_i = pref * sum_m0 (left coefficient x Y), one warp per energy, fixed order
__global__ void k_energy_sums(int variant, int grid, const double2 *__restrict__ Y1, const double2 *__restrict__ Y2,
                              int num_div, int M0, double pref, double xbound, double *__restrict__ kern) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, l = threadIdx.x & 31;
  if (w >= num_div) return;
  const double x = grid_energy(grid, w, num_div, xbound);
  double acc = 0.0;
  for (int m0 = l; m0 < M0; m0 += 32) {
    const double2 y1 = Y1[(size_t)w * M0 + m0];
    switch (variant) {
      case 0:  // Bastin: delta(m0) Im(DG(m1) mu)
      case 1:  // Greenwood: delta(m0) Im(G(m1) mu)
      case 2:  // Bastin I: as Greenwood
        acc += coef(COEF_DELTA, x, m0).x * y1.y;
        break;
      case 3: {  // Bastin II: -Re(G(m0) DG(m1) mu - DG(m0) G(m1) mu)
        const double2 y2 = Y2[(size_t)w * M0 + m0];
        const double2 t = csub(cmul(coef(COEF_G, x, m0), y1), cmul(coef(COEF_DG, x, m0), y2));
        acc += -t.x;
        break;
      }
      case 4: {  // sea: -Re((G - conj G)(m0) (2 Re DG)(m1) mu)
        const double2 g = coef(COEF_G, x, m0);
        acc += -cmul(csub(g, cconj(g)), y1).x;
        break;
      }
      default:  // surface: delta(m0) delta(m1) Re mu
        acc += coef(COEF_DELTA, x, m0).x * y1.x;
        break;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (l == 0) kern[w] = acc * pref;
}

// the drivers' output columns (num_div - 1 points); single thread, fixed order, FP64
__global__ void k_energy_output(int variant, int grid, const double *__restrict__ kern, int num_div, double xbound,
                                double a, double bc, double *__restrict__ E, double *__restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double acc = 0.0;
  for (int i = 0; i < num_div - 1; ++i) {
    const double e0 = grid_energy(grid, i, num_div, xbound), e1 = grid_energy(grid, i + 1, num_div, xbound);
    const double de = e1 - e0;
    E[i] = e0 * a + bc;
    switch (variant) {
      case 0: acc += kern[i] * de; out[i] = acc; break;
      case 1: out[i] = kern[i]; break;
      case 2: out[i] = 0.5 * (kern[i] + kern[i + 1]); break;
      case 3: acc += (kern[i] + kern[i + 1]) * de; out[i] = acc; break;
      case 4: acc += 0.5 * (kern[i] + kern[i + 1]) * de; out[i] = acc; break;
      default: out[i] = (kern[i + 1] + kern[i]) / 2.0; break;
    }
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

namespace {
// C(t_n) = scale * sum_{m < T} delta(x, m) (g_m Re mu(m, n)), one thread per time step
__global__ void k_time_correlation(const double2 *__restrict__ mu, int NT, int T, double x, double scale, double dt,
                                   double *__restrict__ t_out, double *__restrict__ c_out) {
  const double phi = M_PI / (double)(T + 1.0);
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < NT; n += gridDim.x * blockDim.x) {
    double out = 0.0;
    for (int m = 0; m < T; ++m) {
      const double g = ((T - m + 1) * cos(phi * m) + sin(phi * m) * cos(phi) / sin(phi)) * phi / M_PI;
      out += coef(COEF_DELTA, x, m).x * (mu[(size_t)m * NT + n].x * g);
    }
    t_out[n] = n * dt;
    c_out[n] = out * scale;
  }
}
}  // namespace

void time_correlation(Session *s, const double2 *mu, int M, int NT, int N, double band_width, double band_center,
                      double dt, double broad_meV, double energy, double *t_out, double *c_out, int *T_out) {
  const int T = jackson_cut(M, band_width, broad_meV);
  const double hw = band_width / 2;
  k_time_correlation<<<(NT + 127) / 128, 128, 0, s->stream>>>(mu, NT, T, (energy - band_center) / hw, N / hw, dt,
                                                               t_out, c_out);
  LQ_LAUNCHED();
  *T_out = T;
}

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
  spectral_grid(s, mu, M, N, band_width, band_center, 1, M, E, dos);
}

void spectral_grid(Session *s, const double2 *mu, int M, int N, double band_width, double band_center, int grid,
                   int num_div, double *E, double *out) {
  LQ_REQUIRE((grid == 0 || grid == 1) && num_div >= 2, "spectral function: bad grid");
  k_dos<<<num_div, 256, 0, s->stream>>>(mu, M, (double)N, band_width / 2.0, band_center, grid, num_div, E, out);
  LQ_LAUNCHED();
}

void energy_sums(Session *s, const double2 *mu, int M0, int M1, int N, double band_width, double band_center,
                 int variant, int grid, double xbound, int num_div, double *E, double *out) {
  LQ_REQUIRE(variant >= 0 && variant <= 5 && grid >= 0 && grid <= 2 && num_div >= 2, "energy sums: bad argument");
  static const int kind1[6] = {COEF_DG, COEF_G, COEF_G, COEF_DG, COEF_REDG2, COEF_DELTA};
  double2 *tab = (double2 *)s->get("esum_tab", sizeof(double2) * (size_t)num_div * M1);
  double2 *Y1 = (double2 *)s->get("esum_y1", sizeof(double2) * (size_t)num_div * M0);
  double2 *Y2 = variant == 3 ? (double2 *)s->get("esum_y2", sizeof(double2) * (size_t)num_div * M0) : nullptr;
  double *kern = (double *)s->get("esum_kern", sizeof(double) * (size_t)num_div);
  const long tot = (long)num_div * M1;
  const int g = (int)std::max(1L, std::min((tot + 255) / 256, (long)s->sm_count * 16));
  // Y(i, m0) = sum_m1 conj(tab(i, m1)) mu(m0, m1) = sum_m1 B(x_i, m1) mu(m0, m1)
  k_coef_table<<<g, 256, 0, s->stream>>>(kind1[variant], grid, num_div, M1, xbound, tab);
  LQ_LAUNCHED();
  zgemm_cn(s, tab, num_div, mu, M0, M1, Y1, false);
  if (Y2) {
    k_coef_table<<<g, 256, 0, s->stream>>>(COEF_G, grid, num_div, M1, xbound, tab);
    LQ_LAUNCHED();
    zgemm_cn(s, tab, num_div, mu, M0, M1, Y2, false);
  }
  const double a = band_width / 2.0, w = N / a / a;
  const double pref[6] = {-2.0 * w, -w, -w, w / 2 / M_PI, w / 2 / M_PI, M_PI * w};
  k_energy_sums<<<(num_div * 32 + 255) / 256, 256, 0, s->stream>>>(variant, grid, Y1, Y2, num_div, M0,
                                                                    pref[variant], xbound, kern);
  LQ_LAUNCHED();
  k_energy_output<<<1, 32, 0, s->stream>>>(variant, grid, kern, num_div, xbound, a, band_center, E, out);
  LQ_LAUNCHED();
}

void bastin_grid(Session *s, const double2 *mu, int M0, int M1, int N, double band_width, double band_center,
                 double xbound, int num_div, double *E, double *sigma) {
  energy_sums(s, mu, M0, M1, N, band_width, band_center, 0, 0, xbound, num_div, E, sigma);
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
