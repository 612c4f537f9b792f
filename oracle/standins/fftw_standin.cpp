// Implementation of the FFTW3 stand-in declared in fftw3.h.  Test
// infrastructure only.  Complex transforms: iterative radix-2 decimation in time
// (bit-reversal permutation, then log2(n) butterfly passes) when n is a power of
// two, a direct O(n^2) sum with an exact twiddle table otherwise.  Twiddles
// exp(sign*2*pi*i*k/n) are computed per index from cos/sin (no recurrences), so
// the error grows like log2(n)*eps, as for FFTW.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef std::complex<double> cplx;

struct fftw_plan_s {
  int n = 0;
  bool is_r2r = false;
  int sign = 0;
  fftw_r2r_kind kind = FFTW_R2HC;
  fftw_complex *cin = nullptr, *cout = nullptr;
  double *rin = nullptr, *rout = nullptr;
  std::vector<cplx> twiddle;  // exp(sign*2*pi*i*k/n), k < n
  std::vector<int> bitrev;    // only for powers of two
  std::vector<cplx> work;
};

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

extern "C" {

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
  if (n <= 0) return nullptr;
  fftw_plan p = new fftw_plan_s;
  p->n = n;
  p->sign = sign;
  p->cin = in;
  p->cout = out;
  p->twiddle.resize(n);
  for (int k = 0; k < n; k++) {
    const double ang = (double)sign * 2.0 * M_PI * (double)k / (double)n;
    p->twiddle[k] = cplx(std::cos(ang), std::sin(ang));
  }
  if (is_pow2(n)) {
    int lg = 0;
    while ((1 << lg) < n) lg++;
    p->bitrev.resize(n);
    for (int i = 0; i < n; i++) {
      int r = 0;
      for (int b = 0; b < lg; b++)
        if (i & (1 << b)) r |= 1 << (lg - 1 - b);
      p->bitrev[i] = r;
    }
  }
  p->work.resize(n);
  return p;
}

fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned) {
  if (n <= 0) return nullptr;
  fftw_plan p = new fftw_plan_s;
  p->n = n;
  p->is_r2r = true;
  p->kind = kind;
  p->rin = in;
  p->rout = out;
  return p;
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  const int n = p->n;
  if (p->is_r2r) {
    if (p->kind != FFTW_REDFT01) std::abort();
    std::vector<double> res(n);
    for (int k = 0; k < n; k++) {
      double acc = p->rin[0];
      for (int j = 1; j < n; j++) acc += 2.0 * p->rin[j] * std::cos(M_PI * j * (k + 0.5) / n);
      res[k] = acc;
    }
    std::memcpy(p->rout, res.data(), sizeof(double) * n);
    return;
  }
  const cplx *in = reinterpret_cast<const cplx *>(p->cin);
  cplx *w = p->work.data();
  if (!p->bitrev.empty()) {
    for (int i = 0; i < n; i++) w[p->bitrev[i]] = in[i];
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1, stride = n / len;
      for (int s = 0; s < n; s += len)
        for (int j = 0; j < half; j++) {
          const cplx t = p->twiddle[j * stride] * w[s + j + half];
          const cplx u = w[s + j];
          w[s + j] = u + t;
          w[s + j + half] = u - t;
        }
    }
  } else {
    for (int k = 0; k < n; k++) {
      cplx acc = 0.0;
      for (int j = 0; j < n; j++) acc += in[j] * p->twiddle[((long)j * k) % n];
      w[k] = acc;
    }
  }
  std::memcpy(p->cout, w, sizeof(cplx) * n);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

void *fftw_malloc(size_t n) { return std::malloc(n ? n : 1); }

void fftw_free(void *p) { std::free(p); }

}  // extern "C"
