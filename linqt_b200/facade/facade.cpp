// The LinQT C++ interface (facade/include/*.hpp) implemented on the C ABI of
// include/linqt_gpu.h.  Every heavy call goes to the GPU library; this file only moves
// arguments, reads and writes LinQT's text formats, and turns error codes into the
// reference's failure mode (its MKL status asserts: a message and abort()).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "Kubo_solver_FFT.hpp"
#include "chebyshev_moments.hpp"
#include "chebyshev_solver.hpp"
#include "linqt_gpu.h"
#include "quantum_states.hpp"
#include "sparse_matrix.hpp"

namespace {

void check(int rc, const char *what) {
  if (rc != LINQT_OK) {
    std::cerr << "linqt_b200: " << what << " failed (" << rc << "): " << linqt_last_error() << std::endl;
    std::abort();
  }
}

linqt_op *need_op(const SparseMatrixType &A, const char *who) {
  if (!A.device_op()) {
    std::cerr << "linqt_b200: " << who << ": the operator has not been built" << std::endl;
    std::abort();
  }
  return A.device_op();
}

const double *dp(const std::complex<double> *p) { return reinterpret_cast<const double *>(p); }
double *dp(std::complex<double> *p) { return reinterpret_cast<double *>(p); }

}  // namespace

// ---------------------------------------------------------------------------
// sparse operators
// ---------------------------------------------------------------------------
bool Sparse::OPERATOR_FromCSRFile(const std::string input, int &dim, vector<int> &columns, vector<int> &rowIndex,
                                  vector<complex<double> > &values) {
  std::cout << "\nReading the CSR file located at: " << input << std::endl;
  std::ifstream f(input.c_str());
  if (!f.is_open()) {
    std::cerr << "ERROR: Can not open the matrix file";
    return false;
  }
  // The reference reads without checks and goes on with whatever a short or malformed file
  // leaves in the arrays; here a failed read is reported and the file rejected.
  int nnz = 0;
  f >> dim >> nnz;
  if (!f || dim <= 0 || nnz < 0) {
    std::cerr << "ERROR: malformed CSR header (dim nnz) in " << input << std::endl;
    return false;
  }
  values.assign(nnz, complex<double>(0, 0));
  columns.assign(nnz, 0);
  rowIndex.assign(dim + 1, 0);
  for (int i = 0; i < nnz && f; i++) {
    double re = 0, im = 0;
    f >> re >> im;
    values[i] = complex<double>(re, im);
  }
  for (int i = 0; i < nnz && f; i++) f >> columns[i];
  for (int i = 0; i <= dim && f; i++) f >> rowIndex[i];
  if (!f) {
    std::cerr << "ERROR: truncated or malformed CSR file " << input << " (expected " << nnz << " values, " << nnz
              << " columns and " << dim + 1 << " row pointers)" << std::endl;
    return false;
  }
  std::cout << "FINISH READING.Status: SUCCEED" << std::endl;
  return true;
}

void SparseMatrixType::ConvertFromCSR(vector<int> &rowIndex, vector<int> &cols, vector<complex<double> > &vals) {
  rows_ = rowIndex;
  cols_ = cols;
  vals_ = vals;
  linqt_op *h = nullptr;
  check(linqt_csr_create(nullptr, numRows(), rows_.data(), cols_.data(), dp(vals_.data()),
                         LINQT_STORAGE_HERMITIAN_UPPER, &h),
        "linqt_csr_create");
  op_.reset(h, [](linqt_op *p) { linqt_op_destroy(p); });
}

void SparseMatrixType::ConvertFromCOO(vector<int> &rows, vector<int> &cols, vector<complex<double> > &vals) {
  // sort the triplets by (row, column) and build the row pointers
  const int n = numRows();
  std::vector<size_t> order(vals.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return rows[a] != rows[b] ? rows[a] < rows[b] : cols[a] < cols[b];
  });
  vector<int> rp(n + 1, 0), c(vals.size());
  vector<complex<double> > v(vals.size());
  for (size_t i = 0; i < order.size(); ++i) {
    c[i] = cols[order[i]];
    v[i] = vals[order[i]];
    rp[rows[order[i]] + 1]++;
  }
  for (int i = 0; i < n; ++i) rp[i + 1] += rp[i];
  ConvertFromCSR(rp, c, v);
}

void SparseMatrixType::Multiply(const value_t a, const value_t *x, const value_t b, value_t *y) {
  check(linqt_op_multiply(nullptr, need_op(*this, "Multiply"), dp(&a), dp(x), dp(&b), dp(y), 1),
        "linqt_op_multiply");
}

void SparseMatrixType::Multiply(const value_t a, const vector_t &x, const value_t b, vector_t &y) {
  Multiply(a, x.data(), b, y.data());
}

void SparseMatrixType::BatchMultiply(const int batchSize, const value_t a, const value_t *x, const value_t b,
                                     value_t *y) {
  check(linqt_op_multiply(nullptr, need_op(*this, "BatchMultiply"), dp(&a), dp(x), dp(&b), dp(y), batchSize),
        "linqt_op_multiply");
}

void SparseMatrixType::Rescale(const value_t a, const value_t b) {
  check(linqt_op_rescale(need_op(*this, "Rescale"), dp(&a), dp(&b)), "linqt_op_rescale");
}

// ---------------------------------------------------------------------------
// moment containers
// ---------------------------------------------------------------------------
namespace chebyshev {

int Moments::JacksonKernelMomCutOff(const double broad) {
  assert(broad > 0);
  return (int)std::ceil(M_PI / (2.0 * broad / 1000 / BandWidth()));
}

double Moments::JacksonKernel(const double m, const double Mom) {
  const double phi = M_PI / (Mom + 1.0);
  return ((Mom - m + 1) * std::cos(phi * m) + std::sin(phi * m) * std::cos(phi) / std::sin(phi)) / (Mom + 1.0);
}

static void print_info(Moments &m, const std::string &title, const std::string &size) {
  std::cout << "\n\n" << title << std::endl;
  std::cout << "\tSYSTEM:\t\t\t" << m.SystemLabel() << std::endl;
  if (m.SystemSize() > 0) std::cout << "\tSIZE:\t\t\t" << m.SystemSize() << std::endl;
  std::cout << "\tMOMENTS SIZE:\t\t" << size << std::endl;
  std::cout << "\tSCALE FACTOR:\t\t" << m.ScaleFactor() << std::endl;
  std::cout << "\tSHIFT FACTOR:\t\t" << m.ShiftFactor() << std::endl;
  std::cout << "\tENERGY SPECTRUM:\t(" << -m.HalfWidth() + m.BandCenter() << " , " << m.HalfWidth() + m.BandCenter()
            << ")" << std::endl
            << std::endl;
}

// file header "N BW BC" then the moment counts; the label is the file name without extension
static std::ifstream open_moments(Moments &m, const std::string &name, const char *ext) {
  const size_t pos = name.find(ext);
  if (pos == std::string::npos) {
    std::cerr << "The first argument does not seem to be a valid " << ext << " file" << std::endl;
    std::abort();
  }
  m.SystemLabel(name.substr(0, pos));
  std::ifstream f(name.c_str());
  if (!f.is_open()) {
    std::cerr << "cannot open " << name << std::endl;
    std::abort();
  }
  int n = 0;
  double bw = 0, bc = 0;
  f >> n >> bw >> bc;
  m.SystemSize(n);
  m.BandWidth(bw);
  m.BandCenter(bc);
  return f;
}

Moments1D::Moments1D(std::string momfilename) {
  std::ifstream f = open_moments(*this, momfilename, ".chebmom1D");
  f >> _numMoms;
  MomentVector(Moments::vector_t(_numMoms, 0.0));
  for (size_t m = 0; m < _numMoms; m++) {
    double re = 0, im = 0;
    f >> re >> im;
    (*this)(m) = value_t(re, im);
  }
}

void Moments1D::MomentNumber(const size_t numMoms) {
  vector_t mu(numMoms, 0.0);
  for (size_t m = 0; m < numMoms && m < _numMoms; m++) mu[m] = (*this)(m);
  _numMoms = numMoms;
  MomentVector(mu);
}

void Moments1D::saveIn(std::string filename) {
  std::ofstream f(filename.c_str());
  f.precision(std::numeric_limits<double>::digits10);
  f << SystemSize() << " " << BandWidth() << " " << BandCenter() << std::endl;
  f << HighestMomentNumber() << std::endl;
  for (auto mom : MomentVector()) f << mom.real() << " " << mom.imag() << std::endl;
}

void Moments1D::ApplyJacksonKernel(const double broad) {
  int Mt = 0;
  check(linqt_jackson1d(dp(MomentVector().data()), (int)_numMoms, BandWidth(), broad, &Mt), "linqt_jackson1d");
  std::cout << "Kernel reduced the number of moments to " << Mt << " for a broadening of " << M_PI / Mt
            << std::endl;
  MomentNumber(Mt);
}

void Moments1D::Print() { print_info(*this, "CHEBYSHEV 1D MOMENTS INFO", std::to_string(HighestMomentNumber())); }

// .chebmomTD: "N BW BC NT dt", "M NT", then mu(m, n) row-major (src/chebyshev_momentsTD.cpp:49-99)
MomentsTD::MomentsTD(std::string momfilename) : _numMoms(0), _maxTimeStep(0), _timeStep(0), _dt(0) {
  std::ifstream f = open_moments(*this, momfilename, ".chebmomTD");
  f >> _maxTimeStep >> _dt >> _numMoms >> _maxTimeStep;
  MomentVector(Moments::vector_t(_numMoms * _maxTimeStep, 0.0));
  for (size_t q = 0; q < _numMoms * _maxTimeStep; q++) {
    double re = 0, im = 0;
    f >> re >> im;
    MomentVector((int)q) = value_t(re, im);
  }
}

void MomentsTD::MomentNumber(const size_t numMoms) {
  assert(numMoms <= _numMoms);
  vector_t mu(numMoms * _maxTimeStep, 0.0);
  for (size_t m = 0; m < numMoms; m++)
    for (size_t n = 0; n < _maxTimeStep; n++) mu[m * _maxTimeStep + n] = (*this)(m, n);
  _numMoms = numMoms;
  MomentVector(mu);
}

// Jackson factors over m for every time step (src/chebyshev_momentsTD.cpp:135-154)
void MomentsTD::ApplyJacksonKernel(const double broad) {
  assert(broad > 0);
  const double eta = 2.0 * broad / 1000 / BandWidth();
  size_t maxMom = (size_t)ceil(M_PI / eta);
  if (maxMom > HighestMomentNumber()) maxMom = HighestMomentNumber();
  std::cout << "Kernel reduced the number of moments to " << maxMom << " for a broadening of " << M_PI / maxMom
            << std::endl;
  MomentNumber(maxMom);
  const double phi_J = M_PI / (double)(maxMom + 1.0);
  for (size_t m = 0; m < maxMom; m++) {
    const double g = ((maxMom - m + 1) * cos(phi_J * m) + sin(phi_J * m) * cos(phi_J) / sin(phi_J)) * phi_J / M_PI;
    for (size_t n = 0; n < MaxTimeStep(); n++) (*this)(m, n) *= g;
  }
}

void MomentsTD::saveIn(std::string filename) {
  std::ofstream f(filename.c_str());
  f.precision(std::numeric_limits<double>::digits10);
  f << SystemSize() << " " << BandWidth() << " " << BandCenter() << " " << MaxTimeStep() << " " << TimeDiff() << " "
    << std::endl;
  f << HighestMomentNumber() << " " << MaxTimeStep() << " " << std::endl;
  for (auto mom : MomentVector()) f << mom.real() << " " << mom.imag() << std::endl;
}

void MomentsTD::Print() {
  print_info(*this, "CHEBYSHEV TD MOMENTS INFO",
             std::to_string(HighestMomentNumber()) + " x " + std::to_string(MaxTimeStep()));
}

Moments2D::Moments2D(std::string momfilename) {
  std::ifstream f = open_moments(*this, momfilename, ".chebmom2D");
  f >> numMoms[0] >> numMoms[1];
  MomentVector(Moments::vector_t((size_t)numMoms[0] * numMoms[1], 0.0));
  for (int m0 = 0; m0 < numMoms[0]; m0++)
    for (int m1 = 0; m1 < numMoms[1]; m1++) {
      double re = 0, im = 0;
      f >> re >> im;
      (*this)(m0, m1) = value_t(re, im);
    }
}

void Moments2D::MomentNumber(const int mom0, const int mom1) {
  assert(mom0 <= numMoms[0] && mom1 <= numMoms[1]);
  vector_t mu((size_t)mom0 * mom1, 0.0);
  for (int m0 = 0; m0 < mom0; m0++)
    for (int m1 = 0; m1 < mom1; m1++) mu[(size_t)m0 * mom1 + m1] = (*this)(m0, m1);
  numMoms = {mom0, mom1};
  MomentVector(mu);
}

void Moments2D::ApplyJacksonKernel(const double b0, const double b1) {
  int M0 = 0, M1 = 0;
  check(linqt_jackson2d(dp(MomentVector().data()), numMoms[0], numMoms[1], BandWidth(), b0, b1, &M0, &M1),
        "linqt_jackson2d");
  std::cout << "Kernel reduced the number of moments to " << M0 << " " << M1 << std::endl;
  // linqt_jackson2d leaves the truncated table in the leading M0 x M1 block, row pitch M1
  vector_t mu(MomentVector().begin(), MomentVector().begin() + (size_t)M0 * M1);
  numMoms = {M0, M1};
  MomentVector(mu);
}

void Moments2D::saveIn(std::string filename) {
  std::ofstream f(filename.c_str());
  f.precision(std::numeric_limits<double>::digits10);
  f << SystemSize() << " " << BandWidth() << "  " << BandCenter() << std::endl;
  for (auto x : numMoms) f << x << " ";
  f << std::endl;
  for (auto mom : MomentVector()) f << mom.real() << " " << mom.imag() << std::endl;
}

void Moments2D::Print() {
  print_info(*this, "CHEBYSHEV 2D MOMENTS INFO",
             "(" + std::to_string(HighestMomentNumber(0)) + " x " + std::to_string(HighestMomentNumber(1)) + ")");
}

// ---------------------------------------------------------------------------
// solvers
// ---------------------------------------------------------------------------
std::array<double, 2> utility::SpectralBounds(SparseMatrixType &) {
  double lowest = -100, highest = 100;
  std::ifstream f("BOUNDS");
  if (f.is_open()) f >> lowest >> highest;
  return {lowest, highest};
}

int TimeDependentCorrelations(SparseMatrixType &OPL, SparseMatrixType &OPR, chebyshev::MomentsTD &chebMoms,
                              qstates::generator &gen) {
  const int N = (int)chebMoms.SystemSize(), M = (int)chebMoms.HighestMomentNumber();
  const int NT = (int)chebMoms.MaxTimeStep();
  int R = 0;
  std::vector<std::complex<double> > st = qstates::collect_states(gen, N, &R);
  if (R == 0 || M == 0 || NT == 0) return 0;
  std::vector<std::complex<double> > mu((size_t)M * NT);
  check(linqt_moments_td(nullptr, need_op(chebMoms.Hamiltonian(), "TimeDependentCorrelations"),
                         OPL.isIdentity() ? nullptr : need_op(OPL, "TimeDependentCorrelations"),
                         OPR.isIdentity() ? nullptr : need_op(OPR, "TimeDependentCorrelations"), dp(st.data()), R, M,
                         NT, chebMoms.TimeDiff(), chebMoms.BandWidth(), chebMoms.BandCenter(), nullptr,
                         dp(mu.data())),
        "linqt_moments_td");
  for (size_t q = 0; q < mu.size(); q++) chebMoms.MomentVector((int)q) += mu[q];  // accumulates, as the reference
  return 0;
}

int SpectralMoments(SparseMatrixType &OP, chebyshev::Moments1D &chebMoms, qstates::generator &gen) {
  const int N = (int)chebMoms.SystemSize(), M = (int)chebMoms.HighestMomentNumber();
  int R = 0;
  std::vector<std::complex<double> > st = qstates::collect_states(gen, N, &R);
  if (R == 0 || M == 0) return 0;
  std::vector<std::complex<double> > mu(M);
  check(linqt_moments1d(nullptr, need_op(chebMoms.Hamiltonian(), "SpectralMoments"),
                        OP.isIdentity() ? nullptr : need_op(OP, "SpectralMoments"), dp(st.data()), R, M, nullptr,
                        dp(mu.data())),
        "linqt_moments1d");
  for (int m = 0; m < M; m++) chebMoms(m) += mu[m];  // the reference accumulates onto the table
  return 0;
}

int SpectralMoments_nonOrth(SparseMatrixType &OP, chebyshev::Moments1D_nonOrth &chebMoms, qstates::generator &gen) {
  const int N = (int)chebMoms.SystemSize(), M = (int)chebMoms.HighestMomentNumber();
  SparseMatrixType *S = chebMoms.overlap();
  if (!S) {
    std::cerr << "SpectralMoments_nonOrth: no overlap matrix (set_S)" << std::endl;
    std::abort();
  }
  int R = 0;
  std::vector<std::complex<double> > st = qstates::collect_states(gen, N, &R);
  if (R == 0 || M == 0) return 0;
  // the solver sees S's CSR arrays as stored (linalg::orthogonalize maps them into Eigen as
  // they are, src/mkl_linear_algebra.cpp:100-118): a general-storage operator of the same arrays
  linqt_op *s_op = nullptr;
  check(linqt_csr_create(nullptr, S->numRows(), S->rows()->data(), S->cols()->data(), dp(S->vals()->data()),
                         LINQT_STORAGE_GENERAL, &s_op),
        "linqt_csr_create (S)");
  std::vector<std::complex<double> > mu(M);
  long iters = 0;
  const int rc = linqt_moments1d_nonorth(nullptr, need_op(chebMoms.Hamiltonian(), "SpectralMoments_nonOrth"),
                                         OP.isIdentity() ? nullptr : need_op(OP, "SpectralMoments_nonOrth"), s_op,
                                         dp(st.data()), R, M, 1e-4, 2000, nullptr, dp(mu.data()), &iters);
  linqt_op_destroy(s_op);
  check(rc, "linqt_moments1d_nonorth");
  std::cout << "#BiCGSTAB iterations (all solves): " << iters << std::endl;
  for (int m = 0; m < M; m++) chebMoms(m) += mu[m];  // the reference accumulates onto the table
  return 0;
}

int CorrelationExpansionMoments(SparseMatrixType &OPL, SparseMatrixType &OPR, chebyshev::Moments2D &chebMoms,
                                qstates::generator &gen) {
  const int N = (int)chebMoms.SystemSize();
  const int M0 = chebMoms.HighestMomentNumber(0), M1 = chebMoms.HighestMomentNumber(1);
  const int M = std::max(M0, M1);
  int R = 0;
  std::vector<std::complex<double> > st = qstates::collect_states(gen, N, &R);
  if (R == 0 || M == 0) return 0;
  std::vector<std::complex<double> > mu((size_t)M * M);
  check(linqt_moments2d(nullptr, need_op(chebMoms.Hamiltonian(), "CorrelationExpansionMoments"),
                        OPL.isIdentity() ? nullptr : need_op(OPL, "CorrelationExpansionMoments"),
                        OPR.isIdentity() ? nullptr : need_op(OPR, "CorrelationExpansionMoments"), dp(st.data()), R,
                        M, nullptr, dp(mu.data())),
        "linqt_moments2d");
  // The reference sums the raw table onto chebMoms and then symmetrises and scales the
  // whole table (src/chebyshev_solver.cpp:148-162); both steps are linear, so the result is
  // the symmetrised, scaled old table plus the finished moments of these states.
  for (int i = 0; i < M0; i++)
    for (int j = i; j < M1; j++) {
      double scal = 4.0 / R;
      if (i == 0) scal *= 0.5;
      if (j == 0) scal *= 0.5;
      const bool has_ji = j < M0 && i < M1;
      const std::complex<double> old = scal * (chebMoms(i, j) + (has_ji ? std::conj(chebMoms(j, i)) : 0.0)) / 2.0;
      const std::complex<double> v = old + mu[(size_t)i * M + j];
      chebMoms(i, j) = v;
      if (has_ji) chebMoms(j, i) = std::conj(v);
    }
  return 0;
}

// ---------------------------------------------------------------------------
// Kubo_solver_FFT
// ---------------------------------------------------------------------------
Kubo_solver_FFT::r_value_t Kubo_solver_FFT::Jackson_kernel(const int m, const int M) {
  const double x = M_PI / (M + 1.0);
  return ((M - m + 1.0) * std::cos(x * m) + std::sin(x * m) / std::tan(x)) / (M + 1.0);
}

void Kubo_solver_FFT::compute(SparseMatrixType &OPL, SparseMatrixType &OPR, qstates::generator &gen) {
  Vectors_sliced &vec = chebVecL_;
  const int N = (int)vec.SystemSize();
  section_size_ = N / num_sections_ + N % num_sections_;
  int R = 0;
  std::vector<std::complex<double> > st = qstates::collect_states(gen, N, &R);
  if (R == 0) return;
  std::vector<double> E(nump_), sigma(nump_), integ(nump_);
  const int f = sym_formula_ == KUBO_BASTIN ? LINQT_KUBO_BASTIN : LINQT_KUBO_GREENWOOD;
  check(linqt_kubo_fft(nullptr, need_op(vec.Hamiltonian(), "Kubo_solver_FFT"),
                       OPL.isIdentity() ? nullptr : need_op(OPL, "Kubo_solver_FFT"),
                       OPR.isIdentity() ? nullptr : need_op(OPR, "Kubo_solver_FFT"), dp(st.data()), R, M_, nump_, f,
                       vec.BandWidth(), vec.BandCenter(), nullptr, E.data(), sigma.data(), integ.data()),
        "linqt_kubo_fft");
  std::cout << "Computed " << R << " states on the GPU" << std::endl;
  std::ofstream out(outputfilename_);
  for (int e = 0; e < nump_; e++) out << E[e] << "  " << sigma[e] << std::endl;
  if (sym_formula_ == KUBO_BASTIN) {
    std::ofstream out2(outputfilename_ + "_integrand");
    for (int e = 0; e < nump_; e++) out2 << E[e] << "  " << integ[e] << std::endl;
  }
}

}  // namespace chebyshev
