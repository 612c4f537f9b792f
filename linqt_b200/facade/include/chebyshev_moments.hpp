// LinQT's Chebyshev-moment containers (include/chebyshev_moments.hpp of LinQT) for the
// B200 library: Moments (expansion parameters and the non-owning Hamiltonian pointer),
// Moments1D / Moments2D (moment tables with LinQT's .chebmom1D / .chebmom2D files) and
// Vectors_sliced (the parameter carrier Kubo_solver_FFT takes).  The recursion vectors the
// reference keeps in these objects live on the GPU inside the solvers instead.
#ifndef CHEBYSHEV_MOMENTS
#define CHEBYSHEV_MOMENTS

#include <array>
#include <cassert>
#include <complex>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

#include "sparse_matrix.hpp"

namespace chebyshev {
const double CUTOFF = 1.00;

class Moments {
 public:
  typedef std::complex<double> value_t;
  typedef std::vector<value_t> vector_t;

  Moments() {}

  void getMomentsParams(Moments &mom) {
    SetHamiltonian(mom.Hamiltonian());
    SystemLabel(mom.SystemLabel());
    BandWidth(mom.BandWidth());
    BandCenter(mom.BandCenter());
  }

  size_t SystemSize() const { return system_size; }
  string SystemLabel() const { return system_label; }
  double BandWidth() const { return band_width; }
  double HalfWidth() const { return BandWidth() / 2.0; }
  double BandCenter() const { return band_center; }
  double ScaleFactor() const { return chebyshev::CUTOFF / HalfWidth(); }
  double ShiftFactor() const { return -BandCenter() / HalfWidth() / chebyshev::CUTOFF; }
  vector_t &MomentVector() { return mu; }
  value_t &MomentVector(const int i) { return mu[i]; }
  SparseMatrixType &Hamiltonian() const { return *_pNHAM; }

  void SetHamiltonian(SparseMatrixType &NHAM) {
    if (SystemSize() == 0) SystemSize(NHAM.rank());
    assert(NHAM.rank() == (int)SystemSize());
    _pNHAM = &NHAM;
  }
  // H <- ScaleFactor H + ShiftFactor I, on the device copy of the operator
  int Rescale2ChebyshevDomain() {
    Hamiltonian().Rescale(ScaleFactor(), ShiftFactor());
    return 0;
  }
  void SetAndRescaleHamiltonian(SparseMatrixType &NHAM) {
    SetHamiltonian(NHAM);
    Rescale2ChebyshevDomain();
  }
  void SystemSize(const int dim) { system_size = dim; }
  void SystemLabel(string label) { system_label = label; }
  void BandWidth(const double x) { band_width = x; }
  void BandCenter(const double x) { band_center = x; }
  void MomentVector(const vector_t _mu) { mu = _mu; }
  double Rescale2ChebyshevDomain(const double energ) { return (energ - BandCenter()) / HalfWidth(); }

  // the moment cut-off and Jackson factor of src/chebyshev_moments.cpp:24-40
  int JacksonKernelMomCutOff(const double broad);
  double JacksonKernel(const double m, const double Mom);

 private:
  SparseMatrixType *_pNHAM = nullptr;
  std::string system_label;
  size_t system_size = 0;
  double band_width = 0, band_center = 0;
  vector_t mu;
};

class Moments1D : public Moments {
 public:
  Moments1D() : _numMoms(0) {}
  Moments1D(const size_t m0) : _numMoms(m0) { MomentVector(Moments::vector_t(_numMoms, 0.0)); }
  Moments1D(std::string momfilename);

  size_t MomentNumber() const { return _numMoms; }
  size_t HighestMomentNumber() const { return _numMoms; }
  Moments::value_t &operator()(const size_t m0) { return MomentVector(m0); }
  void MomentNumber(const size_t numMoms);
  void saveIn(std::string filename);
  void ApplyJacksonKernel(const double broad);
  void Print();

 private:
  size_t _numMoms;
};

// 1D moments in a non-orthogonal basis (Moments1D_nonOrth of LinQT's
// include/chebyshev_moments.hpp:194-220): a Moments1D plus the overlap matrix S, whose stored
// CSR arrays chebyshev::SpectralMoments_nonOrth hands to the GPU BiCGSTAB solves.
class Moments1D_nonOrth : public Moments1D {
 public:
  Moments1D_nonOrth(const size_t m0) : Moments1D(m0), S_(NULL) {}
  Moments1D_nonOrth(SparseMatrixType &S) : Moments1D(), S_(&S) {}
  Moments1D_nonOrth(const size_t m0, SparseMatrixType &S) : Moments1D(m0), S_(&S) {}
  Moments1D_nonOrth(std::string &momfilename, SparseMatrixType &S) : Moments1D(momfilename), S_(&S) {}

  void set_S(SparseMatrixType &S) { S_ = &S; }
  SparseMatrixType *overlap() const { return S_; }

 private:
  SparseMatrixType *S_;
};

class Moments2D : public Moments {
 public:
  Moments2D() : numMoms({0, 0}) {}
  Moments2D(const size_t m0, const size_t m1) : numMoms({int(m0), int(m1)}) {
    MomentVector(Moments::vector_t((size_t)numMoms[1] * numMoms[0], 0.0));
  }
  Moments2D(std::string momfilename);
  Moments2D(Moments2D mom, const size_t m0, const size_t m1) {
    getMomentsParams(mom);
    numMoms = {int(m0), int(m1)};
    MomentVector(Moments::vector_t((size_t)numMoms[1] * numMoms[0], 0.0));
  }

  array<int, 2> MomentNumber() const { return numMoms; }
  int HighestMomentNumber(const int i) const { return numMoms[i]; }
  int HighestMomentNumber() const { return numMoms[1] > numMoms[0] ? numMoms[1] : numMoms[0]; }
  void MomentNumber(const int mom0, const int mom1);
  Moments::value_t &operator()(const int m0, const int m1) { return MomentVector(m0 * numMoms[1] + m1); }
  void ApplyJacksonKernel(const double b0, const double b1);
  void saveIn(std::string filename);
  void AddSubMatrix(Moments2D &sub, const int mL, const int mR) {
    for (int m0 = 0; m0 < sub.HighestMomentNumber(0); m0++)
      for (int m1 = 0; m1 < sub.HighestMomentNumber(1); m1++) (*this)(mL + m0, mR + m1) += sub(m0, m1);
  }
  void InsertSubMatrix(Moments2D &sub, const int mL, const int mR) {
    for (int m0 = 0; m0 < sub.HighestMomentNumber(0); m0++)
      for (int m1 = 0; m1 < sub.HighestMomentNumber(1); m1++) (*this)(mL + m0, mR + m1) = sub(m0, m1);
  }
  void Print();

 private:
  array<int, 2> numMoms;
};

// Time-domain moment table mu(m, n), m < numMoms, n < maxTimeStep (MomentsTD of LinQT's
// include/chebyshev_moments.hpp:287-360), with LinQT's .chebmomTD file.  The evolution runs
// inside chebyshev::TimeDependentCorrelations on the GPU.
class MomentsTD : public Moments {
 public:
  const double HBAR = 0.6582119624;  // eV fs

  MomentsTD() : _numMoms(1), _maxTimeStep(1), _timeStep(0), _dt(0) {}
  MomentsTD(const size_t m, const size_t n) : _numMoms(m), _maxTimeStep(n), _timeStep(0), _dt(0) {
    MomentVector(Moments::vector_t(m * n, 0.0));
  }
  MomentsTD(std::string momfilename);

  size_t MomentNumber() const { return _numMoms; }
  size_t HighestMomentNumber() const { return _numMoms; }
  size_t CurrentTimeStep() const { return _timeStep; }
  size_t MaxTimeStep() const { return _maxTimeStep; }
  double TimeDiff() const { return _dt; }
  double ChebyshevFreq() const { return HalfWidth() / chebyshev::CUTOFF / HBAR; }
  double ChebyshevFreq_0() const { return BandCenter() / HBAR; }

  void MomentNumber(const size_t mom);
  void MaxTimeStep(const size_t maxTimeStep) { _maxTimeStep = maxTimeStep; }
  void IncreaseTimeStep() { _timeStep++; }
  void ResetTime() { _timeStep = 0; }
  void TimeDiff(const double dt) { _dt = dt; }

  Moments::value_t &operator()(const size_t m, const size_t n) { return MomentVector(m * MaxTimeStep() + n); }
  void ApplyJacksonKernel(const double broad);
  void saveIn(std::string filename);
  void Print();

 private:
  size_t _numMoms, _maxTimeStep, _timeStep;
  double _dt;
};

// Parameters of Kubo_solver_FFT's recursion (number of moments, sections).  The vectors
// themselves are device buffers of the solver.
class Vectors_sliced : public Moments {
 public:
  Vectors_sliced() : numVecs_(0), num_sections_(1) {}
  Vectors_sliced(const int numVecs, const size_t num_sections) : numVecs_(numVecs), num_sections_(num_sections) {}
  Vectors_sliced(Moments &mom, const int numVecs, const size_t num_sections)
      : numVecs_(numVecs), num_sections_(num_sections) {
    getMomentsParams(mom);
  }

  int NumberOfVectors() const { return numVecs_; }
  int NumberOfSections() const { return (int)num_sections_; }
  void SetNumberOfVectors(const int x) { numVecs_ = x; }
  int SetNumSections(const int x) {
    num_sections_ = x;
    return 0;
  }

 private:
  int numVecs_;
  size_t num_sections_;
};

}  // namespace chebyshev

#endif
