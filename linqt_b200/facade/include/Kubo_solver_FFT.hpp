// LinQT's Kubo_solver_FFT (include/Kubo_solver_FFT.hpp of LinQT) on the B200 library:
// compute(OPL, OPR, gen) runs the recursion, the per-site transforms and the sum over
// sites for all states of the generator on the GPU (linqt_kubo_fft), then writes the
// reference's output files: for KUBO_BASTIN "<out>" (E sigma) and "<out>_integrand"
// (E integrand), for KUBO_GREENWOOD "<out>" (E sigma); two-space separated, default stream
// precision (src/Kubo_solver_FFT_postProcess.cpp:236-268, 370-378).  The reference
// rewrites these files after every state with the running mean; the files after its last
// state are the ones written here.
#ifndef KUBO_BASTIN_SOLVER_HPP
#define KUBO_BASTIN_SOLVER_HPP

#include <complex>
#include <cstring>
#include <iostream>
#include <string>

#include "chebyshev_moments.hpp"
#include "chebyshev_solver.hpp"
#include "sparse_matrix.hpp"

namespace chebyshev {

enum formula { NIL = -1, KUBO_GREENWOOD = 0, KUBO_BASTIN = 1 };

class Kubo_solver_FFT {
 public:
  typedef double r_value_t;

  Kubo_solver_FFT(int M, int num_sections, int nump, formula sym_formula, chebyshev::Vectors_sliced &chebVec,
                  std::string &outputfilename)
      : M_(M), num_sections_(num_sections), nump_(nump), sym_formula_(sym_formula), chebVecL_(chebVec),
        chebVecR_(chebVec), outputfilename_(outputfilename) {}

  void compute(SparseMatrixType &OPL, SparseMatrixType &OPR, qstates::generator &gen);

  int nump() { return nump_; }
  int num_sections() { return num_sections_; }
  size_t section_size() { return section_size_; }
  int num_vectors() { return M_; }
  chebyshev::Vectors_sliced Hamiltonian() { return chebVecL_; }
  std::string &OutputFilename() { return outputfilename_; }
  formula SolverFormula() { return sym_formula_; }

  r_value_t Jackson_kernel(const int m, const int M);

 private:
  int M_, num_sections_, nump_;
  size_t section_size_ = 0;
  formula sym_formula_;
  chebyshev::Vectors_sliced chebVecL_, chebVecR_;
  std::string outputfilename_;
};

}  // namespace chebyshev

#endif
