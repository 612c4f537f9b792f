// LinQT's solver entry points (include/chebyshev_solver.hpp of LinQT) on the B200 library.
// SpectralMoments and CorrelationExpansionMoments take all states of the generator as one
// block of vectors and run the whole expansion on the GPU (linqt_moments1d /
// linqt_moments2d); the results are those of the reference's state-by-state loops
// (src/chebyshev_solver.cpp:86-199), including accumulation onto the table passed in.
#ifndef CHEBYSHEV_SOLVER
#define CHEBYSHEV_SOLVER

#include <algorithm>
#include <array>
#include <cassert>
#include <complex>
#include <fstream>
#include <limits>
#include <numeric>
#include <vector>

#include "chebyshev_moments.hpp"
#include "kpm_noneqop.hpp"
#include "quantum_states.hpp"
#include "sparse_matrix.hpp"

namespace chebyshev {
typedef std::complex<double> value_t;
typedef std::vector<value_t> vector_t;

namespace utility {
// ./BOUNDS ("lowest highest"), else (-100, 100): src/chebyshev_solver.cpp:8-23
std::array<double, 2> SpectralBounds(SparseMatrixType &HAM);
}  // namespace utility

int CorrelationExpansionMoments(SparseMatrixType &OPL, SparseMatrixType &OPR, chebyshev::Moments2D &chebMoms,
                                qstates::generator &gen);

int SpectralMoments(SparseMatrixType &OP, chebyshev::Moments1D &chebMoms, qstates::generator &gen);

// SpectralMoments in a non-orthogonal basis (src/chebyshev_solver.cpp:203-229): every S^-1 a
// BiCGSTAB solve with the reference's settings (tolerance 1e-4, at most 2000 iterations) on
// the CSR arrays of S as stored, all states as one block (linqt_moments1d_nonorth)
int SpectralMoments_nonOrth(SparseMatrixType &OP, chebyshev::Moments1D_nonOrth &chebMoms, qstates::generator &gen);

// all states of the generator as one block through linqt_moments_td
int TimeDependentCorrelations(SparseMatrixType &OPL, SparseMatrixType &OPR, chebyshev::MomentsTD &chebMoms,
                              qstates::generator &gen);

}  // namespace chebyshev

#endif
