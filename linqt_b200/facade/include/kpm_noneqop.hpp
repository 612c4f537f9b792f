// Console helpers of LinQT's drivers (include/kpm_noneqop.hpp of LinQT): usage text and
// the BATCH_SIZE environment variable.  The B200 solvers do not batch moments, so
// GetBatchSize only reports the variable.
#ifndef KPM_NONEQ_HELPER
#define KPM_NONEQ_HELPER

#include <cstdlib>
#include <iostream>

namespace chebyshev {

inline void printHelpMessage() {
  std::cout << "Arguments: Label Op1 Op2 numMom [state file]" << std::endl
            << "  operators are read from operators/Label.<Op>.CSR, the energy bounds from ./BOUNDS" << std::endl;
}

inline void printWelcomeMessage() {
  std::cout << "Chebyshev expansion of a correlation function on the GPU (linqt_b200)" << std::endl;
}

inline bool GetBatchSize(int &batchSize) {
  const char *v = getenv("BATCH_SIZE");
  if (v && atoi(v) > 0) {
    batchSize = atoi(v);
    return true;
  }
  batchSize = 3;
  return false;
}

}  // namespace chebyshev

#endif
