// LinQT's state generator (include/quantum_states.hpp of LinQT): the states a solver
// iterates over.  Behaviour kept from the reference:
//   * a default generator yields one state, the delta at dim/2 (quantum_states.hpp:85-93);
//   * LoadStateFile reads a "local" file (count, then site indices: delta states) or a
//     "vector" file (count, dim, then count*dim "re im" pairs); any other first word, or a
//     missing file, gives the default generator; the label is the file name.
// The B200 solvers read every state of a generator at once (qstates::collect_states).
#ifndef QUANTUM_STATES
#define QUANTUM_STATES

#include <cassert>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>
using namespace std;

enum StateType { LOCAL_STATE, USER_STATE, RANDOM_STATE };

typedef std::complex<double> Complex;
typedef std::vector<Complex> Vector;

namespace qstates {
typedef std::complex<double> scalar;

struct generator {
 public:
  generator() : label("default"), count(0), dim(0), num_states(1), kind(RANDOM_STATE) {}

  int SystemSize() const { return dim; }
  int NumberOfStates() const { return num_states; }
  void NumberOfStates(const int n) {
    num_states = n;
    spos.reserve(n);
  }
  void SystemSize(const int n) {
    if (SystemSize() == 0) {
      dim = n;
      out = std::vector<scalar>(dim);
      return;
    }
    assert(SystemSize() == n);
  }

  // next state into State(); false once all states were produced
  bool getQuantumState() {
    if (count >= NumberOfStates()) return false;
    if (kind == LOCAL_STATE) {
      std::fill(out.begin(), out.end(), scalar(0.0));
      out[spos[count]] = 1.0;
    } else if (kind == USER_STATE) {
      out.assign(data.begin() + spos[count], data.begin() + spos[count] + out.size());
    } else {
      std::fill(out.begin(), out.end(), scalar(0.0));
      out[dim / 2] = 1.0;
    }
    count++;
    return true;
  }

  std::string StateLabel() { return label; }
  std::vector<scalar> &State() { return out; }

  std::string label;
  int count;
  std::vector<scalar> out;
  std::vector<scalar> data;
  std::vector<int> spos;
  int dim;
  int num_states;
  StateType kind;
};

inline StateType String2State(std::string kind) {
  if (kind == "local") return LOCAL_STATE;
  if (kind == "vector") return USER_STATE;
  return RANDOM_STATE;
}

// A state file that ends early or holds something else than numbers: the reference reads on
// with zeros; here the program stops with a message.
inline void state_file_error(const std::string &what) {
  std::cerr << "ERROR: state file: " << what << std::endl;
  std::abort();
}

inline void readLocalState(std::ifstream &file, generator &g) {
  int n = 0;
  file >> n;
  if (!file || n < 0) state_file_error("malformed count of local states");
  g.NumberOfStates(n);
  for (int i = 0; i < n; i++) {
    int site = 0;
    file >> site;
    if (!file) state_file_error("truncated list of local states");
    g.spos.push_back(site);
  }
}

inline void readCustomState(std::ifstream &file, generator &g) {
  int n = 0, dim = 0;
  file >> n;
  g.NumberOfStates(n);
  file >> dim;
  if (!file || n < 0 || dim <= 0) state_file_error("malformed vector header (num_states dim)");
  g.SystemSize(dim);
  g.data.assign((size_t)dim * n, scalar(0.0));
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < dim; j++) {
      double re = 0, im = 0;
      file >> re >> im;
      if (!file) state_file_error("truncated vector states");
      g.data[(size_t)i * dim + j] = scalar(re, im);
    }
    g.spos.push_back(i * dim);
  }
}

inline generator CreateStateSet(std::ifstream &file, std::string kind) {
  generator g;
  g.kind = String2State(kind);
  if (g.kind == LOCAL_STATE) readLocalState(file, g);
  if (g.kind == USER_STATE) readCustomState(file, g);
  return g;
}

inline generator LoadStateFile(string filename) {
  std::ifstream infile(filename);
  std::string kind("random_phase");
  if (infile.good())
    infile >> kind;
  else
    std::cout << "State file not found, using default" << std::endl;
  generator g = CreateStateSet(infile, kind);
  g.label = filename;
  return g;
}

// All remaining states of a generator as one R x dim block (state-major); advances it.
inline std::vector<scalar> collect_states(generator &gen, int dim, int *R) {
  gen.SystemSize(dim);
  std::vector<scalar> block;
  int n = 0;
  while (gen.getQuantumState()) {
    block.insert(block.end(), gen.State().begin(), gen.State().end());
    n++;
  }
  *R = n;
  return block;
}

}  // namespace qstates
#endif
