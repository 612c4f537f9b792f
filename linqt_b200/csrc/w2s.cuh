// Operator builder: LinQT's utilities/wannier2sparse (Wannier90 model -> supercell CSR).
//
// Host side (tbmodel.cu): the model files, the unit-cell operator lists in the order the
// reference iterates them, and the supercell plan -- per orbital, the distinct matrix
// entries of a row ("keys") with their values already summed.  Device side
// (supercell.cu): the rows of the supercell written straight from the plan.
#pragma once

#include <array>
#include <complex>
#include <string>
#include <vector>

#include "internal.cuh"

namespace linqt {
namespace w2s {

using cplx = std::complex<double>;

// one hopping <e0, cell 0| O |e1, cell R> of a unit-cell list
struct Hop {
  std::array<int, 3> cell;
  int e0, e1;
  cplx v;
};

struct Model {
  int num_wann = 0;
  double lat[3][3] = {};
  std::vector<std::string> labels;
  std::vector<std::array<double, 3>> pos;
  std::vector<Hop> hops;  // the Hamiltonian, in the reference's iteration order
};

Model load_model(const std::string &label);
// unit-cell list of an operator (HAM, the 18 names of include/operator_utils.hpp:31-35, or
// a spinorial NAME.OP file in the working directory), in the reference's iteration order
std::vector<Hop> operator_list(const Model &m, const std::string &op);
bool is_builtin_op(const std::string &op);  // HAM or one of the 18 names

// A row of the supercell is (cell s, orbital g).  Its entries are the keys of group g: the
// distinct (R mod dims, target orbital o1) of g's hoppings.  Column of key (a, b, c, o1) in
// cell s = (sx, sy, sz): cell ((sz + a) mod Dz, (sy + b) mod Dy, (sx + c) mod Dx), orbital o1.
// Keys are sorted by (a, b, c, o1); in a given row the column order is that order rotated
// level by level (z, then y inside a z value, then x), the values >= D - s of each level
// coming first.  The tree below gives, for each level, the runs of equal a / b / c:
//   val   the run's value (a, b or c)
//   pre   keys before the run inside its parent (group, z run or y run)
//   size  keys in the run
//   c0    first child run (next level) or, on the x level, the first key
//   nc    number of child runs
//   par   parent: the group (z runs), the z run (y runs) or the y run (x runs)
struct Node {
  int val, pre, size, c0, nc, par;
};

struct Plan {
  int wbb = 0;
  int dims[3] = {1, 1, 1};
  long ncells = 0;
  long n = 0;  // rows = ncells * wbb
  std::vector<int> grp_key0;  // [wbb + 1] key ranges of the groups
  std::vector<int> grp_z0;    // [wbb + 1] z-run ranges of the groups
  std::vector<Node> zn, yn, xn;
  // per key: its z, y, x runs, index inside the x run, target orbital, group
  std::vector<int> kz, ky, kx, kleaf, ko1, kgrp;
  std::vector<double2> kval;
  std::vector<int4> kpack;  // per key {z run, y run, x run, index in the x run}
  std::vector<int> kgo;     // per key group << 16 | target orbital
  int keys() const { return (int)ko1.size(); }
};

Plan make_plan(const std::vector<Hop> &uc, int wbb, const int dims[3]);

// text of a CSR file as hopping_list.cpp:260-282 writes it (std::ostream defaults)
void write_csr_text(const std::string &path, long n, const std::vector<int> &rowptr, const std::vector<int> &col,
                    const std::vector<double2> &val);

}  // namespace w2s
}  // namespace linqt
