// wannier2sparse on the GPU library: the command line of LinQT's utilities/wannier2sparse
// (src/main.cpp, include/w2sp_arguments.hpp) with the supercell operators assembled on the
// device (linqt_supercell_write_csr).
//
//   wannier2sparse LABEL Dim0 Dim1 Dim2 [all | OP ...]
//
// reads LABEL.xyz, LABEL.uc and LABEL_hr.dat and writes LABEL.HAM.CSR plus LABEL.OP.CSR for
// every operator asked for ("all": the 18 of include/operator_utils.hpp:31-35), the same
// bytes the reference writes.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "linqt_gpu.h"

static const char *kAll[] = {"VX",   "VY",   "VZ",   "VXSX", "VXSY", "VXSZ", "VYSX", "VYSY", "VYSZ",
                             "VZSX", "VZSY", "VZSZ", "SX",   "SY",   "SZ",   "TX",   "TY",   "TZ"};

static int usage(const char *prog) {
  std::fprintf(stderr,
               "usage: %s LABEL Dim0 Dim1 Dim2 [all | OP ...]\n"
               "  reads LABEL.xyz, LABEL.uc, LABEL_hr.dat; writes LABEL.HAM.CSR and LABEL.OP.CSR per operator\n"
               "  OP: VX VY VZ, V{X,Y,Z}S{X,Y,Z}, SX SY SZ, TX TY TZ, or NAME with a NAME.OP file\n",
               prog);
  return 1;
}

static int check(int rc, const std::string &what) {
  if (rc != LINQT_OK) {
    std::fprintf(stderr, "wannier2sparse: %s failed: %s\n", what.c_str(), linqt_last_error());
    std::exit(1);
  }
  return rc;
}

int main(int argc, char **argv) {
  if (argc < 2 || std::string(argv[1]) == "help") return usage(argv[0]);
  if (argc < 5) return usage(argv[0]);
  const std::string label = argv[1];
  int dims[3];
  for (int i = 0; i < 3; ++i) {
    char *end = nullptr;
    dims[i] = (int)std::strtol(argv[2 + i], &end, 10);
    if (!end || *end || dims[i] <= 0) return usage(argv[0]);
  }
  std::vector<std::string> ops;
  for (int i = 5; i < argc; ++i) {
    if (std::string(argv[i]) == "all")
      for (const char *o : kAll) ops.push_back(o);
    else
      ops.push_back(argv[i]);
  }
  linqt_tbmodel *m = nullptr;
  check(linqt_tbmodel_load(label.c_str(), &m), "reading " + label);
  std::printf("Creating Hamiltonian\n");
  check(linqt_supercell_write_csr(nullptr, m, "HAM", dims, (label + ".HAM.CSR").c_str()), "HAM");
  for (const auto &op : ops) {
    std::printf("Creating %s\n", op.c_str());
    check(linqt_supercell_write_csr(nullptr, m, op.c_str(), dims, (label + "." + op + ".CSR").c_str()), op);
  }
  linqt_tbmodel_destroy(m);
  return 0;
}
