// ref_harness -- times the reference's own solvers in-process (TEST / BASELINE
// INFRASTRUCTURE ONLY).  It links oracle/_ref/libkpm_ref.a (the reference's
// src/*.cpp built against the stand-ins) and mirrors what the reference drivers
// do (src/inline_compute-kpm-spectralOp.cpp:32-84, src/inline_compute-kpm-nonEqOp.cpp:39-187,
// src/inline_compute-Kubo-kpm-FFT.cpp:39-291): operators from operators/<LABEL>.<ID>.CSR,
// bounds from ./BOUNDS, states from a `vector` state file.  Only the solver call is
// timed; one JSON line is printed on stdout.
//
//   ref_harness spectral LABEL OP M STATEFILE
//   ref_harness nonEq    LABEL OPR OPL M STATEFILE
//   ref_harness kuboFFT  LABEL OPR OPL M NUMP FORMULA(0=Greenwood,1=Bastin) STATEFILE
//   ref_harness frommom  II|Sea FILE.chebmom2D BROADENING XBOUND NUM_DIV(0 = 30 M)
#include <omp.h>

#include <chrono>
#include <cstdio>
#include <fstream>
#include <vector>
#include <cstdlib>
#include <iostream>
#include <string>

#include "Kubo_solver_FFT.hpp"
#include "chebyshev_moments.hpp"
#include "chebyshev_solver.hpp"
#include "quantum_states.hpp"
#include "sparse_matrix.hpp"

static void load(SparseMatrixType &op, const std::string &label, const std::string &id) {
  op.SetID(id);
  if (op.isIdentity()) return;
  SparseMatrixBuilder builder;
  builder.setSparseMatrix(&op);
  builder.BuildOPFromCSRFile("operators/" + label + "." + id + ".CSR");
}

static void report(const char *mode, double seconds, const std::string &out) {
  std::printf("{\"mode\": \"%s\", \"seconds\": %.9f, \"threads\": %d, \"out\": \"%s\"}\n", mode, seconds,
              omp_get_max_threads(), out.c_str());
}

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: ref_harness spectral|nonEq|kuboFFT ...\n");
    return 2;
  }
  const std::string mode = argv[1];
  typedef std::chrono::steady_clock clk;
  if (mode == "spectral" && argc == 6) {
    const std::string label = argv[2], sop = argv[3];
    const int M = std::atoi(argv[4]);
    chebyshev::Moments1D mom(M);
    SparseMatrixType OP[2];
    load(OP[0], label, "HAM");
    load(OP[1], label, sop);
    std::array<double, 2> b = chebyshev::utility::SpectralBounds(OP[0]);
    mom.SystemLabel(label);
    mom.BandWidth(b[1] - b[0]);
    mom.BandCenter((b[1] + b[0]) * 0.5);
    mom.SetAndRescaleHamiltonian(OP[0]);
    qstates::generator gen = qstates::LoadStateFile(argv[5]);
    const auto t0 = clk::now();
    chebyshev::SpectralMoments(OP[1], mom, gen);
    const double dt = std::chrono::duration<double>(clk::now() - t0).count();
    const std::string out = "ref_spectral.chebmom1D";
    mom.saveIn(out);
    report("spectral", dt, out);
    return 0;
  }
  if (mode == "nonEq" && argc == 7) {
    const std::string label = argv[2], sopr = argv[3], sopl = argv[4];
    const int M = std::atoi(argv[5]);
    chebyshev::Moments2D mom(M, M);
    SparseMatrixType OP[3];
    load(OP[0], label, "HAM");
    load(OP[1], label, sopr);
    load(OP[2], label, sopl);
    std::array<double, 2> b = chebyshev::utility::SpectralBounds(OP[0]);
    mom.SystemLabel(label);
    mom.BandWidth(b[1] - b[0]);
    mom.BandCenter((b[1] + b[0]) * 0.5);
    mom.SetAndRescaleHamiltonian(OP[0]);
    qstates::generator gen = qstates::LoadStateFile(argv[6]);
    const auto t0 = clk::now();
    chebyshev::CorrelationExpansionMoments(OP[1], OP[2], mom, gen);
    const double dt = std::chrono::duration<double>(clk::now() - t0).count();
    const std::string out = "ref_nonEq.chebmom2D";
    mom.saveIn(out);
    report("nonEq", dt, out);
    return 0;
  }
  if (mode == "kuboFFT" && argc == 9) {
    const std::string label = argv[2], sopr = argv[3], sopl = argv[4];
    const int M = std::atoi(argv[5]), nump = std::atoi(argv[6]), formula = std::atoi(argv[7]);
    chebyshev::Vectors_sliced vec(M, 1);
    SparseMatrixType OP[3];
    load(OP[0], label, "HAM");
    load(OP[1], label, sopr);
    load(OP[2], label, sopl);
    std::array<double, 2> b = chebyshev::utility::SpectralBounds(OP[0]);
    vec.SystemLabel(label);
    vec.BandWidth(b[1] - b[0]);
    vec.BandCenter((b[1] + b[0]) * 0.5);
    vec.SetAndRescaleHamiltonian(OP[0]);
    qstates::generator gen = qstates::LoadStateFile(argv[8]);
    std::string out = "ref_kuboFFT.conductivity";
    chebyshev::Kubo_solver_FFT solver(M, 1, nump, formula == 1 ? chebyshev::KUBO_BASTIN : chebyshev::KUBO_GREENWOOD,
                                      vec, out);
    const auto t0 = clk::now();
    solver.compute(OP[1], OP[2], gen);
    const double dt = std::chrono::duration<double>(clk::now() - t0).count();
    report("kuboFFT", dt, out);
    return 0;
  }
  if (mode == "frommom" && argc == 7) {
    // The energy sums of kuboBastinIIFromChebmom.cpp:62-88 / kuboBastinSeaFromChebmom.cpp:
    // 62-88 on a uniform grid of the given half width (the drivers fix it at CUTOFF = 1,
    // where the first point divides by zero), with the reference's own Moments2D reader,
    // Jackson kernel and chebyshev_coefficients.hpp functions.
    const std::string variant = argv[2];
    chebyshev::Moments2D mu(argv[3]);
    const double broad = std::atof(argv[4]), xbound = std::atof(argv[5]);
    mu.ApplyJacksonKernel(broad, broad);
    const int num_div = std::atoi(argv[6]) > 0 ? std::atoi(argv[6]) : 30 * mu.HighestMomentNumber();
    std::vector<double> en(num_div), kernel(num_div, 0.0);
    for (int i = 0; i < num_div; i++) en[i] = -xbound + i * (2 * xbound) / (num_div - 1);
    const double w = mu.SystemSize() / mu.HalfWidth() / mu.HalfWidth() / 2 / M_PI;
    for (int i = 0; i < num_div; i++) {
      double out = 0.0;
      const double x = en[i];
      for (int m0 = 0; m0 < mu.HighestMomentNumber(0); m0++)
        for (int m1 = 0; m1 < mu.HighestMomentNumber(1); m1++) {
          if (variant == "II") {
            out += -((greenR_chebF(x, m0) * DgreenR_chebF(x, m1) - DgreenR_chebF(x, m0) * greenR_chebF(x, m1)) *
                     mu(m0, m1)).real();
          } else {
            const auto Gr = greenR_chebF(x, m0);
            const auto Ga = std::conj(greenR_chebF(x, m0));
            const auto DGr = DgreenR_chebF(x, m1).real();
            const auto DGa = std::conj(DGr);
            out += -((Gr - Ga) * (DGr + DGa) * mu(m0, m1)).real();
          }
        }
      kernel[i] = out * w;
    }
    std::ofstream f("ref_frommom.dat");
    f.precision(17);
    double acc = 0;
    for (int i = 0; i < num_div - 1; i++) {
      const double de = en[i + 1] - en[i];
      acc += (variant == "II" ? 1.0 : 0.5) * (kernel[i] + kernel[i + 1]) * de;
      f << en[i] * mu.HalfWidth() + mu.BandCenter() << " " << acc << "\n";
    }
    report("frommom", 0.0, "ref_frommom.dat");
    return 0;
  }
  std::fprintf(stderr, "bad arguments\n");
  return 2;
}
