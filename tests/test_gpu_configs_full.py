"""Parity at the benchmark configurations themselves, not only on small lattices.

  config 1: plain DOS, square lattice L = 256 (N = 65,536), Anderson W = 1 (seed 11), one
            random-phase vector (seed 12), M = 1024 moments, bounds +-1.05 (4 + 0.5), and the
            DOS of spectralFunctionFromChebmom_FFTgrid at 1024 energies;
  config 2: Kubo-Bastin sigma_xx(E) on honeycomb graphene 128 x 128 cells (N = 32,768),
            t = -2.7 eV, W = 1 eV (seed 21), V_x, M = 512, nump = 1024, the first of the eight
            random-phase vectors (seed 22) of the benchmark.

The GPU results are compared with the reference's own solvers built from its sources
(oracle/_ref/ref_harness: SpectralMoments, CorrelationExpansionMoments and Kubo_solver_FFT,
which write the moment tables with 15 digits and sigma with 6) and with the C restatement
(1e-10 for FP64).  The mixed-precision solve is checked against FP64 at the bounds DESIGN
states for it (moments 1e-7, sigma 1e-6 of the maximum)."""
import os

import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import formats, lattices

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


def ref_or_skip(oracle_lib):
    if not oracle_lib.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference checkout at build time)")


def test_config1_square_256_dos_full_size(oracle_lib, tmp_path):
    ref_or_skip(oracle_lib)
    N, H = lattices.square_lattice(256, t=1.0, W=1.0, seed=11)
    st = lattices.random_phase_states(N, 1, seed=12)
    lo, hi = -1.05 * 4.5, 1.05 * 4.5
    bw, bc = hi - lo, 0.0
    M = 1024
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    mu = lq.moments1d(Hg, None, st, M)
    # the reference's SpectralMoments on the same files (15 printed digits)
    (tmp_path / "operators").mkdir()
    formats.write_csr(str(tmp_path / "operators" / "sq.HAM.CSR"), N, *H)
    (tmp_path / "BOUNDS").write_text("%.17g %.17g\n" % (lo, hi))
    formats.write_vector_states(str(tmp_path / "st.txt"), st)
    out = oracle_lib.run_ref_harness(["spectral", "sq", "1", M, "st.txt"], str(tmp_path))
    n, bw_r, bc_r, mu_ref = formats.read_chebmom1d(os.path.join(str(tmp_path), out["out"]))
    assert n == N and abs(bw_r - bw) <= 1e-14 * bw  # the file prints 15 digits
    assert rel(mu, mu_ref) < 1e-12
    # the C restatement at full precision
    Ho = oracle_lib.Op(*H).rescale(2 / bw, -bc / (bw / 2))
    mu_o = oracle_lib.moments1d(Ho, None, st, M)
    assert rel(mu, mu_o) < 1e-10
    # the DOS on 1024 energies (FFT grid), as spectralFunctionFromChebmom_FFTgrid computes it
    E, dos = lq.spectral_function_from_moments(mu, N, bw, bc, 1.0, grid=lq.GRID_CHEBYSHEV)
    muj = oracle_lib.jackson1d(mu_o, bw, 1.0)
    Eo, doso = oracle_lib.spectral_function(muj, N, bw, bc, grid=1)
    assert len(E) == 1024 and np.array_equal(np.isfinite(dos), np.isfinite(doso))
    assert rel(E, Eo) < 1e-14 and rel(dos, doso) < 1e-10
    # the DOS integrates to N (algebraic check, trapezoid on the Chebyshev grid)
    order = np.argsort(E)
    assert abs(np.trapezoid(dos[order], E[order]) / N - 1) < 2e-2


@pytest.fixture(scope="module")
def graphene128(oracle_lib, tmp_path_factory):
    ref_or_skip(oracle_lib)
    N, H, V = lattices.honeycomb(128, 128, t=-2.7, W=1.0, seed=21, a=1.42)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    st = lattices.random_phase_states(N, 8, seed=22)[:1]
    d = tmp_path_factory.mktemp("graphene128")
    (d / "operators").mkdir()
    formats.write_csr(str(d / "operators" / "gr.HAM.CSR"), N, *H)
    formats.write_csr(str(d / "operators" / "gr.VX.CSR"), N, *V)
    (d / "BOUNDS").write_text("%.17g %.17g\n" % (bc - bw / 2, bc + bw / 2))
    formats.write_vector_states(str(d / "st.txt"), st)
    M, nump = 512, 1024
    a = oracle_lib.run_ref_harness(["nonEq", "gr", "VX", "VX", M, "st.txt"], str(d))
    b = oracle_lib.run_ref_harness(["kuboFFT", "gr", "VX", "VX", M, nump, 1, "st.txt"], str(d))
    _, _, _, mu_ref = formats.read_chebmom2d(os.path.join(str(d), a["out"]))
    sig_ref = np.loadtxt(os.path.join(str(d), b["out"]))
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    Vg = lq.Operator.from_csr(N, *V)
    return dict(N=N, H=H, V=V, bw=bw, bc=bc, st=st, M=M, nump=nump, mu_ref=mu_ref, sig_ref=sig_ref, Hg=Hg, Vg=Vg)


def test_config2_graphene_128_moments_and_sigma_vs_reference(graphene128):
    g = graphene128
    mu, (E, sig, integ) = lq.kubo_bastin(g["Hg"], g["Vg"], g["Vg"], g["st"], g["M"], g["nump"], g["bw"], g["bc"])
    assert mu.shape == (512, 512)
    assert rel(mu, g["mu_ref"]) < 1e-12  # the table is printed with 15 digits
    ref = g["sig_ref"]
    assert ref.shape == (g["nump"], 2)
    # the reference writes a E - b and sigma with 6 significant digits
    assert np.abs(E - ref[:, 0]).max() <= 1e-5 * np.abs(ref[:, 0]).max()
    lo, hi = int(0.05 * g["nump"]), int(0.95 * g["nump"])
    assert np.abs(sig - ref[:, 1])[lo:hi].max() <= 2e-6 * np.abs(ref[lo:hi, 1]).max()


def test_config2_sigma_vs_restatement_fp64(graphene128, oracle_lib):
    """sigma(E) at full precision against the C restatement of Kubo_solver_FFT (1e-10 over the
    interior 90 % of the window, where the Bastin integrand's 1/(1 - E^2)^2 stays bounded)."""
    g = graphene128
    _, (E, sig, integ) = lq.kubo_bastin(g["Hg"], g["Vg"], g["Vg"], g["st"], g["M"], g["nump"], g["bw"], g["bc"])
    Ho = oracle_lib.Op(*g["H"]).rescale(2 / g["bw"], -g["bc"] / (g["bw"] / 2))
    Vo = oracle_lib.Op(*g["V"])
    Eo, so, io, _ = oracle_lib.kubo_fft(Ho, Vo, Vo, g["st"], g["M"], g["nump"], 1, g["N"], g["bw"], g["bc"])
    lo, hi = int(0.05 * g["nump"]), int(0.95 * g["nump"])
    assert rel(E, Eo) < 1e-14
    assert np.abs(sig - so)[lo:hi].max() <= 1e-10 * np.abs(so[lo:hi]).max()
    assert np.abs(integ - io)[lo:hi].max() <= 1e-10 * np.abs(io[lo:hi]).max()


def test_config2_mixed_precision_at_its_stated_bound(graphene128):
    g = graphene128
    args = (g["Hg"], g["Vg"], g["Vg"], g["st"], g["M"], g["nump"], g["bw"], g["bc"])
    mu64, (_, s64, _) = lq.kubo_bastin(*args)
    mumx, (_, smx, _) = lq.kubo_bastin(*args, opts=lq.make_opts(precision=lq.PREC_MIXED))
    lo, hi = int(0.05 * g["nump"]), int(0.95 * g["nump"])
    e_mu = rel(mumx, mu64)
    e_s = float(np.abs(smx - s64)[lo:hi].max() / np.abs(s64[lo:hi]).max())
    assert 0 < e_mu < 1e-7  # measured 7e-9 at R = 8
    assert e_s < 1e-6
    assert rel(mumx, g["mu_ref"]) < 1e-7  # and against the reference's own table
