"""Pin the C restatement against the reference's own sources (oracle/_ref).

oracle/_ref holds LinQT's src/*.cpp compiled unmodified against stand-in MKL /
FFTW / Eigen headers, plus its CLI drivers and ref_harness (an in-process timing
harness).  These tests feed both the same seeded synthetic operators and states,
through the reference's own file formats, and compare the results.
"""
import os
import subprocess

import numpy as np
import pytest

from linqt_b200 import formats, lattices

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                                "ref_harness")),
                                reason="oracle/_ref not built (needs the reference checkout)")


def setup_dir(oracle_lib, tmp_path, label, ops, bounds, states):
    d = tmp_path
    (d / "operators").mkdir()
    for name, (n, csr) in ops.items():
        formats.write_csr(str(d / "operators" / ("%s.%s.CSR" % (label, name))), n, *csr)
    (d / "BOUNDS").write_text("%.17g %.17g\n" % bounds)
    formats.write_vector_states(str(d / "states.txt"), states)
    return str(d)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def test_spectral_moments_vs_ref(oracle_lib, tmp_path):
    N, H = lattices.square_lattice(16, t=1.0, W=1.0, seed=11)
    st = lattices.random_phase_states(N, 2, seed=12)
    lo, hi = -4.725, 4.725
    d = setup_dir(oracle_lib, tmp_path, "sq", {"HAM": (N, H)}, (lo, hi), st)
    out = oracle_lib.run_ref_harness(["spectral", "sq", "1", 64, "states.txt"], d)
    n, bw, bc, mu_ref = formats.read_chebmom1d(os.path.join(d, out["out"]))
    assert n == N and bw == hi - lo
    Ho = oracle_lib.Op(*formats.read_csr(os.path.join(d, "operators", "sq.HAM.CSR"))[1:])
    Ho.rescale(2 / bw, -bc / (bw / 2))
    st_file = formats.read_state_file(os.path.join(d, "states.txt"))
    mu = oracle_lib.moments1d(Ho, None, st_file, 64)
    assert rel(mu, mu_ref) < 1e-12


def test_correlation_moments_vs_ref(oracle_lib, tmp_path):
    N, H, V = lattices.honeycomb(6, 5, t=-2.7, W=1.0, seed=21)
    st = lattices.random_phase_states(N, 3, seed=22)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    d = setup_dir(oracle_lib, tmp_path, "gr", {"HAM": (N, H), "VX": (N, V)}, (1.05 * lo, 1.05 * hi), st)
    env = dict(os.environ)
    env.pop("BATCH_SIZE", None)
    out = oracle_lib.run_ref_harness(["nonEq", "gr", "VX", "VX", 40, "states.txt"], d)
    n, bw, bc, mu_ref = formats.read_chebmom2d(os.path.join(d, out["out"]))
    _, rp, cl, vl = formats.read_csr(os.path.join(d, "operators", "gr.HAM.CSR"))
    Ho = oracle_lib.Op(rp, cl, vl).rescale(2 / bw, -bc / (bw / 2))
    _, rp, cl, vl = formats.read_csr(os.path.join(d, "operators", "gr.VX.CSR"))
    Vo = oracle_lib.Op(rp, cl, vl)
    mu = oracle_lib.moments2d(Ho, Vo, Vo, formats.read_state_file(os.path.join(d, "states.txt")), 40)
    assert rel(mu, mu_ref) < 1e-12


@pytest.mark.parametrize("formula,nump", [(1, 64), (0, 64), (1, 50)])
def test_kubo_fft_vs_ref(oracle_lib, tmp_path, formula, nump):
    N, H, V = lattices.honeycomb(5, 4, t=-2.7, W=1.0, seed=21)
    st = lattices.random_phase_states(N, 2, seed=23)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    d = setup_dir(oracle_lib, tmp_path, "gr", {"HAM": (N, H), "VX": (N, V)}, (1.05 * lo, 1.05 * hi), st)
    M = 32
    out = oracle_lib.run_ref_harness(["kuboFFT", "gr", "VX", "VX", M, nump, formula, "states.txt"], d)
    ref = np.loadtxt(os.path.join(d, out["out"]))
    bw, bc = 1.05 * (hi - lo), 1.05 * (hi + lo) / 2
    _, rp, cl, vl = formats.read_csr(os.path.join(d, "operators", "gr.HAM.CSR"))
    Ho = oracle_lib.Op(rp, cl, vl).rescale(2 / bw, -bc / (bw / 2))
    _, rp, cl, vl = formats.read_csr(os.path.join(d, "operators", "gr.VX.CSR"))
    Vo = oracle_lib.Op(rp, cl, vl)
    E, s, integ, _ = oracle_lib.kubo_fft(Ho, Vo, Vo, formats.read_state_file(os.path.join(d, "states.txt")), M, nump,
                                         formula, N, bw, bc)
    # the reference prints with 6 significant digits
    assert np.abs(E - ref[:, 0]).max() < 1e-5 * np.abs(E).max()
    assert np.abs(s - ref[:, 1]).max() < 2e-6 * np.abs(s).max() + 1e-300
    if formula == 1:
        ri = np.loadtxt(os.path.join(d, out["out"] + "_integrand"))
        assert np.abs(integ - ri[:, 1]).max() < 2e-6 * np.abs(integ).max()


def test_reference_driver_on_golden_chain(tmp_path):
    """The reference's own inline_compute-kpm-nonEqOp, built here, reproduces the shipped table."""
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "linear_chain.npz"))
    (tmp_path / "operators").mkdir()
    for op in ("HAM", "VX"):
        rp, cl, vl = golden[op + "_rowptr"], golden[op + "_col"], golden[op + "_val"]
        formats.write_csr(str(tmp_path / "operators" / ("linear_chain.%s.CSR" % op)), len(rp) - 1, rp, cl,
                          vl[0::2] + 1j * vl[1::2])
    (tmp_path / "BOUNDS").write_text("-5 5\n")
    exe = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "inline_compute-kpm-nonEqOp")
    subprocess.run([exe, "linear_chain", "VX", "VX", "100"], cwd=str(tmp_path), check=True, capture_output=True)
    n, bw, bc, mu = formats.read_chebmom2d(str(tmp_path / "NonEqOpVX-VXlinear_chainKPM_M100x100_statedefault.chebmom2D"))
    ref = golden["mu100"][..., 0] + 1j * golden["mu100"][..., 1]
    assert rel(mu, ref) < 1e-13


def _graphene_with_diagonal(tmp_path, oracle_lib, R, seed):
    """Graphene with V_x and a second, diagonal operator DG, so that OPL != OPR."""
    N, H, V = lattices.honeycomb(6, 5, t=-2.7, W=1.0, seed=21)
    D = lattices.upper_csr(N, np.arange(N), np.arange(N), lattices.disorder(N, 2.0, 5) + 0j)
    st = lattices.random_phase_states(N, R, seed=seed)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    d = setup_dir(oracle_lib, tmp_path, "gr", {"HAM": (N, H), "VX": (N, V), "DG": (N, D)},
                  (1.05 * lo, 1.05 * hi), st)
    ops = {k: oracle_lib.Op(*formats.read_csr(os.path.join(d, "operators", "gr.%s.CSR" % k))[1:])
           for k in ("VX", "DG")}
    return N, d, ops, (1.05 * (hi - lo), 1.05 * (hi + lo) / 2)


def test_correlation_moments_operator_order_vs_ref(oracle_lib, tmp_path):
    """CorrelationExpansionMoments(OPL, OPR, ...) (src/chebyshev_solver.cpp:86): the first operator
    is OPL, the one the first moment index follows."""
    N, d, ops, _ = _graphene_with_diagonal(tmp_path, oracle_lib, 3, 22)
    out = oracle_lib.run_ref_harness(["nonEq", "gr", "VX", "DG", 40, "states.txt"], d)
    n, bw, bc, mu_ref = formats.read_chebmom2d(os.path.join(d, out["out"]))
    Ho = oracle_lib.Op(*formats.read_csr(os.path.join(d, "operators", "gr.HAM.CSR"))[1:]).rescale(2 / bw,
                                                                                                   -bc / (bw / 2))
    st = formats.read_state_file(os.path.join(d, "states.txt"))
    assert rel(oracle_lib.moments2d(Ho, ops["VX"], ops["DG"], st, 40), mu_ref) < 1e-12
    assert rel(oracle_lib.moments2d(Ho, ops["DG"], ops["VX"], st, 40), mu_ref) > 1e-3  # the order matters


@pytest.mark.parametrize("formula", [0, 1])
def test_kubo_fft_operator_order_vs_ref(oracle_lib, tmp_path, formula):
    """Kubo_solver_FFT::compute(OPL, OPR, gen) (src/Kubo_solver_FFT.cpp:12) with OPL != OPR."""
    N, d, ops, (bw, bc) = _graphene_with_diagonal(tmp_path, oracle_lib, 2, 23)
    M, nump = 32, 64
    out = oracle_lib.run_ref_harness(["kuboFFT", "gr", "VX", "DG", M, nump, formula, "states.txt"], d)
    ref = np.loadtxt(os.path.join(d, out["out"]))
    Ho = oracle_lib.Op(*formats.read_csr(os.path.join(d, "operators", "gr.HAM.CSR"))[1:]).rescale(2 / bw,
                                                                                                   -bc / (bw / 2))
    st = formats.read_state_file(os.path.join(d, "states.txt"))
    E, s, integ, _ = oracle_lib.kubo_fft(Ho, ops["VX"], ops["DG"], st, M, nump, formula, N, bw, bc)
    assert np.abs(s - ref[:, 1]).max() < 2e-6 * np.abs(s).max()


def test_time_correlations_vs_ref(oracle_lib, tmp_path):
    """TimeDependentCorrelations through the reference's own inline_compute-kpm-CorrOp
    (its default state, a delta at N/2, with OPL != OPR) against the C restatement."""
    N, d, ops, (bw, bc) = _graphene_with_diagonal(tmp_path, oracle_lib, 1, 3)
    M, NT, tmax = 32, 5, 10.0
    exe = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "inline_compute-kpm-CorrOp")
    subprocess.run([exe, "gr", "VX", "DG", str(M), str(NT), str(tmax)], cwd=d, check=True, capture_output=True,
                   timeout=600)
    n, bw_f, bc_f, dt, mu_ref = formats.read_chebmomtd(os.path.join(d, "TimeCorrVX-DGgrKPM_M%d_statedefault.chebmomTD"
                                                                    % M))
    assert n == N and mu_ref.shape == (M, NT) and abs(dt - tmax / (NT - 1)) < 1e-14
    lo, hi = [float(x) for x in open(os.path.join(d, "BOUNDS")).read().split()]
    bw, bc = hi - lo, (hi + lo) / 2
    Ho = oracle_lib.Op(*formats.read_csr(os.path.join(d, "operators", "gr.HAM.CSR"))[1:])
    Ho.rescale(2 / bw, -bc / (bw / 2))
    delta = np.zeros((1, N), np.complex128)
    delta[0, N // 2] = 1.0
    mu = oracle_lib.moments_td(Ho, ops["VX"], ops["DG"], delta, M, NT, tmax / (NT - 1), bw, bc)
    assert rel(mu, mu_ref) < 1e-12


def test_time_correlation_postprocessor_vs_ref(oracle_lib, tmp_path):
    """timeCorrelationsFromChebmom built from the reference's sources against the C
    restatement, on a TD table the restatement computed (6 printed digits)."""
    N, H, V = lattices.honeycomb(6, 5, t=-2.7, W=1.0, seed=21)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), 1.05 * (hi + lo) / 2
    Ho = oracle_lib.Op(*H)
    Ho.rescale(2 / bw, -bc / (bw / 2))
    st = lattices.random_phase_states(N, 2, seed=8)
    M, NT, dt = 96, 7, 1.5
    mu = oracle_lib.moments_td(Ho, oracle_lib.Op(*V), oracle_lib.Op(*V), st, M, NT, dt, bw, bc)
    formats.write_chebmomtd(str(tmp_path / "tdchain.chebmomTD"), N, bw, bc, dt, mu)
    exe = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "inline_timeCorrelationsFromChebmom")
    for broad, ef in ((200.0, 0.5), (60.0, -1.25)):
        subprocess.run([exe, "tdchain.chebmomTD", str(broad), str(ef)], cwd=str(tmp_path), check=True,
                       capture_output=True, timeout=600)
        ref = np.loadtxt(str(tmp_path / ("meantdchainEF%.6fJACKSON.dat" % ef)))
        mu_f = formats.read_chebmomtd(str(tmp_path / "tdchain.chebmomTD"))[4]
        t, c = oracle_lib.time_correlation(mu_f, N, bw, bc, dt, broad, ef)
        assert np.abs(t - ref[:, 0]).max() < 1e-5 * max(1.0, np.abs(t).max())
        assert np.abs(c - ref[:, 1]).max() < 2e-6 * np.abs(c).max()


def _nonorth_dir(oracle_lib, tmp_path, L=8, R=2):
    N, H = lattices.square_lattice(L, t=1.0, W=1.0, seed=11)
    S = lattices.overlap_matrix(N, H, s=0.08, seed=13)
    st = lattices.random_phase_states(N, R, seed=12)
    d = setup_dir(oracle_lib, tmp_path, "sq", {"HAM": (N, H), "S": (N, S)}, (-4.725, 4.725), st)
    return d, N


@pytest.mark.parametrize("opname", ["1", "HAM"])
def test_nonorth_moments_vs_reference_driver(oracle_lib, tmp_path, opname):
    """SpectralMoments_nonOrth: LinQT's own inline_compute-kpm-spectralOp-nonOrth (its Eigen
    BiCGSTAB solve of S x = b given by the stand-in, tolerance 1e-4) against the restatement,
    both on the stored upper triangle of S."""
    d, N = _nonorth_dir(oracle_lib, tmp_path)
    exe = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "inline_compute-kpm-spectralOp-nonOrth")
    M = 48
    p = subprocess.run([exe, "sq", opname, str(M), "states.txt"], cwd=d, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-500:]
    out = [f for f in os.listdir(d) if f.endswith(".chebmom1D-nonOrth")]
    assert len(out) == 1
    n, bw, bc, mu_ref = formats.read_chebmom1d(os.path.join(d, out[0]))
    assert n == N and abs(bw - 9.45) < 1e-12
    iters_ref = [int(l.split()[1]) for l in p.stdout.splitlines() if l.startswith("#iterations:")]
    _, rp, cl, vl = formats.read_csr(os.path.join(d, "operators", "sq.HAM.CSR"))
    Ho = oracle_lib.Op(rp, cl, vl).rescale(2 / bw, -bc / (bw / 2))
    OPo = oracle_lib.Op(rp, cl, vl) if opname == "HAM" else None  # the operator file, not rescaled
    S = formats.read_csr(os.path.join(d, "operators", "sq.S.CSR"))[1:]
    mu, its = oracle_lib.moments1d_nonorth(Ho, OPo, S, formats.read_state_file(os.path.join(d, "states.txt")), M)
    # per state the reference solves twice to start and once after every moment; the solves
    # after moments M-2 and M-1 (T_M, T_{M+1}) never reach mu and the restatement skips them
    assert len(iters_ref) == 2 * (M + 2)
    assert its == sum(iters_ref) - sum(iters_ref[(M + 2) * k + M] + iters_ref[(M + 2) * k + M + 1] for k in range(2))
    assert rel(mu, mu_ref) < 1e-12
