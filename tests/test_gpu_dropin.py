"""Drop-in check: LinQT's own driver programs (src/inline_compute-kpm-spectralOp.cpp,
inline_compute-kpm-nonEqOp.cpp, inline_compute-Kubo-kpm-FFT.cpp), compiled unchanged against
the C++ facade (linqt_b200/facade) and so running on the GPU library, write the same files as
the same programs built from the reference's sources on the CPU (oracle/_ref); also
inline_compute-kpm-CorrOp (time-domain correlations).

Inputs: the golden linear chain (N = 20000, upper-triangle CSR), a second diagonal operator
DG so that OPL != OPR, ./BOUNDS, and either the default state (delta at N/2) or a `vector`
state file with three random-phase states."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from linqt_b200 import formats, lattices

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FACADE = os.path.join(ROOT, "linqt_b200", "facade", "_drivers")
REFBIN = os.path.join(ROOT, "oracle", "_ref")
DRIVERS = ["inline_compute-kpm-spectralOp", "inline_compute-kpm-nonEqOp", "inline_compute-Kubo-kpm-FFT",
           "inline_compute-kpm-CorrOp"]


def _need(path):
    if not os.path.exists(path):
        pytest.skip("%s not built (needs the reference checkout at build time)" % os.path.relpath(path, ROOT))


@pytest.fixture(scope="module")
def workdir(tmp_path_factory):
    golden = np.load(os.path.join(HERE, "golden", "linear_chain.npz"))
    d = tmp_path_factory.mktemp("dropin")
    (d / "operators").mkdir()
    N = 0
    for op in ("HAM", "VX"):
        rp, cl, vl = golden[op + "_rowptr"], golden[op + "_col"], golden[op + "_val"]
        N = len(rp) - 1
        formats.write_csr(str(d / "operators" / ("linear_chain.%s.CSR" % op)), N, rp, cl, vl[0::2] + 1j * vl[1::2])
    D = lattices.upper_csr(N, np.arange(N), np.arange(N), lattices.disorder(N, 1.0, 7) + 0j)
    formats.write_csr(str(d / "operators" / "linear_chain.DG.CSR"), N, *D)
    (d / "BOUNDS").write_text("-5 5\n")
    formats.write_vector_states(str(d / "states.txt"), lattices.random_phase_states(N, 3, seed=77))
    return d


def _run(exe, args, src, dst):
    shutil.copytree(src, dst)
    p = subprocess.run([exe] + [str(a) for a in args], cwd=dst, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return dst


def _both(name, args, workdir, tmp_path):
    _need(os.path.join(FACADE, name))
    _need(os.path.join(REFBIN, name))
    gpu = _run(os.path.join(FACADE, name), args, workdir, tmp_path / "gpu")
    cpu = _run(os.path.join(REFBIN, name), args, workdir, tmp_path / "cpu")
    new_gpu = sorted(set(os.listdir(gpu)) - set(os.listdir(workdir)))
    new_cpu = sorted(set(os.listdir(cpu)) - set(os.listdir(workdir)))
    assert new_gpu == new_cpu and new_gpu, (new_gpu, new_cpu)  # same output files, same names
    return gpu, cpu, new_gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("op,state", [("1", None), ("VX", "states.txt"), ("DG", "states.txt")])
def test_spectral_driver(workdir, tmp_path, op, state):
    args = ["linear_chain", op, 256] + ([state] if state else [])
    gpu, cpu, files = _both("inline_compute-kpm-spectralOp", args, workdir, tmp_path)
    (f,) = files
    n1, bw1, bc1, mu1 = formats.read_chebmom1d(str(gpu / f))
    n2, bw2, bc2, mu2 = formats.read_chebmom1d(str(cpu / f))
    assert (n1, bw1, bc1) == (n2, bw2, bc2)
    assert _rel(mu1, mu2) < 1e-12  # 15 printed digits


@pytest.mark.parametrize("opr,opl,M,state", [("VX", "VX", 100, None), ("VX", "DG", 64, "states.txt"),
                                             ("DG", "VX", 48, "states.txt")])
def test_correlation_driver(workdir, tmp_path, opr, opl, M, state):
    args = ["linear_chain", opr, opl, M] + ([state] if state else [])
    gpu, cpu, files = _both("inline_compute-kpm-nonEqOp", args, workdir, tmp_path)
    (f,) = files
    n1, bw1, bc1, mu1 = formats.read_chebmom2d(str(gpu / f))
    n2, bw2, bc2, mu2 = formats.read_chebmom2d(str(cpu / f))
    assert (n1, bw1, bc1) == (n2, bw2, bc2) and mu1.shape == mu2.shape == (M, M)
    assert _rel(mu1, mu2) < 1e-12
    if M == 100 and state is None:  # the table shipped with LinQT
        g = np.load(os.path.join(HERE, "golden", "linear_chain.npz"))["mu100"]
        assert _rel(mu1, g[..., 0] + 1j * g[..., 1]) < 1e-13


@pytest.mark.parametrize("opr,opl", [("VX", "VX"), ("VX", "DG")])
def test_kubo_fft_driver(workdir, tmp_path, opr, opl):
    args = ["linear_chain", opr, opl, 64, "states.txt"]
    gpu, cpu, files = _both("inline_compute-Kubo-kpm-FFT", args, workdir, tmp_path)
    (f,) = files
    a, b = np.loadtxt(str(gpu / f)), np.loadtxt(str(cpu / f))
    assert a.shape == b.shape
    # both write 6 significant digits (default stream precision)
    assert np.abs(a[:, 0] - b[:, 0]).max() <= 1e-5 * np.abs(b[:, 0]).max()
    assert np.abs(a[:, 1] - b[:, 1]).max() <= 2e-6 * np.abs(b[:, 1]).max()


@pytest.mark.parametrize("opl,opr,M,NT,tmax", [("VX", "VX", 64, 6, 20.0), ("VX", "DG", 48, 4, 6.0)])
def test_time_correlation_driver(workdir, tmp_path, opl, opr, M, NT, tmax):
    """inline_compute-kpm-CorrOp (its default state, a delta at N/2): the .chebmomTD tables."""
    args = ["linear_chain", opl, opr, M, NT, tmax]
    gpu, cpu, files = _both("inline_compute-kpm-CorrOp", args, workdir, tmp_path)
    (f,) = files
    n1, bw1, bc1, dt1, mu1 = formats.read_chebmomtd(str(gpu / f))
    n2, bw2, bc2, dt2, mu2 = formats.read_chebmomtd(str(cpu / f))
    assert (n1, bw1, bc1, dt1) == (n2, bw2, bc2, dt2) and mu1.shape == mu2.shape == (M, NT)
    assert _rel(mu1, mu2) < 1e-12  # 15 printed digits


@pytest.fixture(scope="module")
def nonorth_dir(tmp_path_factory):
    """A square lattice (16 x 16) with an overlap matrix S on its bonds, for
    inline_compute-kpm-spectralOp-nonOrth (operators/sq.{HAM,S}.CSR, BOUNDS, states)."""
    d = tmp_path_factory.mktemp("dropin_nonorth")
    (d / "operators").mkdir()
    N, H = lattices.square_lattice(16, t=1.0, W=1.0, seed=11)
    S = lattices.overlap_matrix(N, H, s=0.08, seed=13)
    formats.write_csr(str(d / "operators" / "sq.HAM.CSR"), N, *H)
    formats.write_csr(str(d / "operators" / "sq.S.CSR"), N, *S)
    (d / "BOUNDS").write_text("-4.725 4.725\n")
    formats.write_vector_states(str(d / "states.txt"), lattices.random_phase_states(N, 3, seed=12))
    return d


@pytest.mark.parametrize("op,state", [("1", "states.txt"), ("HAM", "states.txt"), ("1", None)])
def test_nonorth_spectral_driver(nonorth_dir, tmp_path, op, state):
    """inline_compute-kpm-spectralOp-nonOrth: S^-1 by BiCGSTAB (the reference through its Eigen
    stand-in, the facade on the GPU), the same .chebmom1D-nonOrth file."""
    args = ["sq", op, 96] + ([state] if state else [])
    gpu, cpu, files = _both("inline_compute-kpm-spectralOp-nonOrth", args, nonorth_dir, tmp_path)
    (f,) = files
    n1, bw1, bc1, mu1 = formats.read_chebmom1d(str(gpu / f))
    n2, bw2, bc2, mu2 = formats.read_chebmom1d(str(cpu / f))
    assert (n1, bw1, bc1) == (n2, bw2, bc2)
    assert _rel(mu1, mu2) < 1e-11
