"""Failure handling on the host (no GPU needed): malformed operators and files are rejected
with an error code, a Python exception or a stopped program, never read on as garbage.

The reference reads CSR and state files without checks (include/sparse_matrix.hpp:100-108,
src/sparse_matrix.cpp:3-50, include/quantum_states.hpp:135-228) and hands MKL whatever a
short file leaves in its arrays.  Here:
  - linqt_csr_create validates the CSR structure before it touches the device;
  - the Python readers (linqt_b200.formats) raise on truncated files;
  - the C++ facade stops LinQT's own driver programs with a message."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import formats, lattices

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FACADE = os.path.join(ROOT, "linqt_b200", "facade", "_drivers")


def _csr_error(n, rp, cl, vl):
    with pytest.raises(lq.LinqtError) as e:
        lq.Operator.from_csr(n, rp, cl, vl)
    return e.value


@pytest.mark.parametrize("bad", ["rowptr0", "decreasing", "col_high", "col_negative", "dim"])
def test_csr_create_rejects_malformed_structure(bad):
    N, (rp, cl, vl) = lattices.square_lattice(4, t=1.0, W=1.0, seed=11)
    rp, cl = rp.copy(), cl.copy()
    n = N
    if bad == "rowptr0":
        rp[0] = 1
    elif bad == "decreasing":
        rp[3] = rp[4] + 1
    elif bad == "col_high":
        cl[5] = N
    elif bad == "col_negative":
        cl[2] = -1
    else:
        n = 0
        rp = rp[:1]
    if bad == "dim":
        with pytest.raises((lq.LinqtError, ValueError)):
            lq.Operator.from_csr(n, rp, cl, vl)
        return
    err = _csr_error(n, rp, cl, vl)
    assert err.code == -1  # LINQT_ERR_INVALID, found before any device work


def test_solvers_reject_null_operators():
    L = lq.load()
    mu = np.zeros(16)
    st = np.zeros(2 * 8)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert L.linqt_moments1d(None, None, None, dp(st), 1, 8, None, dp(mu)) == -1
    assert L.linqt_moments2d(None, None, None, None, dp(st), 1, 8, None, dp(mu)) == -1
    assert L.linqt_moments1d_nonorth(None, None, None, None, dp(st), 1, 8, 1e-4, 10, None, dp(mu), None) == -1
    assert b"NULL" in L.linqt_last_error() or b"H" in L.linqt_last_error()


def _write_csr_truncated(path, keep):
    N, H = lattices.square_lattice(4, t=1.0, W=1.0, seed=11)
    formats.write_csr(path, N, *H)
    text = open(path).read()
    open(path, "w").write(text[: int(len(text) * keep)])


@pytest.mark.parametrize("keep", [0.0, 0.3, 0.7, 0.97])
def test_python_reader_rejects_truncated_csr(tmp_path, keep):
    p = str(tmp_path / "x.HAM.CSR")
    _write_csr_truncated(p, keep)
    with pytest.raises((ValueError, IndexError)):
        formats.read_csr(p)


def test_python_readers_reject_truncated_state_and_moment_files(tmp_path):
    st = lattices.random_phase_states(10, 2, seed=1)
    p = str(tmp_path / "states.txt")
    formats.write_vector_states(p, st)
    text = open(p).read()
    open(p, "w").write(text[: len(text) // 2])
    with pytest.raises(ValueError):
        formats.read_state_file(p)
    open(p, "w").write("local\n3\n1 2\n")
    with pytest.raises(ValueError):
        formats.read_state_file(p, dim=10)
    open(p, "w").write("gaussian\n1\n")
    with pytest.raises(ValueError):
        formats.read_state_file(p)
    m = str(tmp_path / "a.chebmom1D")
    formats.write_chebmom1d(m, 10, 8.0, 0.0, np.ones(20))
    text = open(m).read()
    open(m, "w").write(text[: len(text) - 40])
    with pytest.raises(ValueError):
        formats.read_chebmom1d(m)


def _driver(name):
    exe = os.path.join(FACADE, name)
    if not os.path.exists(exe):
        pytest.skip("facade drivers not built (needs the reference checkout at build time)")
    return exe


def _run(exe, args, cwd):
    return subprocess.run([exe] + [str(a) for a in args], cwd=cwd, capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("keep", [0.3, 0.9])
def test_facade_driver_stops_on_truncated_csr(tmp_path, keep):
    """LinQT's inline_compute-kpm-spectralOp on the facade: a short operator file stops the
    program (nonzero exit, message) before any device work."""
    exe = _driver("inline_compute-kpm-spectralOp")
    (tmp_path / "operators").mkdir()
    _write_csr_truncated(str(tmp_path / "operators" / "sq.HAM.CSR"), keep)
    (tmp_path / "BOUNDS").write_text("-4.725 4.725\n")
    p = _run(exe, ["sq", "1", 16], str(tmp_path))
    assert p.returncode != 0
    assert "CSR" in p.stderr
