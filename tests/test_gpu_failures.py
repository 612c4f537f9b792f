"""Failure handling on the GPU: a bounded device wait that runs out is reported as
LINQT_ERR_TIMEOUT and leaves the session usable; a facade driver stops on a truncated
state file (it reads the states after building its operators on the device).

The timeout is made on purpose with the session's test hook
(linqt_session_inject_barrier_timeout): the grid barriers of its persistent kernels wait for
one CTA that was never launched and give up after 1024 polls (well under a millisecond), the
kernels return through their normal exit, and the host reads the error flag.  No GPU fault,
trap or endless wait is involved."""
import os
import subprocess

import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import formats, lattices

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FACADE = os.path.join(ROOT, "linqt_b200", "facade", "_drivers")
BW = 2 * 1.05 * 4.5


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def square(oracle_lib):
    N, H = lattices.square_lattice(24, t=1.0, W=1.0, seed=11)
    st = lattices.random_phase_states(N, 3, seed=12)
    Ho = oracle_lib.Op(*H).rescale(2 / BW, 0.0)
    return N, H, st, Ho


def test_barrier_timeout_is_reported_and_the_session_recovers(oracle_lib, square):
    N, H, st, Ho = square
    sess = lq.Session(0)
    Hg = lq.Operator.from_csr(N, *H, session=sess)
    Hg.rescale_to_chebyshev(BW, 0.0)
    M = 64
    ref = oracle_lib.moments1d(Ho, None, st, M)
    sess.inject_barrier_timeout(1, 1024)
    for _ in range(2):  # every solve fails while the hook is set
        with pytest.raises(lq.LinqtError) as e:
            lq.moments1d(Hg, None, st, M, session=sess)
        assert e.value.code == -6  # LINQT_ERR_TIMEOUT
    # a session without the hook is not affected meanwhile
    other = lq.Session(0)
    assert rel(lq.moments1d(Hg, None, st, M, session=other), ref) < 1e-10
    sess.inject_barrier_timeout(0, 0)
    assert rel(lq.moments1d(Hg, None, st, M, session=sess), ref) < 1e-10


def test_timeout_in_the_2d_and_nonorthogonal_recursions(oracle_lib, square):
    N, H, st, Ho = square
    sess = lq.Session(0)
    Hg = lq.Operator.from_csr(N, *H, session=sess)
    Hg.rescale_to_chebyshev(BW, 0.0)
    V = lq.Operator.from_csr(N, *H, session=sess)
    S = lq.Operator.from_csr(N, *lattices.overlap_matrix(N, H), storage=lq.STORAGE_GENERAL, session=sess)
    sess.inject_barrier_timeout(1, 512)
    with pytest.raises(lq.LinqtError) as e:
        lq.moments2d(Hg, V, V, st, 32, session=sess)
    assert e.value.code == -6
    with pytest.raises(lq.LinqtError) as e:
        lq.moments1d_nonorth(Hg, None, S, st, 16, session=sess)
    assert e.value.code == -6
    sess.inject_barrier_timeout(0, 0)
    Vo = oracle_lib.Op(*H)
    assert rel(lq.moments2d(Hg, V, V, st, 32, session=sess), oracle_lib.moments2d(Ho, Vo, Vo, st, 32)) < 1e-10


def test_facade_driver_stops_on_truncated_state_file(tmp_path):
    exe = os.path.join(FACADE, "inline_compute-kpm-spectralOp")
    if not os.path.exists(exe):
        pytest.skip("facade drivers not built (needs the reference checkout at build time)")
    (tmp_path / "operators").mkdir()
    N, H = lattices.square_lattice(4, t=1.0, W=1.0, seed=11)
    formats.write_csr(str(tmp_path / "operators" / "sq.HAM.CSR"), N, *H)
    (tmp_path / "BOUNDS").write_text("-4.725 4.725\n")
    sp = tmp_path / "states.txt"
    formats.write_vector_states(str(sp), lattices.random_phase_states(N, 2, seed=3))
    sp.write_text(sp.read_text()[:200])
    p = subprocess.run([exe, "sq", "1", "16", "states.txt"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=120)
    assert p.returncode != 0
    assert "state file" in p.stderr
