"""1D moments in a non-orthogonal basis (chebyshev::SpectralMoments_nonOrth,
src/chebyshev_solver.cpp:203-229) on the GPU: linqt_moments1d_nonorth against the oracle
restatement (lo_moments1d_nonorth), which tests/test_oracle_vs_ref.py pins to the reference's
own inline_compute-kpm-spectralOp-nonOrth.  Every S^-1 is a BiCGSTAB solve; at the
reference's tolerance (1e-4) the GPU solver takes the same iterations as the oracle, so the
moments agree to rounding (1e-10); at a tight tolerance both reach S^-1 itself."""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu

TOL = 1e-10
BW, BC = 2 * 1.05 * 4.5, 0.0


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def expand_upper(N, csr):
    """The full Hermitian CSR of an upper-stored one (rows sorted by column)."""
    rp, cl, vl = csr
    rows = np.repeat(np.arange(N), np.diff(rp))
    low = cl != rows
    r = np.concatenate([rows, cl[low]])
    c = np.concatenate([cl, rows[low]])
    v = np.concatenate([vl, np.conj(vl[low])])
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    rowptr = np.zeros(N + 1, np.int64)
    np.add.at(rowptr, r + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), c.astype(np.int32), v


def case(L=12, R=3, s=0.08):
    N, H = lattices.square_lattice(L, t=1.0, W=1.0, seed=11)
    S = lattices.overlap_matrix(N, H, s=s, seed=13)
    st = lattices.random_phase_states(N, R, seed=12)
    return N, H, S, st


def gpu_ops(N, H, S, storage, with_op):
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(BW, BC)
    Sg = lq.Operator.from_csr(N, *S, storage=storage)
    return Hg, Sg, (lq.Operator.from_csr(N, *H) if with_op else None)


def oracle_ops(oracle_lib, H, with_op):
    Ho = oracle_lib.Op(*H).rescale(2 / BW, -BC / (BW / 2))
    return Ho, (oracle_lib.Op(*H) if with_op else None)


@pytest.mark.parametrize("with_op", [False, True])
def test_nonorth_matches_oracle_at_reference_tolerance(oracle_lib, with_op):
    """S as the reference's solver sees it (the stored upper triangle), tolerance 1e-4."""
    N, H, S, st = case()
    M = 96
    Hg, Sg, OPg = gpu_ops(N, H, S, lq.STORAGE_GENERAL, with_op)
    mu, its = lq.moments1d_nonorth(Hg, OPg, Sg, st, M)
    Ho, OPo = oracle_ops(oracle_lib, H, with_op)
    mu_o, its_o = oracle_lib.moments1d_nonorth(Ho, OPo, S, st, M)
    assert its == its_o  # the same BiCGSTAB iterations, solve by solve summed
    assert rel(mu, mu_o) < TOL


def test_nonorth_tight_tolerance_hermitian_overlap(oracle_lib):
    """The full Hermitian S (Hermitian-upper storage expands it) solved to 1e-13."""
    N, H, S, st = case(L=10, R=2)
    M = 64
    Hg, Sg, _ = gpu_ops(N, H, S, lq.STORAGE_HERMITIAN_UPPER, False)
    mu, its = lq.moments1d_nonorth(Hg, None, Sg, st, M, tol=1e-13)
    Ho, _ = oracle_ops(oracle_lib, H, False)
    mu_o, its_o = oracle_lib.moments1d_nonorth(Ho, None, expand_upper(N, S), st, M, tol=1e-13)
    assert its > 2 * M  # several iterations per solve at this tolerance
    assert rel(mu, mu_o) < TOL


def test_nonorth_identity_overlap_is_the_orthogonal_expansion():
    """S = I: one BiCGSTAB iteration per solve and the moments of SpectralMoments."""
    N, H, _, st = case(L=16, R=4)
    M = 80
    ident = (np.arange(N + 1, dtype=np.int32), np.arange(N, dtype=np.int32), np.ones(N, np.complex128))
    Hg, Sg, _ = gpu_ops(N, H, ident, lq.STORAGE_GENERAL, False)
    mu, its = lq.moments1d_nonorth(Hg, None, Sg, st, M)
    assert its == 4 * M  # M solves per state, one iteration each
    ref = lq.moments1d(Hg, None, st, M, opts=lq.make_opts(doubling=2))
    assert rel(mu, ref) < 1e-13


def test_nonorth_more_states_than_one_block(oracle_lib):
    """R = 40: two launches (32 + 8 states), the second zero-padded."""
    N, H, S, st = case(L=8, R=40)
    M = 32
    Hg, Sg, _ = gpu_ops(N, H, S, lq.STORAGE_GENERAL, False)
    mu, its = lq.moments1d_nonorth(Hg, None, Sg, st, M)
    Ho, _ = oracle_ops(oracle_lib, H, False)
    mu_o, its_o = oracle_lib.moments1d_nonorth(Ho, None, S, st, M)
    assert its == its_o
    assert rel(mu, mu_o) < TOL


def test_nonorth_device_entry_point_and_repeat():
    """The _dev form on a session stream equals the host form, call after call."""
    torch = pytest.importorskip("torch")
    N, H, S, st = case(L=12, R=5)
    M = 40
    Hg, Sg, _ = gpu_ops(N, H, S, lq.STORAGE_GENERAL, False)
    ref, its_ref = lq.moments1d_nonorth(Hg, None, Sg, st, M)
    st_dev = torch.from_numpy(st.view(np.float64).copy()).cuda()
    sess = lq.Session(0)
    for _ in range(2):
        out = torch.full((2 * M,), float("nan"), dtype=torch.float64, device="cuda")
        its = lq.moments1d_nonorth_dev(Hg, None, Sg, st_dev, 5, M, out, session=sess, iterations=True)
        sess.synchronize()
        assert its == its_ref
        assert np.array_equal(out.cpu().numpy().view(np.complex128), ref)


def test_nonorth_is_fp64_only():
    N, H, S, st = case(L=6, R=1)
    Hg, Sg, _ = gpu_ops(N, H, S, lq.STORAGE_GENERAL, False)
    with pytest.raises(lq.LinqtError) as e:
        lq.moments1d_nonorth(Hg, None, Sg, st, 8, opts=lq.make_opts(precision=lq.PREC_MIXED))
    assert e.value.code == -4
