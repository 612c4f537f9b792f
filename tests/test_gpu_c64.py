"""Complex64 operators in the 1D recursions (opts.operator_precision = 1): each value of the
rescaled, Hermitian-expanded H rounded once to FP32, the products accumulated in FP64.

Parity: the GPU result equals the oracle run on the same rounded operator to 1e-10 (the
rounding is the only change), and differs from the complex128 result by the stated error of
the option (measured 3e-7 at M = 512 and 9e-7 at M = 2048 on the cubic Anderson lattice)."""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu

BW = 2 * 1.05 * 7.0


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def rounded_oracle_op(oracle_lib, Ho):
    """The oracle operator with every expanded value rounded to complex64."""
    n, nnz = Ho.n, Ho.nnz
    rp, cl, vl = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(2 * nnz)
    oracle_lib.lib().lo_op_export(Ho.h, oracle_lib._ip(rp), oracle_lib._ip(cl), oracle_lib._dp(vl))
    v = (vl[0::2] + 1j * vl[1::2]).astype(np.complex64).astype(np.complex128)
    rows = np.repeat(np.arange(n), np.diff(rp))
    up = cl >= rows
    rpu = np.zeros(n + 1, np.int64)
    np.add.at(rpu, rows[up] + 1, 1)
    return oracle_lib.Op(np.cumsum(rpu).astype(np.int32), cl[up], v[up])


@pytest.fixture(scope="module")
def cubic(oracle_lib):
    N, H = lattices.cubic_lattice(12, 1.0, 2.0, 41)
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(BW, 0.0)
    Ho = oracle_lib.Op(*H).rescale(2 / BW, 0.0)
    return N, H, Hg, Ho, rounded_oracle_op(oracle_lib, Ho)


@pytest.mark.parametrize("fmt", [0, 1, 2, 3])  # CSR, SELL, autotuned, SELL over the locality order
def test_c64_operator_matches_the_oracle_on_the_rounded_operator(oracle_lib, cubic, fmt):
    N, H, Hg, Ho, H32 = cubic
    st = lattices.random_phase_states(N, 8, seed=45)
    M = 512
    mu = lq.moments1d(Hg, None, st, M, opts=lq.make_opts(fmt=fmt, operator_precision=lq.OP_C64))
    assert rel(mu, oracle_lib.moments1d(H32, None, st, M)) < 1e-10
    e = rel(mu, oracle_lib.moments1d(Ho, None, st, M))
    assert 1e-9 < e < 1e-6  # the stated error of complex64 values (measured 2.9e-7 here)


def test_c64_operator_with_fp32_vectors(oracle_lib, cubic):
    N, H, Hg, Ho, H32 = cubic
    st = lattices.random_phase_states(N, 16, seed=46)
    M = 256
    mu = lq.moments1d(Hg, None, st, M, opts=lq.make_opts(precision=lq.PREC_MIXED, operator_precision=lq.OP_C64))
    assert rel(mu, oracle_lib.moments1d(Ho, None, st, M)) < 1e-6


def test_c64_realisations_stacked_and_separate(oracle_lib):
    S, Rs, M = 3, 8, 200
    ops, oracle_ops = [], []
    for r in range(S):
        N, H = lattices.cubic_lattice(10, 1.0, 2.0, 41 + r)
        Hg = lq.Operator.from_csr(N, *H)
        Hg.rescale_to_chebyshev(BW, 0.0)
        ops.append(Hg)
        oracle_ops.append(rounded_oracle_op(oracle_lib, oracle_lib.Op(*H).rescale(2 / BW, 0.0)))
    st = lattices.random_phase_states(N, S * Rs, seed=47)
    for mode in (1, 2):
        mu = lq.moments1d_realisations(ops, st, M, opts=lq.make_opts(realisations=mode, operator_precision=lq.OP_C64))
        for r in range(S):
            ref = oracle_lib.moments1d(oracle_ops[r], None, st[r * Rs:(r + 1) * Rs], M)
            assert rel(mu[r], ref) < 1e-10


def test_c64_operator_is_a_1d_option_only(cubic):
    N, H, Hg, Ho, H32 = cubic
    st = lattices.random_phase_states(N, 2, seed=48)
    with pytest.raises(lq.LinqtError) as e:
        lq.moments2d(Hg, Hg, Hg, st, 16, opts=lq.make_opts(operator_precision=lq.OP_C64))
    assert e.value.code == -4
    with pytest.raises(lq.LinqtError) as e:
        lq.moments1d(Hg, None, st, 16, opts=lq.make_opts(operator_precision=lq.OP_C64, step_launches=1))
    assert e.value.code == -4
