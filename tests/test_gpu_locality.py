"""LINQT_FORMAT_LOCAL: the persistent recursions visiting the rows of H in the locality
order (recursive bisection of the operator's graph into parts of at most 8192 rows).

Only the traversal changes: each row's gather keeps the order of its entries, so the 2D tables
(no cross-row sums) equal the CSR ones bit for bit, and the 1D moments differ only by the order
of their per-CTA dot-product sums.  Sizes are above 8192 rows so that the order is not the
natural one.
"""
import re

import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def setup(orc, N, H, extra=()):
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    Ho = orc.Op(*H).rescale(2 / bw, -bc / (bw / 2))
    return Hg, Ho, [(lq.Operator.from_csr(N, *X), orc.Op(*X)) for X in extra]


@pytest.mark.parametrize("R", [1, 8, 64])
def test_cubic_dos_local_order(oracle_lib, R):
    N, H = lattices.cubic_lattice(32, t=1.0, W=2.0, seed=48)  # 32768 rows: four parts
    Hg, Ho, _ = setup(oracle_lib, N, H)
    st = lattices.random_phase_states(N, R, seed=49)
    M = 200
    loc = lq.moments1d(Hg, None, st, M, opts=lq.make_opts(fmt=lq.FORMAT_LOCAL))
    csr = lq.moments1d(Hg, None, st, M)
    assert rel(loc, csr) < 1e-13
    assert rel(loc, oracle_lib.moments1d(Ho, None, st, M)) < TOL
    # mixed precision: FP32 blocks, the same per-row rounding in both layouts
    o = lq.make_opts(precision=lq.PREC_MIXED, fmt=lq.FORMAT_LOCAL)
    mloc = lq.moments1d(Hg, None, st, M, opts=o)
    mcsr = lq.moments1d(Hg, None, st, M, opts=lq.make_opts(precision=lq.PREC_MIXED))
    assert rel(mloc, mcsr) < 1e-12


def test_kane_mele_2d_tables_bitwise(oracle_lib):
    N, H, V = lattices.kane_mele(48, 48, seed=31)  # 9216 rows
    Hg, Ho, ((Vg, Vo),) = setup(oracle_lib, N, H, [V])
    st = lattices.random_phase_states(N, 3, seed=35)
    M = 48
    loc = lq.moments2d(Hg, Vg, Vg, st, M, opts=lq.make_opts(fmt=lq.FORMAT_LOCAL))
    csr = lq.moments2d(Hg, Vg, Vg, st, M)
    assert np.array_equal(loc, csr)
    assert rel(loc, oracle_lib.moments2d(Ho, Vo, Vo, st, M)) < TOL


def test_kubo_bastin_local_order(oracle_lib):
    N, H, V = lattices.kane_mele(48, 48, seed=32)
    Hg, Ho, ((Vg, Vo),) = setup(oracle_lib, N, H, [V])
    st = lattices.random_phase_states(N, 2, seed=36)
    M, nump = 64, 256
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    mu_a, fa = lq.kubo_bastin(Hg, Vg, Vg, st, M, nump, bw, bc, opts=lq.make_opts(fmt=lq.FORMAT_LOCAL))
    mu_b, fb = lq.kubo_bastin(Hg, Vg, Vg, st, M, nump, bw, bc)
    assert np.array_equal(mu_a, mu_b)
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)


def test_autotuner_considers_the_local_order(oracle_lib):
    """At 64 columns of a 2e5-row cubic lattice a block exceeds 64 MB, so the autotuner times
    the locality layout too; whatever it picks gives the oracle's moments."""
    N, H = lattices.cubic_lattice(60, t=1.0, W=2.0, seed=50)
    Hg, Ho, _ = setup(oracle_lib, N, H)
    st = lattices.random_phase_states(N, 64, seed=51)
    mu = lq.moments1d(Hg, None, st, 40, opts=lq.make_opts(fmt=lq.FORMAT_AUTO))
    assert rel(mu, oracle_lib.moments1d(Ho, None, st, 40)) < TOL
    tuned = Hg.tuned()  # linqt_op_tuned: the cached layout and width decisions
    layouts = [v for k, v in tuned.items() if k.startswith("1d:")]
    assert layouts and all(re.fullmatch(r"(csr|csr_nocache|sell\d+(_local)?) shape \d", v) for v in layouts)
    assert any(k.startswith("1dw:") and re.fullmatch(r"width \d+", v) for k, v in tuned.items())


@pytest.mark.parametrize("R", [1, 2, 8, 64])
def test_every_1d_thread_shape(oracle_lib, R):
    """Each thread shape of the 1D recursion (opts.thread_shape), in the natural and the
    locality order, against the oracle, FP64 blocks at the FP64 tolerance and FP32 blocks at
    the mixed path's."""
    N, H = lattices.cubic_lattice(24, t=1.0, W=2.0, seed=52)  # 13,824 rows: two parts
    Hg, Ho, _ = setup(oracle_lib, N, H)
    st = lattices.random_phase_states(N, R, seed=53)
    M = 96
    ref = oracle_lib.moments1d(Ho, None, st, M)
    shapes = {1: 1, 2: 2, 8: 4, 64: 3}[R]  # threads per row min(R, 32) >> s, <= 8 columns each
    for fmt in (lq.FORMAT_CSR, lq.FORMAT_LOCAL):
        for s in range(shapes):
            mu = lq.moments1d(Hg, None, st, M, opts=lq.make_opts(fmt=fmt, block_width=R, thread_shape=s + 1))
            assert rel(mu, ref) < TOL, (fmt, s)
            mx = lq.moments1d(Hg, None, st, M, opts=lq.make_opts(precision=lq.PREC_MIXED, fmt=fmt, block_width=R,
                                                                  thread_shape=s + 1))
            assert rel(mx, ref) < 1e-7, (fmt, s)
    with pytest.raises(lq.LinqtError):
        lq.moments1d(Hg, None, st, M, opts=lq.make_opts(block_width=R, thread_shape=shapes + 1))
