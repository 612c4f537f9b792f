"""Parity on the other workload families at sizes the oracle finishes in seconds:

- plain DOS on the square lattice (1 vector, M = 1024, DOS on the Chebyshev grid);
- spin transport on the Kane-Mele honeycomb with spin (4 orbitals per cell, NNN spin-orbit
  and Rashba terms) with the spin-velocity operator {s_z, V_x}/2, FP64 and mixed;
- large-DOS batching on the 3D cubic Anderson lattice (7-point stencil): many vectors in one
  block, several disorder seeds, FP64 and mixed.
"""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def ops(orc, N, H, extra=(), pad=1.05):
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = pad * (hi - lo), (hi + lo) / 2
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    Ho = orc.Op(*H).rescale(2 / bw, -bc / (bw / 2))
    return bw, bc, Hg, Ho, [(lq.Operator.from_csr(N, *X), orc.Op(*X)) for X in extra]


def test_square_dos_one_vector_m1024(oracle_lib):
    N, H = lattices.square_lattice(64, t=1.0, W=1.0, seed=11)
    bw, bc = 2 * 1.05 * 4.5, 0.0
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    Ho = oracle_lib.Op(*H).rescale(2 / bw, -bc / (bw / 2))
    st = lattices.random_phase_states(N, 1, seed=12)
    mu = lq.moments1d(Hg, None, st, 1024)
    ref = oracle_lib.moments1d(Ho, None, st, 1024)
    assert rel(mu, ref) < TOL
    assert abs(mu[0] - 1.0) < 1e-12  # mu_0 = <r|r> for one normalised state
    E, d = lq.dos_from_moments(mu, N, bw, bc, broad_meV=5.0)
    Eo, do = oracle_lib.dos_fftgrid(oracle_lib.jackson1d(ref, bw, 5.0), N, bw, bc)
    assert rel(E, Eo) < 1e-14 and rel(d, do) < 1e-10


@pytest.fixture(scope="module")
def kane_mele(oracle_lib):
    N, H, J = lattices.kane_mele(6, 5, seed=31)
    bw, bc, Hg, Ho, ((Jg, Jo),) = ops(oracle_lib, N, H, [J])
    return dict(N=N, bw=bw, bc=bc, Hg=Hg, Ho=Ho, Jg=Jg, Jo=Jo)


def test_kane_mele_spin_correlation(oracle_lib, kane_mele):
    k = kane_mele
    st = lattices.random_phase_states(k["N"], 3, seed=32)
    M = 96
    mu = lq.moments2d(k["Hg"], k["Jg"], k["Jg"], st, M)
    ref = oracle_lib.moments2d(k["Ho"], k["Jo"], k["Jo"], st, M)
    assert rel(mu, ref) < TOL
    assert np.abs(mu - mu.conj().T).max() < 1e-13 * np.abs(mu).max()


@pytest.mark.parametrize("precision,tol", [(lq.PREC_FP64, 1e-10), (lq.PREC_MIXED, 1e-6)])
def test_kane_mele_spin_kubo_bastin(oracle_lib, kane_mele, precision, tol):
    k = kane_mele
    st = lattices.random_phase_states(k["N"], 2, seed=33)
    M, nump = 64, 256
    mu, (E, s, integ) = lq.kubo_bastin(k["Hg"], k["Jg"], k["Jg"], st, M, nump, k["bw"], k["bc"],
                                       opts=lq.make_opts(precision=precision))
    Eo, so, io, _ = oracle_lib.kubo_fft(k["Ho"], k["Jo"], k["Jo"], st, M, nump, lq.KUBO_BASTIN, k["N"], k["bw"],
                                        k["bc"])
    assert rel(E, Eo) < 1e-14
    lo, hi = int(0.05 * nump), int(0.95 * nump)
    assert rel(s[lo:hi], so[lo:hi]) < tol
    assert rel(mu, oracle_lib.moments2d(k["Ho"], k["Jo"], k["Jo"], st, M)) < tol


@pytest.mark.parametrize("seed", [41, 42, 43, 44])
def test_cubic_dos_many_vectors(oracle_lib, seed):
    N, H = lattices.cubic_lattice(10, t=1.0, W=2.0, seed=seed)
    bw, bc, Hg, Ho, _ = ops(oracle_lib, N, H)
    st = lattices.random_phase_states(N, 40, seed=45)  # ragged: padded to a 64-wide block
    M = 512
    mu = lq.moments1d(Hg, None, st, M)
    ref = oracle_lib.moments1d(Ho, None, st, M)
    assert rel(mu, ref) < TOL
    mx = lq.moments1d(Hg, None, st, M, opts=lq.make_opts(precision=lq.PREC_MIXED))
    assert rel(mx, ref) < 1e-7  # FP32 blocks: measured ~2e-10 on the DOS moments


def test_large_operator_rows_not_cached(oracle_lib):
    """N = 1e6 cubic lattice: the per-CTA operator slices exceed the shared-memory cache, so
    the persistent recursions deal rows to CTAs in round-robin tiles."""
    N, H = lattices.cubic_lattice(100, t=1.0, W=2.0, seed=42)
    bw, bc, Hg, Ho, _ = ops(oracle_lib, N, H)
    st = lattices.random_phase_states(N, 1, seed=46)
    mu = lq.moments1d(Hg, None, st, 48)
    assert rel(mu, oracle_lib.moments1d(Ho, None, st, 48)) < TOL
    mu2 = lq.moments2d(Hg, None, None, st, 12)
    assert rel(mu2, oracle_lib.moments2d(Ho, None, None, st, 12)) < TOL


@pytest.mark.parametrize("fmt", [1, 2])  # SELL-C-sigma (C = 32), autotuned
def test_sell_layout_matches_csr(oracle_lib, fmt):
    """The persistent recursions on the SELL-C-sigma layout: the row sums keep their order
    (padding adds exact zeros), so the 2D tables are those of CSR bit for bit; the 1D moments
    sum their dot products over rows in another order (1e-13)."""
    N, H, V = lattices.kane_mele(8, 6, seed=31)  # rows of 9 to 13 non-zeros
    bw, bc, Hg, Ho, ((Vg, Vo),) = ops(oracle_lib, N, H, [V])
    st = lattices.random_phase_states(N, 5, seed=34)
    o = lq.make_opts(fmt=fmt)
    csr2 = lq.moments2d(Hg, Vg, Vg, st, 40)
    sell2 = lq.moments2d(Hg, Vg, Vg, st, 40, opts=o)
    assert np.array_equal(csr2, sell2) or fmt == 2
    assert rel(sell2, oracle_lib.moments2d(Ho, Vo, Vo, st, 40)) < TOL
    csr1 = lq.moments1d(Hg, None, st, 100)
    sell1 = lq.moments1d(Hg, None, st, 100, opts=o)
    assert rel(sell1, csr1) < 1e-13
    assert rel(sell1, oracle_lib.moments1d(Ho, None, st, 100)) < TOL


def test_sell_layout_large_operator(oracle_lib):
    N, H = lattices.cubic_lattice(100, t=1.0, W=2.0, seed=43)
    bw, bc, Hg, Ho, _ = ops(oracle_lib, N, H)
    st = lattices.random_phase_states(N, 2, seed=47)
    mu = lq.moments1d(Hg, None, st, 32, opts=lq.make_opts(fmt=1))
    assert rel(mu, oracle_lib.moments1d(Ho, None, st, 32)) < TOL


@pytest.mark.parametrize("S,Rs", [(4, 32), (2, 64), (3, 8)])
def test_disorder_realisations_in_one_block(oracle_lib, S, Rs):
    """S Anderson disorder seeds x Rs vectors in one persistent recursion: each realisation's
    moments equal its own single-Hamiltonian solve and the oracle's."""
    L, M = 10, 200
    ops_g, ops_o, states = [], [], []
    bw, bc = 2 * 1.05 * (6.0 + 1.0), 0.0  # common bounds for all seeds: |E| <= 6t + W/2
    for r in range(S):
        N, H = lattices.cubic_lattice(L, t=1.0, W=2.0, seed=41 + r)
        Hg = lq.Operator.from_csr(N, *H)
        Hg.rescale_to_chebyshev(bw, bc)
        ops_g.append(Hg)
        ops_o.append(oracle_lib.Op(*H).rescale(2 / bw, -bc / (bw / 2)))
        states.append(lattices.random_phase_states(N, Rs, seed=100 + r))
    mu = lq.moments1d_realisations(ops_g, np.concatenate(states), M, opts=lq.make_opts(realisations=1))
    assert mu.shape == (S, M)
    for mode in (0, 2):  # autotuned, one solve per realisation
        other = lq.moments1d_realisations(ops_g, np.concatenate(states), M, opts=lq.make_opts(realisations=mode))
        assert rel(other, mu) < 1e-12
    for r in range(S):
        alone = lq.moments1d(ops_g[r], None, states[r], M)
        assert rel(mu[r], alone) < 1e-12
        assert rel(mu[r], oracle_lib.moments1d(ops_o[r], None, states[r], M)) < TOL
    mx = lq.moments1d_realisations(ops_g, np.concatenate(states), M, opts=lq.make_opts(precision=lq.PREC_MIXED))
    assert rel(mx, mu) < 1e-5


def test_disorder_realisations_reject_unknown_mode():
    N, H = lattices.cubic_lattice(6, seed=41)
    a = lq.Operator.from_csr(N, *H)
    with pytest.raises(lq.LinqtError) as e:
        lq.moments1d_realisations([a, a], np.ones((2, N)), 16, opts=lq.make_opts(realisations=3))
    assert "realisations" in str(e.value)


def test_disorder_realisations_reject_mismatched_patterns():
    N, H = lattices.cubic_lattice(6, seed=41)
    N2, H2 = lattices.cubic_lattice(7, seed=41)
    a = lq.Operator.from_csr(N, *H)
    b = lq.Operator.from_csr(N2, *H2)
    with pytest.raises(lq.LinqtError):
        lq.moments1d_realisations([a, b], np.ones((64, N)), 16)
