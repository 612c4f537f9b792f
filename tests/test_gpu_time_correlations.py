"""Time-domain correlations (chebyshev::TimeDependentCorrelations with MomentsTD::Evolve)
on the GPU against the C restatement, which is pinned to the reference's
inline_compute-kpm-CorrOp (tests/test_oracle_vs_ref.py).  FP64: 1e-10 relative."""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


@pytest.fixture(scope="module")
def graphene(oracle_lib):
    N, H, V = lattices.honeycomb(8, 6, t=-2.7, W=1.0, seed=21)
    D = lattices.upper_csr(N, np.arange(N), np.arange(N), lattices.disorder(N, 2.0, 5) + 0j)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), 1.05 * (hi + lo) / 2
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    Ho = oracle_lib.Op(*H)
    Ho.rescale(2 / bw, -bc / (bw / 2))
    return dict(N=N, bw=bw, bc=bc, Hg=Hg, Ho=Ho, Vg=lq.Operator.from_csr(N, *V), Vo=oracle_lib.Op(*V),
                Dg=lq.Operator.from_csr(N, *D), Do=oracle_lib.Op(*D))


@pytest.mark.parametrize("R,M,NT,dt", [(1, 32, 4, 1.0), (3, 48, 5, 2.5), (8, 64, 3, 0.2)])
def test_time_correlations_match_oracle(oracle_lib, graphene, R, M, NT, dt):
    g = graphene
    st = lattices.random_phase_states(g["N"], R, seed=40 + R)
    mu = lq.moments_td(g["Hg"], g["Vg"], g["Dg"], st, M, NT, dt, g["bw"], g["bc"])
    ref = oracle_lib.moments_td(g["Ho"], g["Vo"], g["Do"], st, M, NT, dt, g["bw"], g["bc"])
    assert mu.shape == (M, NT)
    assert rel(mu, ref) < TOL


def test_time_correlations_identity_operators_and_t0(oracle_lib, graphene):
    """OPL = OPR = identity: at t = 0 the table is the 1D moments of the same states."""
    g = graphene
    st = lattices.random_phase_states(g["N"], 2, seed=7)
    M = 40
    mu = lq.moments_td(g["Hg"], None, None, st, M, 3, 1.5, g["bw"], g["bc"])
    ref = oracle_lib.moments_td(g["Ho"], None, None, st, M, 3, 1.5, g["bw"], g["bc"])
    assert rel(mu, ref) < TOL
    m1 = lq.moments1d(g["Hg"], None, st, M, opts=lq.make_opts(doubling=2))
    assert rel(mu[:, 0], m1) < 1e-12


def test_time_correlations_device_pointers(graphene):
    torch = pytest.importorskip("torch")
    g = graphene
    st = lattices.random_phase_states(g["N"], 4, seed=9)
    M, NT = 24, 4
    host = lq.moments_td(g["Hg"], g["Vg"], g["Vg"], st, M, NT, 1.0, g["bw"], g["bc"])
    dst = torch.from_numpy(st.view(np.float64).reshape(-1).copy()).cuda()
    dmu = torch.zeros(2 * M * NT, dtype=torch.float64, device="cuda")
    sess = lq.Session(0)
    lq.moments_td_dev(g["Hg"], g["Vg"], g["Vg"], dst, 4, M, NT, 1.0, g["bw"], g["bc"], dmu, session=sess)
    sess.synchronize()
    assert rel(dmu.cpu().numpy().view(np.complex128).reshape(M, NT), host) < 1e-14


def test_time_correlations_reject_mixed_precision(graphene):
    g = graphene
    with pytest.raises(lq.LinqtError) as e:
        lq.moments_td(g["Hg"], None, None, np.ones((1, g["N"])), 8, 2, 1.0, g["bw"], g["bc"],
                      opts=lq.make_opts(precision=lq.PREC_MIXED))
    assert "FP64" in str(e.value)


def test_time_correlation_from_moments_matches_oracle(oracle_lib, graphene):
    g = graphene
    st = lattices.random_phase_states(g["N"], 3, seed=11)
    M, NT, dt = 128, 6, 1.0
    mu = lq.moments_td(g["Hg"], g["Vg"], g["Vg"], st, M, NT, dt, g["bw"], g["bc"])
    for broad, ef in ((150.0, 0.3), (40.0, -2.0)):
        t, c = lq.time_correlation_from_moments(mu, g["N"], g["bw"], g["bc"], dt, broad, ef)
        to, co = oracle_lib.time_correlation(mu, g["N"], g["bw"], g["bc"], dt, broad, ef)
        assert np.array_equal(t, to)
        assert rel(c, co) < 1e-12


@pytest.mark.parametrize("R,NT,dt", [(300, 2, 0.7), (5, 1, 1.0), (4, 3, 0.0)])
def test_time_correlations_edge_cases(oracle_lib, R, NT, dt):
    """R > 256 (two vector chunks), a single time step, dt = 0 (the series is the identity:
    every time step repeats t = 0)."""
    N, H, V = lattices.honeycomb(4, 4, t=-2.7, W=1.0, seed=21)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), 1.05 * (hi + lo) / 2
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    Ho = oracle_lib.Op(*H)
    Ho.rescale(2 / bw, -bc / (bw / 2))
    st = lattices.random_phase_states(N, R, seed=13)
    M = 20
    mu = lq.moments_td(Hg, lq.Operator.from_csr(N, *V), None, st, M, NT, dt, bw, bc)
    ref = oracle_lib.moments_td(Ho, oracle_lib.Op(*V), None, st, M, NT, dt, bw, bc)
    assert rel(mu, ref) < TOL
    if dt == 0.0:
        for t in range(1, NT):
            assert rel(mu[:, t], mu[:, 0]) < 1e-13
