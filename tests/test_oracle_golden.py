"""Pin the C oracle against the golden results shipped with the reference.

examples/utilities/wannier2sparse/linear_chain in adamecius/linqt holds two 2D
moment tables (M = 100 with bounds -5..5, M = 300 with bounds -2.45..2.45; default
state = unit vector at N/2) and the Kubo-Bastin curves computed from them with
xbound 0.9 (M = 100 untruncated, M = 300 Jackson-truncated to 154 moments by a
50 meV broadening).  tests/golden/make_golden.py copied them into linear_chain.npz.
"""
import numpy as np
import pytest


def _ops(oracle_lib, golden, bw):
    H = oracle_lib.Op(golden["HAM_rowptr"], golden["HAM_col"], golden["HAM_val"])
    H.rescale(2 / bw, 0.0)
    V = oracle_lib.Op(golden["VX_rowptr"], golden["VX_col"], golden["VX_val"])
    return H, V


@pytest.mark.parametrize("M,bw", [(100, 10.0), (300, 4.9)])
def test_oracle_reproduces_golden_moments(oracle_lib, golden, M, bw):
    H, V = _ops(oracle_lib, golden, bw)
    N = H.n
    hdr = golden["mu%d_header" % M]
    assert int(hdr[0]) == N and hdr[1] == bw and hdr[2] == 0.0
    st = np.zeros((1, N), np.complex128)
    st[0, N // 2] = 1.0
    mu = oracle_lib.moments2d(H, V, V, st, M)
    g = golden["mu%d" % M]
    ref = g[..., 0] + 1j * g[..., 1]
    assert np.abs(mu - ref).max() / np.abs(ref).max() < 1e-13


@pytest.mark.parametrize("M,b,bw,Mt", [(100, 100.0, 10.0, 100), (300, 50.0, 4.9, 154)])
def test_oracle_reproduces_golden_bastin(oracle_lib, golden, M, b, bw, Mt):
    g = golden["mu%d" % M]
    mu = g[..., 0] + 1j * g[..., 1]
    N = int(golden["mu%d_header" % M][0])
    muj = oracle_lib.jackson2d(mu, bw, b, b)
    assert muj.shape == (Mt, Mt)
    E, s = oracle_lib.bastin_from_moments(muj, N, bw, 0.0, xbound=0.9)
    ref = golden["bastin%d" % M]
    assert len(E) == len(ref) == 30 * Mt - 1
    assert np.abs(E - ref[:, 0]).max() < 1e-5
    # the .dat files print 6 significant digits
    assert np.abs(s - ref[:, 1]).max() / np.abs(ref[:, 1]).max() < 2e-6


def test_oracle_known_answers(oracle_lib):
    """Algebraic checks: mu_0 = 1 for normalised states; for a unit-vector state the
    odd moments vanish on a bipartite lattice without on-site terms (no closed walks of
    odd length); and the recursion agrees with T_m(x) = cos(m arccos x) applied densely."""
    from linqt_b200 import lattices
    N, H = lattices.square_lattice(8, t=1.0, W=0.0, seed=1)
    Ho = oracle_lib.Op(*H).rescale(1 / 4.2, 0.0)
    st = lattices.random_phase_states(N, 2, seed=3)
    mu = oracle_lib.moments1d(Ho, None, st, 40)
    assert abs(mu[0] - 1) < 1e-14
    loc = np.zeros((1, N), np.complex128)
    loc[0, 5] = 1.0
    assert np.abs(oracle_lib.moments1d(Ho, None, loc, 40)[1::2]).max() < 1e-15
    # dense check of the recursion: mu_m = (2/R)(1/2)^{[m=0]} sum_r <r|T_m(Ht)|r>
    Hd = lattices.hermitian_dense(N, *H) / 4.2
    w, U = np.linalg.eigh(Hd)
    ref = []
    for m in range(40):
        Tm = (U * np.cos(m * np.arccos(np.clip(w, -1, 1)))) @ U.conj().T
        v = sum(np.vdot(st[r], Tm @ st[r]) for r in range(2)) * (2 / 2) * (0.5 if m == 0 else 1)
        ref.append(v)
    assert np.abs(mu - np.array(ref)).max() < 1e-12
