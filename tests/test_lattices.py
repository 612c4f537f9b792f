"""Synthetic inputs: Philox4x32-10 known-answer vectors, Hermiticity and sizes of the
lattice families the benchmark configurations name."""
import numpy as np
import pytest

from linqt_b200 import lattices as L


@pytest.mark.parametrize("ctr,key,out", [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(ctr, key, out):
    got = L.philox4x32_10(*[np.array([c], np.uint64) for c in ctr], *key)
    assert tuple(int(g[0]) for g in got) == out


def test_uniform_range_and_determinism():
    u = L.uniform(12, 100000)
    assert u.min() >= 0 and u.max() < 1
    assert abs(u.mean() - 0.5) < 0.01
    assert np.array_equal(u[:10], L.uniform(12, 10))
    assert np.array_equal(u[5:10], L.uniform(12, 5, offset=5))
    assert not np.array_equal(u[:10], L.uniform(13, 10))


def test_random_phase_states_normalised():
    st = L.random_phase_states(1000, 3, seed=12)
    assert np.allclose(np.linalg.norm(st, axis=1), 1.0)
    assert np.allclose(np.abs(st), 1 / np.sqrt(1000))


def _is_hermitian_upper(n, rp, col, val):
    rows = np.repeat(np.arange(n), np.diff(rp))
    assert (col >= rows).all()
    for i in range(n):
        assert np.all(np.diff(col[rp[i]:rp[i + 1]]) > 0)
    d = L.hermitian_dense(n, rp, col, val)
    assert np.abs(d - d.conj().T).max() == 0


def test_square_lattice():
    N, H = L.square_lattice(6, 1.0, 1.0, 11)
    _is_hermitian_upper(N, *H)
    assert N == 36 and len(H[1]) == 3 * N
    assert abs(H[2][H[1] == np.repeat(np.arange(N), np.diff(H[0]))].real).max() <= 0.5


def test_honeycomb_and_velocity():
    N, H, V = L.honeycomb(5, 4, t=-2.7, W=1.0, seed=21, a=1.42)
    _is_hermitian_upper(N, *H)
    _is_hermitian_upper(N, *V)
    assert N == 40
    # expanded: 4 non-zeros per row for H (3 NN + diagonal), 3 for V
    assert len(H[1]) == N + 3 * N // 2 and len(V[1]) == 3 * N // 2
    # |V_ij| = |x_i - x_j| |t| with |dx| in {a, a/2}
    assert set(np.round(np.abs(V[2]), 6)) <= {round(1.42 * 2.7, 6), round(0.71 * 2.7, 6)}
    # clean graphene spectrum within [-3|t|, 3|t|]
    N0, H0, _ = L.honeycomb(6, 6, t=-2.7, W=0.0)
    w = np.linalg.eigvalsh(L.hermitian_dense(N0, *H0))
    assert abs(w.max() - 8.1) < 1e-9 and abs(w.min() + 8.1) < 1e-9


def test_kane_mele():
    N, H, J = L.kane_mele(4, 4)
    _is_hermitian_upper(N, *H)
    _is_hermitian_upper(N, *J)
    expanded = 2 * len(H[1]) - N
    assert N == 64 and expanded == 13 * N


def test_cubic_lattice():
    N, H = L.cubic_lattice(5, 1.0, 2.0, 41)
    _is_hermitian_upper(N, *H)
    assert N == 125 and 2 * len(H[1]) - N == 7 * N


def test_gershgorin_contains_spectrum():
    N, H = L.square_lattice(6, 1.0, 1.0, 11)
    lo, hi = L.gershgorin_bounds(N, *H)
    w = np.linalg.eigvalsh(L.hermitian_dense(N, *H))
    assert lo <= w.min() and w.max() <= hi
