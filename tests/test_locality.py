"""The locality order behind LINQT_FORMAT_LOCAL (host-only entry point, no GPU).

The recursions visit the rows of H in this order; the vector blocks stay in the natural
numbering.  On a periodic cubic lattice numbered x + L(y + Lz) a row's z neighbours are L^2
rows away, so a cache that holds fewer than L^2 rows of T_n loses them between reads; the
order keeps graph neighbours close in time.
"""
import numpy as np
import pytest

import linqt_b200 as lq


def cubic_pattern(L):
    N = L ** 3
    i = np.arange(N)
    x, y, z = i % L, (i // L) % L, i // (L * L)
    cols = [i]
    for d in [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
        cols.append((x + d[0]) % L + L * (((y + d[1]) % L) + L * ((z + d[2]) % L)))
    C = np.sort(np.stack(cols, 1), 1).astype(np.int32)
    return N, np.arange(0, 7 * N + 1, 7, dtype=np.int32), C.reshape(-1)


def row_reads(N, rp, ci, order, window):
    """Reads of T_n rows per row when a row read within `window` visits of its last read is
    served from cache (the first read of a row always counts)."""
    t = np.empty(N, np.int64)
    t[order] = np.arange(N)
    at, ar = np.repeat(t, np.diff(rp)), ci.astype(np.int64)
    o = np.lexsort((at, ar))
    ar, at = ar[o], at[o]
    new = np.ones(len(ar), bool)
    new[1:] = (ar[1:] != ar[:-1]) | (at[1:] - at[:-1] > window)
    return new.sum() / N


def test_permutation_and_deterministic():
    N, rp, ci = cubic_pattern(24)
    a = lq.locality_order(rp, ci, 512)
    b = lq.locality_order(rp, ci, 512)
    assert np.array_equal(np.sort(a), np.arange(N))
    assert np.array_equal(a, b)


def test_small_patterns_keep_the_natural_order():
    N, rp, ci = cubic_pattern(8)
    assert np.array_equal(lq.locality_order(rp, ci, N), np.arange(N))
    assert len(lq.locality_order(np.zeros(1, np.int32), np.zeros(0, np.int32), 4)) == 0


def test_cubic_lattice_neighbours_stay_close():
    # L = 40: L^2 = 1600 rows between z neighbours, a cache of 1000 rows
    N, rp, ci = cubic_pattern(40)
    natural = row_reads(N, rp, ci, np.arange(N), 1000)
    local = row_reads(N, rp, ci, lq.locality_order(rp, ci, 512), 1000)
    assert natural > 2.9
    assert local < 1.7


def test_disconnected_components_and_isolated_rows():
    # two disjoint chains and rows with only a diagonal entry
    n = 3000
    rows, cols = [], []
    for i in range(n):
        rows.append(i)
        cols.append(i)
        j = i + 2  # chains of even and of odd rows
        if j < n and i < 2000:
            rows += [i, j]
            cols += [j, i]
    order = np.lexsort((cols, rows))
    r, c = np.asarray(rows)[order], np.asarray(cols)[order]
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, r + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    o = lq.locality_order(rp, c.astype(np.int32), 100)
    assert np.array_equal(np.sort(o), np.arange(n))


def test_bad_input_is_rejected():
    N, rp, ci = cubic_pattern(4)
    bad = ci.copy()
    bad[5] = N
    with pytest.raises(lq.LinqtError):
        lq.locality_order(rp, bad, 8)
    with pytest.raises(lq.LinqtError):
        lq.locality_order(rp, ci, 0)
    rp2 = rp.copy()
    rp2[3] = rp2[2] - 1
    with pytest.raises(lq.LinqtError):
        lq.locality_order(rp2, ci, 8)
