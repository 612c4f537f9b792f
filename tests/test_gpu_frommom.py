"""LinQT's energy-sum post-processors (kubo*FromChebmom*) on the GPU against the oracle
restatement (itself pinned against the reference's drivers in test_oracle_frommom_vs_ref.py)."""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu
BROAD = 60.0
VARIANTS = ["bastin", "greenwood", "bastin_I", "bastin_II", "bastin_sea", "bastin_surf"]


@pytest.fixture(scope="module")
def table(oracle_lib):
    N, H, V = lattices.honeycomb(8, 6, t=-2.7, W=1.0, seed=21)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    Vg = lq.Operator.from_csr(N, *V)
    mu = lq.moments2d(Hg, Vg, Vg, lattices.random_phase_states(N, 2, seed=22), 64)
    return N, bw, bc, mu, oracle_lib.jackson2d(mu, bw, BROAD, BROAD)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("grid", [lq.GRID_UNIFORM, lq.GRID_CHEBYSHEV, lq.GRID_CHEBYSHEV_ASCENDING])
def test_energy_sums_match_oracle(oracle_lib, table, variant, grid):
    N, bw, bc, mu, muj = table
    E, out = lq.kubo_from_moments(mu, N, bw, bc, BROAD, variant=variant, grid=grid, xbound=0.99)
    Eo, oo = oracle_lib.kubo_from_moments(muj, N, bw, bc, variant, grid=grid, xbound=0.99)
    assert len(E) == len(Eo)
    assert np.abs(E - Eo).max() <= 1e-14 * np.abs(Eo).max()
    assert np.all(np.isfinite(out))
    assert np.abs(out - oo).max() <= 1e-10 * np.abs(oo).max()


@pytest.mark.parametrize("variant", VARIANTS[1:])
def test_energy_sums_at_the_drivers_window(oracle_lib, table, variant):
    """xbound = 1 as the drivers use it: the same points are non-finite, the rest agree."""
    N, bw, bc, mu, muj = table
    E, out = lq.kubo_from_moments(mu, N, bw, bc, BROAD, variant=variant, xbound=1.0)
    Eo, oo = oracle_lib.kubo_from_moments(muj, N, bw, bc, variant, xbound=1.0)
    fin = np.isfinite(oo)
    assert np.array_equal(np.isfinite(out), fin)
    if fin.any():
        assert np.abs(out[fin] - oo[fin]).max() <= 1e-10 * np.abs(oo[fin]).max()


def test_bastin_entry_point_is_the_bastin_variant(table):
    N, bw, bc, mu, _ = table
    E1, s1 = lq.bastin_from_moments(mu, N, bw, bc, BROAD, xbound=0.99)
    E2, s2 = lq.kubo_from_moments(mu, N, bw, bc, BROAD, variant="bastin", xbound=0.99)
    assert np.array_equal(E1, E2) and np.array_equal(s1, s2)


@pytest.mark.parametrize("grid,num_div", [(0, 0), (1, 0), (0, 777)])
def test_spectral_function_from_moments(oracle_lib, grid, num_div):
    """spectralFunctionFromChebmom (uniform grid, raw sums, end points non-finite) and its
    _FFTgrid variant (absolute values) against the oracle, which is pinned to both reference
    drivers (tests/test_oracle_frommom_vs_ref.py)."""
    N, H = lattices.square_lattice(24, t=1.0, W=1.0, seed=11)
    bw, bc = 2 * 1.05 * 4.5, 0.1
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    mu = lq.moments1d(Hg, None, lattices.random_phase_states(N, 3, seed=12), 300)
    E, out = lq.spectral_function_from_moments(mu, N, bw, bc, 40.0, grid=grid, num_div=num_div)
    muj = oracle_lib.jackson1d(mu, bw, 40.0)
    Eo, oo = oracle_lib.spectral_function(muj, N, bw, bc, grid=grid, num_div=num_div or None)
    assert len(E) == len(Eo) == (num_div or (30 * len(muj) if grid == 0 else len(muj)))
    assert np.abs(E - Eo).max() <= 1e-14 * np.abs(Eo).max()
    fin = np.isfinite(oo)
    assert np.array_equal(fin, np.isfinite(out))
    assert fin.sum() == len(E) - (2 if grid == 0 else 0)
    assert np.abs(out[fin] - oo[fin]).max() <= 1e-11 * np.abs(oo[fin]).max()
