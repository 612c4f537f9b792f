"""The restated post-processors (lo_kubo_from_moments) against LinQT's own drivers built from
its sources (oracle/_ref): kuboBastinFromChebmom{,_FFTgrid}, kuboGreenwoodFromChebmom{,_FFTgrid},
kuboBastin{I,II,Sea,Surf}FromChebmom.  The drivers print 6 significant digits.  Several of them
fix the energy window at +-1 (CUTOFF), where the first point divides by zero: those entries are
non-finite in both; the Bastin II and sea sums then stay non-finite along their running
integral, so their values are compared through ref_harness's `frommom` mode on a window of
+-0.99, which evaluates the same sums with the reference's own coefficient functions."""
import os
import subprocess

import numpy as np
import pytest

from linqt_b200 import formats, lattices

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
BROAD = 60.0

# driver, output file prefix, variant, grid, xbound
DRIVERS = [
    ("inline_kuboBastinFromChebmom", "KuboBastin_", "bastin", 0, 0.99),
    ("inline_kuboGreenwoodFromChebmom", "KuboGreenWood_", "greenwood", 0, 1.0),
    ("inline_kuboBastinIFromChebmom", "KuboBastinI_", "bastin_I", 0, 1.0),
    ("inline_kuboBastinIIFromChebmom", "KuboBastinII_", "bastin_II", 0, 1.0),
    ("inline_kuboBastinSeaFromChebmom", "KuboBastinSea_", "bastin_sea", 0, 1.0),
    ("inline_kuboBastinSurfFromChebmom", "KuboBastinSurf_", "bastin_surf", 0, 1.0),
    ("inline_kuboGreenwoodFromChebmom_FFTgrid", "KuboGreenWood_", "greenwood", 1, 1.0),
    ("inline_kuboBastinFromChebmom_FFTgrid", "KuboBastin_", "bastin", 2, 1.0),
]


@pytest.fixture(scope="module")
def table(oracle_lib, tmp_path_factory):
    """A graphene V_x-V_x table (R = 2, M = 48) written as LinQT's .chebmom2D."""
    N, H, V = lattices.honeycomb(6, 5, t=-2.7, W=1.0, seed=21)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    Ho = oracle_lib.Op(*H).rescale(2 / bw, -bc / (bw / 2))
    Vo = oracle_lib.Op(*V)
    mu = oracle_lib.moments2d(Ho, Vo, Vo, lattices.random_phase_states(N, 2, seed=22), 48)
    d = tmp_path_factory.mktemp("frommom")
    path = str(d / "grVX.chebmom2D")
    formats.write_chebmom2d(path, N, bw, bc, mu)
    n, bw2, bc2, mu2 = formats.read_chebmom2d(path)  # what the drivers read (15 digits)
    return d, path, n, bw2, bc2, oracle_lib.jackson2d(mu2, bw2, BROAD, BROAD)


def _run_driver(exe, d, path):
    if not os.path.exists(os.path.join(REF, exe)):
        pytest.skip("reference driver not built")
    # relative name: the drivers build their output name from it
    p = subprocess.run([os.path.join(REF, exe), os.path.basename(path), str(BROAD)], cwd=str(d),
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-1000:]


@pytest.mark.parametrize("exe,prefix,variant,grid,xbound", DRIVERS)
def test_post_processor_vs_reference_driver(oracle_lib, table, exe, prefix, variant, grid, xbound):
    d, path, n, bw, bc, muj = table
    _run_driver(exe, d, path)
    suffix = "JACKSON_FFTgrid.dat" if grid else "JACKSON.dat"
    ref = np.loadtxt(str(d / (prefix + "grVX" + suffix)))
    E, out = oracle_lib.kubo_from_moments(muj, n, bw, bc, variant, grid=grid, xbound=xbound)
    assert ref.shape == (len(E), 2)
    assert np.allclose(E, ref[:, 0], rtol=1e-5, atol=1e-5 * np.abs(E).max())
    fin = np.isfinite(ref[:, 1])
    assert np.array_equal(fin, np.isfinite(out))  # the same points divide by zero
    if fin.any():
        scale = np.abs(ref[fin, 1]).max()
        assert np.abs(out[fin] - ref[fin, 1]).max() <= 2e-6 * scale


@pytest.mark.parametrize("name,variant", [("II", "bastin_II"), ("Sea", "bastin_sea")])
def test_bastin_II_and_sea_sums_vs_reference(oracle_lib, table, name, variant):
    d, path, n, bw, bc, muj = table
    if not oracle_lib.ref_available():
        pytest.skip("reference harness not built")
    out = oracle_lib.run_ref_harness(["frommom", name, os.path.basename(path), BROAD, 0.99, 0], str(d))
    ref = np.loadtxt(os.path.join(str(d), out["out"]))
    E, o = oracle_lib.kubo_from_moments(muj, n, bw, bc, variant, xbound=0.99)
    assert np.all(np.isfinite(o))
    assert np.abs(E - ref[:, 0]).max() <= 1e-12 * np.abs(E).max()
    assert np.abs(o - ref[:, 1]).max() <= 1e-10 * np.abs(ref[:, 1]).max()


# spectralFunctionFromChebmom (uniform grid of 30 M' points in [-1, 1], raw sums, the end
# points divide by zero) and spectralFunctionFromChebmom_FFTgrid (M' Chebyshev points,
# absolute values): driver, output suffix, grid
SPECTRAL = [("inline_spectralFunctionFromChebmom", "JACKSON.dat", 0),
            ("inline_spectralFunctionFromChebmom_FFTgrid", "JACKSON_FFTgrid.dat", 1)]


@pytest.fixture(scope="module")
def table1d(oracle_lib, tmp_path_factory):
    """Square-lattice DOS moments (R = 2, M = 200) written as LinQT's .chebmom1D."""
    N, H = lattices.square_lattice(16, t=1.0, W=1.0, seed=11)
    bw, bc = 2 * 1.05 * 4.5, 0.0
    Ho = oracle_lib.Op(*H).rescale(2 / bw, -bc / (bw / 2))
    mu = oracle_lib.moments1d(Ho, None, lattices.random_phase_states(N, 2, seed=12), 200)
    d = tmp_path_factory.mktemp("frommom1d")
    path = str(d / "sqDOS.chebmom1D")
    formats.write_chebmom1d(path, N, bw, bc, mu)
    n, bw2, bc2, mu2 = formats.read_chebmom1d(path)  # what the drivers read (15 digits)
    return d, path, n, bw2, bc2, oracle_lib.jackson1d(mu2, bw2, BROAD)


@pytest.mark.parametrize("exe,suffix,grid", SPECTRAL)
def test_spectral_function_vs_reference_driver(oracle_lib, table1d, exe, suffix, grid):
    d, path, n, bw, bc, muj = table1d
    _run_driver(exe, d, path)
    ref = np.loadtxt(str(d / ("meansqDOS" + suffix)))
    E, out = oracle_lib.spectral_function(muj, n, bw, bc, grid=grid)
    assert ref.shape == (len(E), 2)
    assert np.allclose(E, ref[:, 0], rtol=1e-5, atol=1e-5 * np.abs(E).max())
    fin = np.isfinite(ref[:, 1])
    assert np.array_equal(fin, np.isfinite(out))  # the same points divide by zero
    assert fin.sum() >= len(E) - 2
    scale = np.abs(ref[fin, 1]).max()
    assert np.abs(out[fin] - ref[fin, 1]).max() <= 2e-6 * scale


def test_dos_fftgrid_equals_spectral_function_fftgrid(oracle_lib, table1d):
    """lo_dos_fftgrid (the checker of linqt_dos_from_moments) is the _FFTgrid driver's sum."""
    d, path, n, bw, bc, muj = table1d
    E1, d1 = oracle_lib.dos_fftgrid(muj, n, bw, bc)
    E2, d2 = oracle_lib.spectral_function(muj, n, bw, bc, grid=1)
    assert np.array_equal(E1, E2) and np.array_equal(d1, d2)
