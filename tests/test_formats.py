"""LinQT file formats: the .chebmom2D write/read round trip the reference's only unit
test intends (test/chebyshev_moments.cpp), byte layout of the headers, CSR and state files."""
import os

import numpy as np

from linqt_b200 import formats


def test_chebmom2d_roundtrip(tmp_path):
    rng = np.random.default_rng(1)
    mu = rng.normal(size=(7, 5)) + 1j * rng.normal(size=(7, 5))
    p = str(tmp_path / "x.chebmom2D")
    formats.write_chebmom2d(p, 100, 4.9, 0.25, mu)
    n, bw, bc, back = formats.read_chebmom2d(p)
    assert (n, bw, bc) == (100, 4.9, 0.25)
    assert np.abs(back - mu).max() <= 1e-14 * np.abs(mu).max()
    lines = open(p).read().split("\n")
    assert lines[0] == "100 4.9  0.25"  # two spaces before the band centre
    assert lines[1] == "7 5 "            # trailing space after the moment counts


def test_chebmom1d_roundtrip(tmp_path):
    mu = np.array([1.0, 0.5 - 0.25j, -0.0, 1e-300])
    p = str(tmp_path / "y.chebmom1D")
    formats.write_chebmom1d(p, 64, 9.45, 0.0, mu)
    n, bw, bc, back = formats.read_chebmom1d(p)
    assert (n, bw, bc) == (64, 9.45, 0.0)
    assert np.array_equal(back, mu)
    assert open(p).read().split("\n")[2] == "1 0"


def test_golden_header_layout_matches_writer(golden, tmp_path):
    g = golden["mu100"]
    mu = np.empty(g.shape[:2], np.complex128)
    mu.real, mu.imag = g[..., 0], g[..., 1]  # keeps the signed zero of mu(0,0)
    p = str(tmp_path / "g.chebmom2D")
    formats.write_chebmom2d(p, 20000, 10.0, 0.0, mu)
    head = open(p).read().split("\n")[:3]
    assert head == ["20000 10  0", "100 100 ", "2 -0"]  # first lines of the shipped table


def test_csr_roundtrip(tmp_path, golden):
    rp, cl, vl = golden["HAM_rowptr"], golden["HAM_col"], golden["HAM_val"]
    p = str(tmp_path / "h.CSR")
    formats.write_csr(p, len(rp) - 1, rp, cl, vl[0::2] + 1j * vl[1::2])
    n, rp2, cl2, vl2 = formats.read_csr(p)
    assert n == len(rp) - 1
    assert np.array_equal(rp, rp2) and np.array_equal(cl, cl2)
    assert np.array_equal(vl2, vl[0::2] + 1j * vl[1::2])


def test_state_files(tmp_path):
    st = np.array([[1, 2j, 3], [0.5, -1, 1e-17]], np.complex128)
    p = str(tmp_path / "s")
    formats.write_vector_states(p, st)
    assert np.array_equal(formats.read_state_file(p), st)
    q = str(tmp_path / "l")
    open(q, "w").write("local\n2\n0 3\n")
    loc = formats.read_state_file(q, dim=4)
    assert loc[0, 0] == 1 and loc[1, 3] == 1 and loc.sum() == 2
    d = formats.default_state(10)
    assert d[0, 5] == 1 and d.sum() == 1
