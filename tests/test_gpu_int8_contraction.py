"""The mixed-precision moment contraction on the INT8 tensor cores: FP32 Chebyshev blocks
split into 7-bit digits under a shared exponent per row and K chunk, products accumulated
exactly in INT32.  PREC_MIXED keeps 4 digits (28 bits of each row chunk's range),
PREC_MIXED_FAST 3 digits (21 bits).

Bounds, against the FP64 MMA contraction of the same FP32 blocks (PREC_FP32): the digit
truncation (half a unit of the last digit of each row chunk's largest value, per operand)
stays below 1e-7 (4 digits) and 1e-6 (3 digits) of max|mu| even for short rows (K ~ 100,
where nothing averages out).  Against the FP64 path, sigma reconstructed from the PREC_MIXED
moment table by the Bastin energy sum stays below 1e-6 of its maximum over the interior
90 % of the window.  The 3xTF32 form (PREC_MIXED_TF32) stays available with its 1e-4 bound.
"""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


def _ops(N, H, V):
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    return Hg, lq.Operator.from_csr(N, *V), bw, bc


@pytest.fixture(scope="module")
def honey():
    N, H, V = lattices.honeycomb(8, 6, t=-2.7, W=1.0, seed=21)
    Hg, Vg, bw, bc = _ops(N, H, V)
    return dict(N=N, H=Hg, V=Vg, bw=bw, bc=bc)


@pytest.mark.parametrize("prec,tol", [(lq.PREC_MIXED, 1e-7), (lq.PREC_MIXED_FAST, 1e-6)])
@pytest.mark.parametrize("R,M", [(1, 16), (2, 32), (3, 100), (8, 130), (5, 257)])
def test_int8_contraction_matches_fp64_mma_of_the_same_blocks(honey, R, M, prec, tol):
    """Ragged sizes: M not a multiple of the 128 x 64 output tile, K = N R padded to the
    128-byte K block."""
    st = lattices.random_phase_states(honey["N"], R, seed=22)
    m32 = lq.moments2d(honey["H"], honey["V"], honey["V"], st, M, opts=lq.make_opts(precision=lq.PREC_FP32))
    mmx = lq.moments2d(honey["H"], honey["V"], honey["V"], st, M, opts=lq.make_opts(precision=prec))
    assert rel(mmx, m32) < tol
    assert np.abs(mmx - mmx.conj().T).max() < 1e-12 * np.abs(mmx).max()


def test_int8_contraction_repeats_bitwise(honey):
    st = lattices.random_phase_states(honey["N"], 4, seed=23)
    o = lq.make_opts(precision=lq.PREC_MIXED)
    a = lq.moments2d(honey["H"], honey["V"], honey["V"], st, 64, opts=o)
    b = lq.moments2d(honey["H"], honey["V"], honey["V"], st, 64, opts=o)
    assert np.array_equal(a, b)


def test_int8_contraction_several_passes():
    """K = 32768 sites x 256 vectors = 8.4e6 complex: 128 K chunks of 131072 bytes, two
    passes of 64 chunks through the partial tiles."""
    N, H, V = lattices.honeycomb(128, 128, t=-2.7, W=1.0, seed=21)
    Hg, Vg, _, _ = _ops(N, H, V)
    st = lattices.random_phase_states(N, 256, seed=24)
    M = 8
    m32 = lq.moments2d(Hg, Vg, Vg, st, M, opts=lq.make_opts(precision=lq.PREC_FP32))
    for prec, tol in ((lq.PREC_MIXED, 1e-7), (lq.PREC_MIXED_FAST, 1e-6)):
        mmx = lq.moments2d(Hg, Vg, Vg, st, M, opts=lq.make_opts(precision=prec))
        assert rel(mmx, m32) < tol


def test_tf32_contraction_still_available(honey):
    st = lattices.random_phase_states(honey["N"], 8, seed=25)
    m32 = lq.moments2d(honey["H"], honey["V"], honey["V"], st, 130, opts=lq.make_opts(precision=lq.PREC_FP32))
    mtf = lq.moments2d(honey["H"], honey["V"], honey["V"], st, 130, opts=lq.make_opts(precision=lq.PREC_MIXED_TF32))
    assert rel(mtf, m32) < 1e-4


def test_sigma_from_mixed_moments_within_1e6():
    """Kane-Mele spin conductivity from the 2D moment table (kuboBastinFromChebmom, every
    moment kept): the mixed solve against the FP64 solve."""
    N, H, J = lattices.kane_mele(16, 16, seed=31)
    Hg, Jg, bw, bc = _ops(N, H, J)
    st = lattices.random_phase_states(N, 8, seed=32)
    M = 256
    mu64 = lq.moments2d(Hg, Jg, Jg, st, M)
    mumx = lq.moments2d(Hg, Jg, Jg, st, M, opts=lq.make_opts(precision=lq.PREC_MIXED))
    E64, s64 = lq.bastin_from_moments(mu64, N, bw, bc, 1e-3, xbound=0.99)
    Emx, smx = lq.bastin_from_moments(mumx, N, bw, bc, 1e-3, xbound=0.99)
    assert np.array_equal(E64, Emx)
    lo, hi = int(0.05 * len(s64)), int(0.95 * len(s64))
    assert rel(smx[lo:hi], s64[lo:hi]) < 1e-6
