"""GPU parity: the CUDA path (through the C ABI) against the C oracle.

FP64 tolerance: max |GPU - oracle| / max |oracle| <= 1e-10 for moments and
conductivities (summation orders differ; the reference's own tables are printed
with 15 digits).  Inputs are seeded synthetic lattices small enough for the oracle
to finish in seconds.
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


def bounds_of(N, csr, pad=1.05):
    lo, hi = lattices.gershgorin_bounds(N, *csr)
    return pad * (hi - lo), (hi + lo) / 2


def gpu_op(N, csr, bw=None, bc=None):
    op = lq.Operator.from_csr(N, *csr)
    if bw is not None:
        op.rescale_to_chebyshev(bw, bc)
    return op


def oracle_op(orc, csr, bw=None, bc=None):
    op = orc.Op(*csr)
    if bw is not None:
        op.rescale(2 / bw, -bc / (bw / 2))
    return op


@pytest.fixture(scope="module")
def honey(oracle_lib):
    N, H, V = lattices.honeycomb(8, 6, t=-2.7, W=1.0, seed=21)
    bw, bc = bounds_of(N, H)
    return dict(N=N, H=H, V=V, bw=bw, bc=bc, Hg=gpu_op(N, H, bw, bc), Vg=gpu_op(N, V),
                Ho=oracle_op(oracle_lib, H, bw, bc), Vo=oracle_op(oracle_lib, V))


@pytest.fixture(scope="module")
def square(oracle_lib):
    N, H = lattices.square_lattice(24, t=1.0, W=1.0, seed=11)
    bw, bc = 2 * 1.05 * 4.5, 0.0
    return dict(N=N, H=H, bw=bw, bc=bc, Hg=gpu_op(N, H, bw, bc), Ho=oracle_op(oracle_lib, H, bw, bc))


def test_operator_info_and_rescale(square):
    N = square["N"]
    n, nnz = square["Hg"].info()
    assert n == N and nnz == 5 * N


@pytest.mark.parametrize("ncols", [1, 3, 8])
def test_multiply_matches_oracle(oracle_lib, honey, ncols):
    rng = np.random.default_rng(5)
    N = honey["N"]
    x = rng.normal(size=(N, ncols)) + 1j * rng.normal(size=(N, ncols))
    y = rng.normal(size=(N, ncols)) + 1j * rng.normal(size=(N, ncols))
    a, b = 2.0 - 0.5j, -1.0 + 0.25j
    got = honey["Vg"].multiply(x, a=a, b=b, y=y)
    want = np.stack([honey["Vo"].mv(x[:, c], a=a, b=b, y=y[:, c]) for c in range(ncols)], axis=1)
    assert rel(got, want) < 1e-13


def test_hermitian_upper_semantics(oracle_lib):
    # strictly lower entries are ignored; the lower triangle is conj(upper)
    n = 5
    rp = np.array([0, 3, 5, 6, 8, 9], np.int32)
    col = np.array([0, 2, 4, 0, 1, 3, 3, 1, 4], np.int32)  # row 1 col 0 and row 3 col 1 are lower: dropped
    val = (np.arange(9) + 1) + 1j * (np.arange(9) - 4)
    val[[0, 4, 6, 8]] = val[[0, 4, 6, 8]].real  # real diagonal
    g = lq.Operator.from_csr(n, rp, col, val)
    o = oracle_lib.Op(rp, col, val)
    x = np.arange(n) + 1j
    assert rel(g.multiply(x), o.mv(x)) < 1e-14
    assert g.nnz == o.nnz


def test_spectral_bounds(honey):
    lo, hi = honey["Hg"].spectral_bounds()
    # after rescaling to (-1/1.05, 1/1.05) Gershgorin stays inside [-1, 1]
    assert -1.0 < lo < 0 < hi < 1.0


@pytest.mark.parametrize("R", [1, 3, 40])
@pytest.mark.parametrize("doubling", [0, 2])
@pytest.mark.parametrize("step_launches", [0, 1])
def test_moments1d_identity(oracle_lib, square, R, doubling, step_launches):
    st = lattices.random_phase_states(square["N"], R, seed=12)
    M = 200
    got = lq.moments1d(square["Hg"], None, st, M, opts=lq.make_opts(doubling=doubling, step_launches=step_launches))
    want = oracle_lib.moments1d(square["Ho"], None, st, M)
    assert rel(got, want) < TOL
    assert abs(got[0] - 1.0) < 1e-12  # normalised states: mu_0 = 1


@pytest.mark.parametrize("step_launches", [0, 1])
def test_moments1d_with_operator(oracle_lib, honey, step_launches):
    st = lattices.random_phase_states(honey["N"], 2, seed=7)
    M = 96
    got = lq.moments1d(honey["Hg"], honey["Vg"], st, M, opts=lq.make_opts(step_launches=step_launches))
    want = oracle_lib.moments1d(honey["Ho"], honey["Vo"], st, M)
    assert rel(got, want) < TOL


def test_moments1d_default_state_odd_M(oracle_lib, square):
    from linqt_b200.formats import default_state
    st = default_state(square["N"])
    got = lq.moments1d(square["Hg"], None, st, 101)
    want = oracle_lib.moments1d(square["Ho"], None, st, 101)
    assert rel(got, want) < TOL


@pytest.mark.parametrize("R,M", [(1, 40), (3, 64), (5, 33), (64, 16)])
@pytest.mark.parametrize("step_launches", [0, 1])
def test_moments2d_velocity(oracle_lib, honey, R, M, step_launches):
    st = lattices.random_phase_states(honey["N"], R, seed=22)
    got = lq.moments2d(honey["Hg"], honey["Vg"], honey["Vg"], st, M, opts=lq.make_opts(step_launches=step_launches))
    want = oracle_lib.moments2d(honey["Ho"], honey["Vo"], honey["Vo"], st, M)
    assert rel(got, want) < TOL
    assert np.abs(got - got.conj().T).max() < 1e-14 * np.abs(got).max()


@pytest.mark.parametrize("step_launches", [0, 1])
def test_moments2d_identity_operators(oracle_lib, honey, step_launches):
    st = lattices.random_phase_states(honey["N"], 2, seed=3)
    M = 48
    got = lq.moments2d(honey["Hg"], None, None, st, M, opts=lq.make_opts(step_launches=step_launches))
    want = oracle_lib.moments2d(honey["Ho"], None, None, st, M)
    assert rel(got, want) < TOL


def test_moments2d_chunked_equals_unchunked(honey):
    st = lattices.random_phase_states(honey["N"], 6, seed=4)
    M = 40
    full = lq.moments2d(honey["Hg"], honey["Vg"], honey["Vg"], st, M)
    chunked = lq.moments2d(honey["Hg"], honey["Vg"], honey["Vg"], st, M, opts=lq.make_opts(block_width=2))
    assert rel(chunked, full) < 1e-13


def test_moments2d_golden_linear_chain(golden):
    """The reference's shipped table (M=100, bounds -5..5, default state) reproduced on the GPU."""
    N = len(golden["HAM_rowptr"]) - 1
    H = lq.Operator.from_csr(N, golden["HAM_rowptr"], golden["HAM_col"],
                             golden["HAM_val"][0::2] + 1j * golden["HAM_val"][1::2])
    V = lq.Operator.from_csr(N, golden["VX_rowptr"], golden["VX_col"],
                             golden["VX_val"][0::2] + 1j * golden["VX_val"][1::2])
    H.rescale_to_chebyshev(10.0, 0.0)
    st = np.zeros((1, N), np.complex128)
    st[0, N // 2] = 1
    mu = lq.moments2d(H, V, V, st, 100)
    g = golden["mu100"]
    ref = g[..., 0] + 1j * g[..., 1]
    assert rel(mu, ref) < 1e-13


@pytest.mark.parametrize("formula,nump", [(lq.KUBO_BASTIN, 256), (lq.KUBO_GREENWOOD, 256), (lq.KUBO_BASTIN, 512),
                                          (lq.KUBO_BASTIN, 1024), (lq.KUBO_GREENWOOD, 2048),
                                          (lq.KUBO_BASTIN, 100), (lq.KUBO_GREENWOOD, 90)])
def test_kubo_fft(oracle_lib, honey, formula, nump):
    R = 2
    M = min(64, nump)
    st = lattices.random_phase_states(honey["N"], R, seed=9)
    E, s, integ = lq.kubo_fft(honey["Hg"], honey["Vg"], honey["Vg"], st, M, nump, formula, honey["bw"], honey["bc"])
    Eo, so, io, _ = oracle_lib.kubo_fft(honey["Ho"], honey["Vo"], honey["Vo"], st, M, nump, formula, honey["N"],
                                        honey["bw"], honey["bc"])
    assert rel(E, Eo) < 1e-14
    assert rel(s, so) < TOL
    if formula == lq.KUBO_BASTIN:
        assert rel(integ, io) < TOL


def test_kubo_bastin_combined_equals_separate(honey):
    st = lattices.random_phase_states(honey["N"], 3, seed=31)
    M, nump = 48, 256
    mu, (E, s, integ) = lq.kubo_bastin(honey["Hg"], honey["Vg"], honey["Vg"], st, M, nump, honey["bw"], honey["bc"])
    mu2 = lq.moments2d(honey["Hg"], honey["Vg"], honey["Vg"], st, M)
    E2, s2, i2 = lq.kubo_fft(honey["Hg"], honey["Vg"], honey["Vg"], st, M, nump, lq.KUBO_BASTIN, honey["bw"],
                             honey["bc"])
    assert np.array_equal(mu, mu2)  # same kernels, same order: bitwise
    assert np.array_equal(s, s2) and np.array_equal(E, E2) and np.array_equal(integ, i2)


@pytest.fixture(scope="module")
def diag_op(oracle_lib, honey):
    """A second operator (diagonal, random) so that OPL != OPR."""
    N = honey["N"]
    D = lattices.upper_csr(N, np.arange(N), np.arange(N), lattices.disorder(N, 2.0, 5) + 0j)
    return dict(Dg=gpu_op(N, D), Do=oracle_op(oracle_lib, D))


def test_moments2d_distinct_operators(oracle_lib, honey, diag_op):
    st = lattices.random_phase_states(honey["N"], 3, seed=44)
    M = 48
    got = lq.moments2d(honey["Hg"], honey["Vg"], diag_op["Dg"], st, M)
    want = oracle_lib.moments2d(honey["Ho"], honey["Vo"], diag_op["Do"], st, M)
    assert rel(got, want) < TOL
    swapped = lq.moments2d(honey["Hg"], diag_op["Dg"], honey["Vg"], st, M)
    assert rel(swapped, want) > 1e-3


@pytest.mark.parametrize("formula", [lq.KUBO_BASTIN, lq.KUBO_GREENWOOD])
def test_kubo_fft_distinct_operators(oracle_lib, honey, diag_op, formula):
    st = lattices.random_phase_states(honey["N"], 2, seed=45)
    M, nump = 48, 256
    E, s, integ = lq.kubo_fft(honey["Hg"], honey["Vg"], diag_op["Dg"], st, M, nump, formula, honey["bw"],
                              honey["bc"])
    Eo, so, io, _ = oracle_lib.kubo_fft(honey["Ho"], honey["Vo"], diag_op["Do"], st, M, nump, formula, honey["N"],
                                        honey["bw"], honey["bc"])
    assert rel(s, so) < TOL
    mu, (E2, s2, i2) = lq.kubo_bastin(honey["Hg"], honey["Vg"], diag_op["Dg"], st, M, nump, honey["bw"],
                                      honey["bc"])
    if formula == lq.KUBO_BASTIN:
        assert np.array_equal(s, s2)
        assert rel(mu, oracle_lib.moments2d(honey["Ho"], honey["Vo"], diag_op["Do"], st, M)) < TOL


def test_dos_from_moments(oracle_lib, square):
    st = lattices.random_phase_states(square["N"], 2, seed=12)
    M = 256
    mu = lq.moments1d(square["Hg"], None, st, M)
    E, d = lq.dos_from_moments(mu, square["N"], square["bw"], square["bc"], broad_meV=10.0)
    muj = oracle_lib.jackson1d(mu, square["bw"], 10.0)
    Eo, do = oracle_lib.dos_fftgrid(muj, square["N"], square["bw"], square["bc"])
    assert len(E) == len(Eo)
    assert rel(E, Eo) < 1e-14
    assert rel(d, do) < 1e-11


@pytest.mark.parametrize("M,b,bw", [(100, 100.0, 10.0), (300, 50.0, 4.9)])
def test_bastin_golden(golden, oracle_lib, M, b, bw):
    """kuboBastinFromChebmom on the shipped tables (written with xbound 0.9)."""
    g = golden["mu%d" % M]
    mu = g[..., 0] + 1j * g[..., 1]
    N = int(golden["mu%d_header" % M][0])
    E, s = lq.bastin_from_moments(mu, N, bw, 0.0, b, xbound=0.9)
    ref = golden["bastin%d" % M]
    assert len(E) == len(ref)
    assert np.abs(E - ref[:, 0]).max() < 1e-5  # file has 6 significant digits
    assert rel(s, ref[:, 1]) < 2e-6
    muj = oracle_lib.jackson2d(mu, bw, b, b)
    Eo, so = oracle_lib.bastin_from_moments(muj, N, bw, 0.0, xbound=0.9)
    assert rel(s, so) < 1e-11


def test_device_pointer_api_matches_host(honey):
    torch = pytest.importorskip("torch")
    st = lattices.random_phase_states(honey["N"], 4, seed=1)
    M = 32
    host = lq.moments2d(honey["Hg"], honey["Vg"], honey["Vg"], st, M)
    dst = torch.from_numpy(st.view(np.float64).copy()).cuda()
    dmu = torch.zeros(2 * M * M, dtype=torch.float64, device="cuda")
    sess = lq.Session(0)
    sess.set_stream(torch.cuda.current_stream())
    lq.moments2d_dev(honey["Hg"], honey["Vg"], honey["Vg"], dst, 4, M, dmu, session=sess)
    torch.cuda.synchronize()
    dev = dmu.cpu().numpy().view(np.complex128).reshape(M, M)
    assert rel(dev, host) < 1e-14


def test_errors_are_reported(honey):
    with pytest.raises(lq.LinqtError) as e:
        lq.kubo_fft(honey["Hg"], honey["Vg"], honey["Vg"], np.ones((1, honey["N"])), 64, 32, lq.KUBO_BASTIN,
                    honey["bw"], honey["bc"])
    assert e.value.code == -1 and "nump" in str(e.value)
    with pytest.raises(lq.LinqtError):
        lq.Operator.from_csr(3, [0, 1, 2, 3], [0, 1, 5], [1.0, 1.0, 1.0])
    with pytest.raises(lq.LinqtError) as e:  # unknown sparse format
        lq.moments1d(honey["Hg"], None, np.ones((1, honey["N"])), 8, opts=lq.make_opts(fmt=7))
    assert e.value.code == -1 and "format" in str(e.value)


# ---------------------------------------------------------------------------
# precision modes: FP32 recursion + FP64 contraction (PREC_FP32) and FP32 recursion +
# tcgen05 INT8 contraction of 4-digit splits (PREC_MIXED).  Bounds sit one order of
# magnitude above the measured accuracy of the modes (FP32 recursion ~1e-8 of max|mu| at
# these sizes, the INT8 contraction of the same blocks ~1e-8), checked against the FP64 path.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("R,M", [(2, 32), (3, 100), (8, 130)])
def test_mixed_precision_moments2d(honey, R, M):
    st = lattices.random_phase_states(honey["N"], R, seed=22)
    m64 = lq.moments2d(honey["Hg"], honey["Vg"], honey["Vg"], st, M)
    m32 = lq.moments2d(honey["Hg"], honey["Vg"], honey["Vg"], st, M, opts=lq.make_opts(precision=lq.PREC_FP32))
    mmx = lq.moments2d(honey["Hg"], honey["Vg"], honey["Vg"], st, M, opts=lq.make_opts(precision=lq.PREC_MIXED))
    assert rel(m32, m64) < 1e-6      # FP32 recursion
    assert rel(mmx, m32) < 1e-7      # tensor-core contraction of the same FP32 blocks
    assert rel(mmx, m64) < 1e-6
    assert np.abs(mmx - mmx.conj().T).max() < 1e-12 * np.abs(mmx).max()


def test_mixed_precision_large_k_multi_pass():
    """K = 2 * 16384 * 32 floats: several K passes of the tensor-core kernel."""
    N, H, V = lattices.honeycomb(128, 64, t=-2.7, W=1.0, seed=21)
    bw, bc = bounds_of(N, H)
    Hg, Vg = gpu_op(N, H, bw, bc), gpu_op(N, V)
    st = lattices.random_phase_states(N, 32, seed=22)
    M = 16
    m32 = lq.moments2d(Hg, Vg, Vg, st, M, opts=lq.make_opts(precision=lq.PREC_FP32))
    mmx = lq.moments2d(Hg, Vg, Vg, st, M, opts=lq.make_opts(precision=lq.PREC_MIXED))
    assert rel(mmx, m32) < 1e-7


@pytest.mark.parametrize("precision", [lq.PREC_FP32, lq.PREC_MIXED])
def test_mixed_precision_kubo_bastin(honey, precision):
    st = lattices.random_phase_states(honey["N"], 4, seed=9)
    M, nump = 64, 256
    mu64, (E64, s64, _) = lq.kubo_bastin(honey["Hg"], honey["Vg"], honey["Vg"], st, M, nump, honey["bw"], honey["bc"])
    mu, (E, s, _) = lq.kubo_bastin(honey["Hg"], honey["Vg"], honey["Vg"], st, M, nump, honey["bw"], honey["bc"],
                                   opts=lq.make_opts(precision=precision))
    assert np.array_equal(E, E64)
    assert rel(s, s64) < 1e-6
    assert rel(mu, mu64) < 1e-6
