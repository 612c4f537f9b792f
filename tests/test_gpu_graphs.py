"""opts.use_graphs: the device-pointer solves replayed from CUDA graphs give the same bits as
the same solves enqueued eagerly.

The first call with a given set of pointers, sizes and operators runs eagerly, the second is
captured and launched, later ones replay.  New contents in the same buffers are picked up by
the replay; a rescaled operator or another output buffer is a new key and is captured anew.
"""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).reshape(-1).copy()).cuda()


@pytest.fixture(scope="module")
def honey():
    N, H, V = lattices.honeycomb(16, 12, t=-2.7, W=1.0, seed=21)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    return dict(N=N, H=Hg, V=lq.Operator.from_csr(N, *V), bw=bw, bc=bc)


def _solve(kind, h, st, R, M, out, opts, sess, mu=None):
    if kind == "m1":
        lq.moments1d_dev(h["H"], h["V"], st, R, M, out, opts=opts, session=sess)
    elif kind == "m2":
        lq.moments2d_dev(h["H"], h["V"], h["V"], st, R, M, out, opts=opts, session=sess)
    elif kind == "kf":
        lq.kubo_fft_dev(h["H"], h["V"], h["V"], st, R, M, 256, lq.KUBO_BASTIN, h["bw"], h["bc"], out, opts=opts,
                        session=sess)
    else:
        lq.kubo_bastin_dev(h["H"], h["V"], h["V"], st, R, M, 256, h["bw"], h["bc"], mu, out, opts=opts, session=sess)


def _size(kind, M):
    return {"m1": 2 * M, "m2": 2 * M * M, "kf": 2 * 256, "kb": 2 * 256}[kind]


@pytest.mark.parametrize("kind,prec", [("m1", lq.PREC_FP64), ("m2", lq.PREC_FP64), ("kf", lq.PREC_FP64),
                                       ("kb", lq.PREC_FP64), ("kb", lq.PREC_MIXED), ("m1", lq.PREC_FP32)])
def test_graph_replay_is_bitwise_eager(honey, kind, prec):
    R, M = 4, 96
    sts = [lattices.random_phase_states(honey["N"], R, seed=s) for s in (3, 4, 5)]
    eager = lq.make_opts(precision=prec)
    graphs = lq.make_opts(precision=prec, use_graphs=1)

    sess = lq.Session(0)
    assert sess.stream() != 0  # a session's own stream: graphs are not captured on the legacy stream
    want = []
    for st in sts:
        out = torch.zeros(_size(kind, M), dtype=torch.float64, device="cuda")
        mu = torch.zeros(2 * M * M, dtype=torch.float64, device="cuda")
        _solve(kind, honey, _dev(st), R, M, out, eager, sess, mu)
        sess.synchronize()
        want.append((out.cpu().numpy(), mu.cpu().numpy()))
    assert sess.graph_stats() == (0, 0)

    st_dev = torch.zeros(2 * honey["N"] * R, dtype=torch.float64, device="cuda")
    out = torch.zeros(_size(kind, M), dtype=torch.float64, device="cuda")
    mu = torch.zeros(2 * M * M, dtype=torch.float64, device="cuda")
    for call in range(5):
        i = call % 3
        st_dev.copy_(_dev(sts[i]))
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        _solve(kind, honey, st_dev, R, M, out, graphs, sess, mu)
        sess.synchronize()
        assert np.array_equal(out.cpu().numpy(), want[i][0]), "call %d" % call
        if kind == "kb":
            assert np.array_equal(mu.cpu().numpy(), want[i][1]), "call %d" % call
    g, replays = sess.graph_stats()
    assert g == 1 and replays == 4  # call 0 eager, call 1 captured + launched, calls 2-4 replayed


def test_new_key_is_captured_anew(honey):
    R, M = 4, 64
    st = lattices.random_phase_states(honey["N"], R, seed=9)
    st_dev = _dev(st)
    sess = lq.Session(0)
    o = lq.make_opts(use_graphs=1)
    outs = [torch.zeros(2 * M, dtype=torch.float64, device="cuda") for _ in range(2)]
    for rep in range(3):
        for out in outs:
            lq.moments1d_dev(honey["H"], None, st_dev, R, M, out, opts=o, session=sess)
    sess.synchronize()
    assert np.array_equal(outs[0].cpu().numpy(), outs[1].cpu().numpy())
    assert sess.graph_stats() == (2, 4)

    # a rescaled operator (new version) gives a new key; the result follows the new scale
    N, Hc, _ = lattices.honeycomb(16, 12, t=-2.7, W=1.0, seed=21)
    H2 = lq.Operator.from_csr(N, *Hc)
    H2.rescale_to_chebyshev(honey["bw"] * 1.1, honey["bc"])
    ref = lq.moments1d(H2, None, st, M)
    for rep in range(3):
        lq.moments1d_dev(H2, None, st_dev, R, M, outs[0], opts=o, session=sess)
        sess.synchronize()
        got = outs[0].cpu().numpy().view(np.complex128)
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    assert sess.graph_stats()[0] == 3


def test_timing_sessions_run_eagerly(honey):
    R, M = 2, 32
    st_dev = _dev(lattices.random_phase_states(honey["N"], R, seed=2))
    out = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
    sess = lq.Session(0)
    sess.enable_timing(True)
    for _ in range(3):
        lq.moments1d_dev(honey["H"], None, st_dev, R, M, out, opts=lq.make_opts(use_graphs=1), session=sess)
    sess.synchronize()
    assert sess.graph_stats() == (0, 0)
    ms, launches = sess.phase_times()
    assert launches[0] >= 3
