"""Serving: requests that run concurrently in the server give the same results as the
same requests run alone (tolerance 1e-12 relative: the reductions have a fixed order and
the chunking depends only on the request), and the request stream is seeded."""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices, serve

pytestmark = pytest.mark.gpu


def _ops(family, N_target, seed):
    N, H, V, (lo, hi) = serve._family(family, N_target, seed)
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(hi - lo, (hi + lo) / 2)
    Vg = lq.Operator.from_csr(N, *V) if V is not None else None
    return N, Hg, Vg


def test_alone_equals_mixed():
    rng_specs = [("square", 5000, serve.REQ_DOS, 200, 3, lq.PREC_FP64),
                 ("honeycomb", 3000, serve.REQ_KUBO_BASTIN, 64, 4, lq.PREC_FP64),
                 ("kane_mele", 2000, serve.REQ_DOS, 150, 8, lq.PREC_MIXED),
                 ("honeycomb", 8000, serve.REQ_KUBO_BASTIN, 48, 2, lq.PREC_MIXED),
                 ("square", 20000, serve.REQ_DOS, 300, 1, lq.PREC_FP64),
                 ("kane_mele", 4000, serve.REQ_KUBO_BASTIN, 32, 3, lq.PREC_FP64)]
    work = []
    for i, (fam, n, kind, M, R, prec) in enumerate(rng_specs):
        N, Hg, Vg = _ops(fam, n, seed=40 + i)
        st = lattices.random_phase_states(N, R, seed=500 + i)
        work.append((kind, Hg, Vg, st, M, prec))
    # alone: one request at a time through the server
    alone = []
    for kind, Hg, Vg, st, M, prec in work:
        srv = serve.Server(0, 0, 1)
        t = srv.submit(kind, Hg, Vg if kind == serve.REQ_KUBO_BASTIN else None, st, M, prec)
        srv.wait_all()
        assert srv.poll(t)[0] == 2
        alone.append(srv.result(t).copy())
        srv.close()
    # mixed: all submitted at once into 4 slots, twice over
    srv = serve.Server(0, 0, 4)
    tickets = []
    for _ in range(2):
        for kind, Hg, Vg, st, M, prec in work:
            tickets.append(srv.submit(kind, Hg, Vg if kind == serve.REQ_KUBO_BASTIN else None, st, M, prec))
    srv.wait_all()
    for j, t in enumerate(tickets):
        status, lat = srv.poll(t)
        assert status == 2 and lat > 0
        got, ref = srv.result(t), alone[j % len(work)]
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    srv.close()
    # a budget that most requests nearly fill: they wait for memory, later ones that fit
    # pass them (a bounded number of times), and every result is still the alone one
    srv = serve.Server(0, 40 << 20, 4)
    tickets = []
    for _ in range(2):
        for kind, Hg, Vg, st, M, prec in work:
            tickets.append(srv.submit(kind, Hg, Vg if kind == serve.REQ_KUBO_BASTIN else None, st, M, prec))
    srv.wait_all()
    for j, t in enumerate(tickets):
        assert srv.poll(t)[0] == 2
        got, ref = srv.result(t), alone[j % len(work)]
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    srv.close()
    # and the FP64 requests agree with the regular entry points
    kind, Hg, Vg, st, M, prec = work[1]
    assert np.abs(alone[1] - lq.moments2d(Hg, Vg, Vg, st, M)).max() <= 1e-12 * np.abs(alone[1]).max()
    kind, Hg, Vg, st, M, prec = work[0]
    assert np.abs(alone[0] - lq.moments1d(Hg, None, st, M)).max() <= 1e-12 * np.abs(alone[0]).max()


def test_admission_rejects_requests_over_budget():
    N, Hg, Vg = _ops("honeycomb", 3000, seed=7)
    st = lattices.random_phase_states(N, 4, seed=1)
    srv = serve.Server(0, 64 << 20, 2)  # 64 MiB budget
    with pytest.raises(lq.LinqtError) as e:
        srv.submit(serve.REQ_KUBO_BASTIN, Hg, Vg, st, 2048)  # 2 x 2048 blocks of N x 4 complex doubles
    assert e.value.code == -3
    srv.close()


def test_device_states_match_host_generator():
    torch = pytest.importorskip("torch")
    N, R, seed = 3001, 5, 2024
    d = torch.empty(2 * R * N, dtype=torch.float64, device="cuda")
    lq.random_phase_states_dev(N, R, seed, d)
    got = d.cpu().numpy().view(np.complex128).reshape(R, N)
    ref = lattices.random_phase_states(N, R, seed)
    # same Philox words; sin/cos may differ from the host's libm in the last bit
    assert np.abs(got - ref).max() * np.sqrt(N) <= 4e-16


def test_seeded_requests_match_host_states():
    N, Hg, Vg = _ops("kane_mele", 2500, seed=3)
    srv = serve.Server(0, 0, 3)
    t1 = srv.submit(serve.REQ_DOS, Hg, None, None, 120, R=3, seed=77)
    t2 = srv.submit(serve.REQ_KUBO_BASTIN, Hg, Vg, None, 40, R=2, seed=78)
    srv.wait_all()
    st1 = lattices.random_phase_states(N, 3, 77)
    st2 = lattices.random_phase_states(N, 2, 78)
    ref1 = lq.moments1d(Hg, None, st1, 120)
    ref2 = lq.moments2d(Hg, Vg, Vg, st2, 40)
    assert np.abs(srv.result(t1) - ref1).max() <= 1e-12 * np.abs(ref1).max()
    assert np.abs(srv.result(t2) - ref2).max() <= 1e-12 * np.abs(ref2).max()
    srv.release(t1)
    with pytest.raises(lq.LinqtError):
        srv.poll(t1)
    srv.close()


def test_cancel_a_queued_request():
    """A request still queued behind others is withdrawn: status LINQT_ERR_CANCELLED, its
    result buffer untouched; the others complete; a finished request cannot be cancelled."""
    N, Hg, _ = _ops("square", 40000, seed=7)
    st = lattices.random_phase_states(N, 2, seed=8)
    srv = serve.Server(0, 0, 1)  # one slot: the third request waits for the first two
    t1 = srv.submit(serve.REQ_DOS, Hg, None, st, 1024, lq.PREC_FP64)
    t2 = srv.submit(serve.REQ_DOS, Hg, None, st, 1024, lq.PREC_FP64)
    t3 = srv.submit(serve.REQ_DOS, Hg, None, st, 1024, lq.PREC_FP64)
    srv.cancel(t3)
    assert srv.poll(t3)[0] == -7  # LINQT_ERR_CANCELLED
    srv.wait_all()
    assert srv.poll(t1)[0] == 2 and srv.poll(t2)[0] == 2
    assert not np.any(srv.result(t3))
    assert np.array_equal(srv.result(t1), srv.result(t2))
    with pytest.raises(lq.LinqtError):
        srv.cancel(t1)
    srv.close()


def test_kubo_bastin_request_returns_sigma():
    """A Kubo-Bastin request with nump > 0 returns sigma_xx(E) from the same recursion as its
    moment table: equal to linqt_kubo_bastin alone, and unchanged when served next to others."""
    N, H, V, (lo, hi) = serve._family("honeycomb", 6000, seed=3)
    bw, bc = hi - lo, (hi + lo) / 2
    Hg = lq.Operator.from_csr(N, *H)
    Hg.rescale_to_chebyshev(bw, bc)
    Vg = lq.Operator.from_csr(N, *V)
    st = lattices.random_phase_states(N, 3, seed=4)
    M, nump = 96, 256
    mu_ref, (E_ref, s_ref, i_ref) = lq.kubo_bastin(Hg, Vg, Vg, st, M, nump, bw, bc)
    srv = serve.Server(0, 0, 3)
    others = [srv.submit(serve.REQ_DOS, Hg, None, st, 200, lq.PREC_MIXED) for _ in range(3)]
    t = srv.submit(serve.REQ_KUBO_BASTIN, Hg, Vg, st, M, lq.PREC_FP64, nump=nump, band_width=bw, band_center=bc)
    srv.wait_all()
    assert srv.poll(t)[0] == 2 and all(srv.poll(o)[0] == 2 for o in others)
    E, s, integ = srv.result_sigma(t)
    assert np.array_equal(E, E_ref)
    assert np.abs(s - s_ref).max() <= 1e-12 * np.abs(s_ref).max()
    assert np.abs(integ - i_ref).max() <= 1e-12 * np.abs(i_ref).max()
    assert np.abs(srv.result(t) - mu_ref).max() <= 1e-12 * np.abs(mu_ref).max()
    srv.close()


def test_sessions_with_sm_shares_run_recursions_side_by_side():
    """Two sessions with SM shares of 0.45 run their persistent recursions at the same time
    from two host threads (grids sized to their share, launched on their own streams): the
    results equal the whole-device solve up to the order of the partial sums."""
    import threading
    N, Hc = lattices.square_lattice(96, t=1.0, W=1.0, seed=11)
    H = lq.Operator.from_csr(N, *Hc)
    H.rescale_to_chebyshev(2 * 1.05 * 4.5, 0.0)
    _, Hk, Jk, (lo, hi) = serve._family("kane_mele", 4000, seed=5)
    Kg = lq.Operator.from_csr(len(Hk[0]) - 1, *Hk)
    Kg.rescale_to_chebyshev(hi - lo, (hi + lo) / 2)
    Jg = lq.Operator.from_csr(len(Jk[0]) - 1, *Jk)
    st1 = lattices.random_phase_states(N, 4, seed=1)
    st2 = lattices.random_phase_states(Kg.n, 3, seed=2)
    ref1 = lq.moments1d(H, None, st1, 512)
    ref2 = lq.moments2d(Kg, Jg, Jg, st2, 96)
    out, errs = {}, []

    def work(key, fn):
        try:
            s = lq.Session(0)
            s.set_sm_share(0.45)
            out[key] = [fn(s) for _ in range(4)]
            s.close()
        except Exception as e:  # reported below
            errs.append(e)

    t1 = threading.Thread(target=work, args=("1d", lambda s: lq.moments1d(H, None, st1, 512, session=s)))
    t2 = threading.Thread(target=work, args=("2d", lambda s: lq.moments2d(Kg, Jg, Jg, st2, 96, session=s)))
    t1.start(), t2.start()
    t1.join(), t2.join()
    assert not errs, errs
    for got in out["1d"]:
        assert np.abs(got - ref1).max() <= 1e-12 * np.abs(ref1).max()
    for got in out["2d"]:
        assert np.abs(got - ref2).max() <= 1e-12 * np.abs(ref2).max()
