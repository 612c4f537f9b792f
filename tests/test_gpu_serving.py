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
