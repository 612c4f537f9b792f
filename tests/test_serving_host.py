"""Host side of serving: the seeded request stream and the FIFO reference queue."""
import numpy as np

from linqt_b200 import serve


def test_stream_is_seeded_and_mixed():
    a, ga = serve.request_stream(50)
    b, gb = serve.request_stream(50)
    assert a == b and np.array_equal(ga, gb)
    kinds = [r["kind"] for r in a]
    assert 0 < kinds.count(serve.REQ_KUBO_BASTIN) < len(kinds)
    assert all(r["family"] != "square" for r in a if r["kind"] == serve.REQ_KUBO_BASTIN)
    assert all(1e4 * 0.999 <= r["N"] <= 2e5 * 1.001 and 1 <= r["R"] <= 16 for r in a)
    assert np.all(ga > 0)


def test_fifo_latencies():
    lat = serve.fifo_latencies([0, 1, 1.5, 10], [2, 2, 2, 1])
    assert np.allclose(lat, [2, 3, 4.5, 1])
