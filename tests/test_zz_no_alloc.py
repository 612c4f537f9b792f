"""The entry point that allocates nothing (linqt_moments1d_noalloc).

It serves callers that must not call cudaMalloc or cudaFree while they run: a
latency-bound serving loop, a thread sharing the GPU with another allocator, or code
that may not use the CUDA allocation API.  Its scratch is a fixed static device array
shared by every call.  These tests call it through the C ABI, twice in a row, and
compare each result with the regular entry point (linqt_moments1d_dev) at the FP64
tolerance the other parity tests use.  The file is named so that pytest collects it
last.
"""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


# (24, 300, 64): R > 256 and not a multiple of 256, so the states run as two chunks of
# 256 columns, the second zero-padded, and the chunks' dot products are summed.
@pytest.mark.parametrize("L,R,M", [(24, 3, 200), (64, 16, 101), (24, 300, 64)])
def test_noalloc_matches_regular_entry_point_twice(L, R, M):
    torch = pytest.importorskip("torch")
    N, Hc = lattices.square_lattice(L, t=1.0, W=1.0, seed=11)
    H = lq.Operator.from_csr(N, *Hc)
    H.rescale_to_chebyshev(2 * 1.05 * 4.5, 0.0)
    st = lattices.random_phase_states(N, R, seed=12)
    st_dev = torch.from_numpy(st.view(np.float64).copy()).cuda()

    ref_dev = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
    sess = lq.Session(0)
    lq.moments1d_dev(H, None, st_dev, R, M, ref_dev, session=sess)
    sess.synchronize()
    ref = ref_dev.cpu().numpy().view(np.complex128)

    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # the shared array keeps the previous call's contents
        out = torch.full((2 * M,), float("nan"), dtype=torch.float64, device="cuda")
        lq.moments1d_noalloc(H, st_dev, R, M, out, stream=stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.complex128)
        assert np.isfinite(got).all()
        assert _rel(got, ref) <= TOL


def test_noalloc_rejects_solves_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    N, Hc = lattices.square_lattice(300, t=1.0, W=1.0, seed=11)  # 90,000 sites
    H = lq.Operator.from_csr(N, *Hc)
    H.rescale_to_chebyshev(2 * 1.05 * 4.5, 0.0)
    R, M = 32, 16  # 2 blocks x 90,000 x 32 x 16 B = 92 MB > 32 MiB
    st_dev = torch.zeros(2 * R * N, dtype=torch.float64, device="cuda")
    out = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
    with pytest.raises(lq.LinqtError) as e:
        lq.moments1d_noalloc(H, st_dev, R, M, out, stream=torch.cuda.current_stream().cuda_stream)
    assert e.value.code == -1
    assert "LINQT_NOALLOC_SCRATCH_BYTES" in str(e.value)
