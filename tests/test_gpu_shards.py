"""Sharded random-phase states on the GPU: per-shard solves through the C ABI, combined with
the weights the cross-rank all-reduce applies (linqt_b200.shards.combine), equal the one
solve over all the states.  One GPU, no collective: the reduction itself is covered on CPU
by tests/test_shards.py.  Tolerance 1e-12 relative (FP64; only the order of the final
sums differs)."""
import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import lattices, shards

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def honey():
    N, Hc, Vc = lattices.honeycomb(16, 12, t=-2.7, W=1.0, seed=21)
    lo, hi = lattices.gershgorin_bounds(N, *Hc)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    H = lq.Operator.from_csr(N, *Hc)
    H.rescale_to_chebyshev(bw, bc)
    V = lq.Operator.from_csr(N, *Vc)
    return dict(N=N, H=H, V=V, bw=bw, bc=bc, st=lattices.random_phase_states(N, 7, seed=22))


@pytest.mark.parametrize("world", [2, 3, 8])
def test_sharded_moments_equal_whole_solve(honey, world):
    H, V, st = honey["H"], honey["V"], honey["st"]
    R, M = st.shape[0], 48
    full1 = lq.moments1d(H, None, st, M)
    full2 = lq.moments2d(H, V, V, st, M)
    counts, p1, p2 = [], [], []
    for k in range(world):
        a, b = shards.shard_range(R, world, k)
        counts.append(b - a)
        p1.append(lq.moments1d(H, None, st[a:b], M) if b > a else np.zeros(M, np.complex128))
        p2.append(lq.moments2d(H, V, V, st[a:b], M) if b > a else np.zeros((M, M), np.complex128))
    assert rel(shards.combine(p1, counts), full1) < TOL
    assert rel(shards.combine(p2, counts), full2) < TOL


def test_sharded_kubo_fft_equal_whole_solve(honey):
    H, V, st = honey["H"], honey["V"], honey["st"]
    R, M, nump = st.shape[0], 48, 128
    E, s, integ = lq.kubo_fft(H, V, V, st, M, nump, lq.KUBO_BASTIN, honey["bw"], honey["bc"])
    counts, ps, pi = [], [], []
    for k in range(2):
        a, b = shards.shard_range(R, 2, k)
        Ek, sk, ik = lq.kubo_fft(H, V, V, st[a:b], M, nump, lq.KUBO_BASTIN, honey["bw"], honey["bc"])
        assert np.array_equal(Ek, E)
        counts.append(b - a)
        ps.append(sk)
        pi.append(ik)
    assert rel(shards.combine(ps, counts), s) < TOL
    assert rel(shards.combine(pi, counts), integ) < TOL


NCCL_SCRIPT = r'''
import datetime, json, sys
import numpy as np
import torch
import torch.distributed as dist
sys.path.insert(0, sys.argv[1])
import linqt_b200 as lq
from linqt_b200 import lattices, shards
dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
torch.cuda.set_device(0)
N, Hc, Vc = lattices.honeycomb(16, 12, t=-2.7, W=1.0, seed=21)
lo, hi = lattices.gershgorin_bounds(N, *Hc)
H = lq.Operator.from_csr(N, *Hc)
H.rescale_to_chebyshev(1.05 * (hi - lo), (hi + lo) / 2)
V = lq.Operator.from_csr(N, *Vc)
st = lattices.random_phase_states(N, 7, seed=22)
st_dev = torch.from_numpy(st.view(np.float64).copy()).cuda()
M = 48
whole = torch.zeros((M, M), dtype=torch.complex128, device="cuda")
lq.moments2d_dev(H, V, V, st_dev, 7, M, torch.view_as_real(whole))
torch.cuda.synchronize()
mu = torch.zeros((M, M), dtype=torch.complex128, device="cuda")
shards.sharded_moments2d_dev(H, V, V, st_dev, 7, 7, M, mu)
torch.cuda.synchronize()
a, b = mu.cpu().numpy(), whole.cpu().numpy()
print(json.dumps({"rel": float(np.abs(a - b).max() / np.abs(b).max())}))
dist.destroy_process_group()
'''


def test_sharded_moments2d_dev_through_nccl_world_of_one(tmp_path):
    """The device form of the sharded solve through a real NCCL all-reduce (a world of one
    rank on this GPU): the collective runs and leaves the table of the whole solve."""
    import json
    import os
    import socket
    import subprocess
    import sys
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-c", NCCL_SCRIPT, root], env=env, capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    res = json.loads(p.stdout.strip().splitlines()[-1])
    assert res["rel"] <= 1e-14
