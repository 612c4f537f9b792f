"""One solve's random-phase states sharded over two ranks (gloo, CPU): each rank solves its
shard with the oracle, the shards are reduced by linqt_b200.shards, and every rank must
hold the result of the whole solve over all the states.  The oracle stands in for the
per-rank GPU solve here; tests/test_gpu_shards.py checks the same weighting on the GPU."""
import os
import socket
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

TOL = 1e-13


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _worker(rank, world, port, R, out):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle as orc
        from linqt_b200 import lattices, shards
        N, Hc, Vc = lattices.honeycomb(6, 5, t=-2.7, W=1.0, seed=21)
        lo, hi = lattices.gershgorin_bounds(N, *Hc)
        bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
        H = orc.Op(*Hc).rescale(2 / bw, -bc / (bw / 2))
        V = orc.Op(*Vc)
        st = lattices.random_phase_states(N, R, seed=22)
        a, b = shards.shard_range(R, world, rank)
        mine = st[a:b]
        M, nump = 24, 64
        if len(mine):
            mu1 = orc.moments1d(H, None, mine, M)
            mu2 = orc.moments2d(H, V, V, mine, M)
            E, s, integ, _ = orc.kubo_fft(H, V, V, mine, M, nump, 1, N, bw, bc)
        else:
            mu1, mu2 = np.zeros(M, np.complex128), np.zeros((M, M), np.complex128)
            E, s, integ = np.zeros(nump), np.zeros(nump), np.zeros(nump)
        g1, g2 = shards.reduce_shard([mu1, mu2], b - a, R)
        gE, gs, gi = shards.reduce_fft_shard(E, s, integ, b - a, R)
        f1 = orc.moments1d(H, None, st, M)
        f2 = orc.moments2d(H, V, V, st, M)
        fE, fs, fi, _ = orc.kubo_fft(H, V, V, st, M, nump, 1, N, bw, bc)
        out[rank] = (b - a, _rel(g1, f1), _rel(g2, f2), _rel(gs, fs), _rel(gi, fi), float(np.abs(gE - fE).max()))
    finally:
        dist.destroy_process_group()


def _run(R, world=2):
    # the result store's server process is spawned too: forking a multi-threaded process can deadlock
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, _free_port(), R, out), nprocs=world, join=True)
        return [out[r] for r in range(world)]


def test_two_ranks_uneven_shards():
    res = _run(R=3)
    assert [r[0] for r in res] == [2, 1]
    for _, e1, e2, es, ei, eE in res:
        assert e1 < TOL and e2 < TOL and es < TOL and ei < TOL, (e1, e2, es, ei)
        assert eE == 0.0


def test_two_ranks_one_state():
    # R < world: the second rank has no states and contributes zeros
    res = _run(R=1)
    assert [r[0] for r in res] == [1, 0]
    for _, e1, e2, es, ei, eE in res:
        assert e1 < TOL and e2 < TOL and es < TOL and ei < TOL, (e1, e2, es, ei)
        assert eE == 0.0


def test_shard_ranges_cover_states():
    sys.path.insert(0, ROOT)
    from linqt_b200 import shards
    for R in (0, 1, 2, 7, 64):
        for world in (1, 2, 3, 8):
            rs = [shards.shard_range(R, world, k) for k in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == R
            assert all(rs[k][1] == rs[k + 1][0] for k in range(world - 1))
            sizes = [b - a for a, b in rs]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    assert shards.combine([np.ones(3), 3 * np.ones(3), np.zeros(3)], [1, 3, 0]).tolist() == [2.5] * 3
