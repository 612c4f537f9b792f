"""Host side of bench.py on several ranks (gloo, world size 2, CPU): each rank solves its own
replica with its own phase seed, the reported time is the slowest rank's, and the rate is
the whole job's."""
import os
import socket
import sys

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        N, H, V, bw, bc, st = bench.build_inputs(rank)
        # replicas: same operator, different random vectors
        sig = torch.tensor([float(np.abs(st).sum()), float(np.real(st[0, :8]).sum()), float(bw)], dtype=torch.float64)
        sigs = [torch.zeros(3, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(sigs, sig)
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        slow = bench.max_over_ranks(local_ms, dist, "cpu")
        value, e2e = bench.whole_job_rates(1000.0, world, slow, 2 * slow)
        out[rank] = (sigs[0].tolist(), sigs[1].tolist(), slow, value, e2e)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_and_max_over_ranks():
    world, port = 2, _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    (s0, s1, slow0, v0, e0), (_, _, slow1, _, _) = res[0], res[1]
    assert abs(s0[0] - s1[0]) < 1e-9 * abs(s0[0])  # |r_i| = 1/sqrt(N) everywhere: same norm sum
    assert s0[1] != s1[1]  # different phases
    assert s0[2] == s1[2]  # same operator bounds
    assert slow0 == slow1 == 15.0
    assert v0 == 2 * 1000.0 / 15e-3 and e0 == 2 * 1000.0 / 30e-3
