"""One solve's random-phase states sharded over ranks; the partial results are combined by
one sum all-reduce.

LinQT averages every result over its random-phase states.  SpectralMoments scales each
state's moments by 2/R (src/chebyshev_solver.cpp:176-199).  CorrelationExpansionMoments
scales each state's table by 4/R (src/chebyshev_solver.cpp:152-162).  Kubo_solver_FFT keeps
a running mean over the states (include/Kubo_solver_FFT.hpp:93-96), and its conductivity and
integrand are linear in that mean (src/Kubo_solver_FFT_postProcess.cpp:120-273).  So a solve
over a subset of R_k of the R states returns the mean over that subset, and the full result
is sum_k (R_k / R) * result_k.

Each rank takes a contiguous shard of the states (`shard_range`), solves it on its own GPU
through the C ABI, scales its result by R_k / R and joins one FP64 sum all-reduce:
M*M*16 bytes for a 2D table, M*16 for 1D moments, 2*nump*8 for sigma and the integrand.
The ranks exchange nothing during the recursion.  On a GPU process group the all-reduce is
NCCL over NVLink; on a CPU group (tests) it is gloo.  Every rank takes the same collective,
including a rank whose shard is empty (R < world size), which contributes zeros.
"""
import numpy as np
import torch
import torch.distributed as dist

from . import core


def shard_range(R, world, rank):
    """Rows [start, stop) of the R states that `rank` of `world` solves: contiguous, sizes
    differing by at most one, the larger shards first."""
    if R < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("shard_range: need R >= 0, world >= 1, 0 <= rank < world")
    base, extra = divmod(R, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_weights(R, world):
    """R_k / R for every rank k (zero for an empty shard)."""
    return [(b - a) / R for a, b in (shard_range(R, world, k) for k in range(world))]


def combine(partials, counts):
    """The full result from per-shard results solved locally: sum_k (R_k / R) * partial_k.
    Shards with R_k = 0 are skipped.  This is the sum the all-reduce computes across ranks."""
    R = sum(counts)
    if R <= 0:
        raise ValueError("combine: no states")
    out = None
    for p, c in zip(partials, counts):
        if c == 0:
            continue
        t = np.asarray(p) * (c / R)
        out = t if out is None else out + t
    return out


def _group_device(group):
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def allreduce_sum(arrays, group=None):
    """Sum numpy arrays (float64 or complex128) over the ranks of `group` with ONE
    all-reduce; returns new arrays of the same shapes and types.  A NCCL group reduces a
    device copy, a gloo group a host one."""
    flats = []
    for a in arrays:
        a = np.ascontiguousarray(a)
        if a.dtype == np.complex128:
            flats.append(a.view(np.float64).ravel())
        elif a.dtype == np.float64:
            flats.append(a.ravel())
        else:
            raise TypeError("allreduce_sum: float64 or complex128 arrays only, got %s" % a.dtype)
    buf = torch.from_numpy(np.concatenate(flats) if flats else np.zeros(0))
    dev = _group_device(group)
    t = buf.to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    host = t.cpu().numpy()
    out, off = [], 0
    for a in arrays:
        a = np.asarray(a)
        n = a.size * (2 if a.dtype == np.complex128 else 1)
        part = host[off:off + n].copy()
        off += n
        out.append(part.view(np.complex128).reshape(a.shape) if a.dtype == np.complex128 else part.reshape(a.shape))
    return out


def reduce_shard(arrays, R_k, R, group=None):
    """This rank's per-shard results (means over its R_k states) -> the results of the whole
    solve over R states on every rank.  A rank with R_k = 0 passes zero arrays."""
    w = R_k / R if R_k else 0.0
    return allreduce_sum([np.asarray(a) * w for a in arrays], group)


def _world(group):
    return dist.get_world_size(group), dist.get_rank(group)


def _my_states(states, group):
    st = np.atleast_2d(np.asarray(states, np.complex128))
    R = st.shape[0]
    if R == 0 or st.shape[1] == 0:
        raise ValueError("sharded solve: no states")
    world, rank = _world(group)
    a, b = shard_range(R, world, rank)
    return st[a:b], R


def sharded_moments1d(H, op, states, M, group=None, opts=None, session=None):
    """chebyshev::SpectralMoments over the R rows of `states` (every rank passes all of
    them), this rank solving its shard; returns mu[M] on every rank."""
    mine, R = _my_states(states, group)
    mu = core.moments1d(H, op, mine, M, opts, session) if len(mine) else np.zeros(M, np.complex128)
    return reduce_shard([mu], len(mine), R, group)[0]


def sharded_moments2d(H, opl, opr, states, M, group=None, opts=None, session=None):
    """chebyshev::CorrelationExpansionMoments over the R rows of `states`, sharded by rank;
    returns mu[M, M] on every rank."""
    mine, R = _my_states(states, group)
    mu = core.moments2d(H, opl, opr, mine, M, opts, session) if len(mine) else np.zeros((M, M), np.complex128)
    return reduce_shard([mu], len(mine), R, group)[0]


def reduce_fft_shard(E, sigma, integrand, R_k, R, group=None):
    """(E, sigma, integrand) of this rank's shard -> those of the whole solve, on every rank.
    E does not depend on the states: the group's first rank (which always holds a shard)
    contributes it to the same all-reduce unscaled and the others zeros, so every rank
    receives it bit for bit."""
    w = R_k / R if R_k else 0.0
    first = _world(group)[1] == 0
    s, integ, E = allreduce_sum([np.asarray(sigma) * w, np.asarray(integrand) * w,
                                 np.asarray(E, np.float64) if first else np.zeros(len(E))], group)
    return E, s, integ


def sharded_kubo_fft(H, opl, opr, states, M, nump, formula, band_width, band_center, group=None, opts=None,
                     session=None):
    """Kubo_solver_FFT over the R rows of `states`, sharded by rank; returns
    (E, sigma, integrand) on every rank."""
    mine, R = _my_states(states, group)
    if len(mine):
        E, s, integ = core.kubo_fft(H, opl, opr, mine, M, nump, formula, band_width, band_center, opts, session)
    else:
        E, s, integ = np.zeros(nump), np.zeros(nump), np.zeros(nump)
    return reduce_fft_shard(E, s, integ, len(mine), R, group)


def sharded_moments2d_dev(H, opl, opr, states_dev, R_k, R, M, mu_dev, group=None, opts=None, session=None):
    """Device form: `states_dev` holds this rank's R_k states (R_k x N complex128 on its GPU,
    may be empty), `mu_dev` an M x M complex128 torch tensor on the same GPU.  On return
    mu_dev holds the table of the whole solve over R states, reduced in place on the device
    (one NCCL all-reduce of M*M*16 bytes).  The solve's stream is synchronised before the
    collective, which runs on torch's current stream."""
    if R_k:
        core.moments2d_dev(H, opl, opr, states_dev, R_k, M, mu_dev, opts, session)
        if session is not None:
            session.synchronize()
        else:
            torch.cuda.synchronize()
        mu_dev.mul_(R_k / R)
    else:
        mu_dev.zero_()
    dist.all_reduce(torch.view_as_real(mu_dev), op=dist.ReduceOp.SUM, group=group)
    return mu_dev
