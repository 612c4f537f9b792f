"""Serving: continuous batching of DOS and Kubo-Bastin moment solves.

`Server` wraps linqt_server_* (csrc/server.cu): requests are queued with their states
copied at submit, admitted in arrival order as execution slots and HBM budget free up,
and run on per-slot CUDA streams, so requests arriving while others run overlap on the
device.  Each slot's workspace budget is fixed, so a request's chunking (and with the
fixed-order reductions its result) does not depend on what else is running.

`request_stream` draws the seeded request mix of the serving benchmark; `run_stream`
replays it with Poisson arrival times and reports p50/p99 latency and throughput.
"""
import ctypes
import time

import numpy as np

from . import lattices
from ._lib import Request, check, load
from .core import (PREC_FP64, PREC_MIXED, Operator, Session, kubo_bastin_dev, make_opts, moments1d_dev,
                   random_phase_states_dev)

REQ_DOS, REQ_KUBO_BASTIN = 0, 1


class Server:
    def __init__(self, device=0, hbm_budget_bytes=0, max_active=4):
        h = ctypes.c_void_p()
        check(load().linqt_server_create(device, hbm_budget_bytes, max_active, ctypes.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, kind, H, op, states, M, precision=PREC_FP64, R=None, seed=None, nump=0, band_width=None,
               band_center=0.0):
        """Queue one request.  `states` (R x N, host) are copied at submit; with states=None
        the server makes R random-phase states on the device from `seed`.  A Kubo-Bastin
        request with nump > 0 (and H's band_width / band_center) also returns sigma_xx(E)
        (result_sigma) from the same recursion."""
        req = Request()
        if states is not None:
            st = np.ascontiguousarray(np.atleast_2d(states), dtype=np.complex128)
            R = st.shape[0]
            req.states = st.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        else:
            if R is None or seed is None:
                raise ValueError("states=None needs R and seed")
            req.states = None
            req.seed = seed
        out = np.zeros(M if kind == REQ_DOS else M * M, np.complex128)
        req.kind, req.H, req.op = kind, H.h, (op.h if op is not None else None)
        req.R, req.M, req.precision = R, M, precision
        req.mu_out = out.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        sig = None
        if kind == REQ_KUBO_BASTIN and nump > 0:
            if band_width is None:
                raise ValueError("sigma needs the band_width H was rescaled with")
            sig = np.zeros(3 * nump)
            req.sigma_out = sig.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            req.nump, req.band_width, req.band_center = nump, band_width, band_center
        t = ctypes.c_long()
        check(load().linqt_server_submit(self.h, ctypes.byref(req), ctypes.byref(t)))
        self._keep[t.value] = (out, H, op, M, kind, sig)
        return t.value

    def poll(self, ticket):
        st, lat = ctypes.c_int(), ctypes.c_double()
        check(load().linqt_server_poll(self.h, ticket, ctypes.byref(st), ctypes.byref(lat)))
        return st.value, lat.value

    def error(self, ticket):
        """The message of a failed request (empty for one that did not fail)."""
        st, lat = ctypes.c_int(), ctypes.c_double()
        check(load().linqt_server_poll(self.h, ticket, ctypes.byref(st), ctypes.byref(lat)))
        msg = load().linqt_last_error() if st.value < 0 else b""
        return msg.decode() if msg else ""

    def result(self, ticket):
        out, _, _, M, kind, _ = self._keep[ticket]
        return out if kind == REQ_DOS else out.reshape(M, M)

    def result_sigma(self, ticket):
        """(E, sigma, integrand) of a Kubo-Bastin request submitted with nump > 0."""
        sig = self._keep[ticket][5]
        n = len(sig) // 3
        return sig[:n], sig[n:2 * n], sig[2 * n:]

    def retries(self):
        """(requests re-run on the device-wide lane after a co-residency timeout, requests
        re-run alone after their workspaces did not fit next to the others)."""
        a, b = ctypes.c_long(), ctypes.c_long()
        check(load().linqt_server_stats(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def cancel(self, ticket):
        """Withdraw a queued request (LinqtError if it already runs or has finished)."""
        check(load().linqt_server_cancel(self.h, ticket))

    def release(self, ticket):
        """Forget a finished request: the server's record and the Python-side buffers."""
        check(load().linqt_server_release(self.h, ticket))
        self._keep.pop(ticket, None)

    def wait_all(self):
        check(load().linqt_server_wait_all(self.h))

    def close(self):
        if getattr(self, "h", None):
            check(load().linqt_server_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _family(name, N_target, seed):
    """A lattice of the family with about N_target sites: (N, H, V or None, bounds)."""
    if name == "square":
        L = max(4, int(round(N_target ** 0.5)))
        N, H = lattices.square_lattice(L, 1.0, 1.0, seed)
        V = None
    elif name == "honeycomb":
        L = max(4, int(round((N_target / 2) ** 0.5)))
        N, H, V = lattices.honeycomb(L, L, -2.7, 1.0, seed)
    else:
        L = max(4, int(round((N_target / 4) ** 0.5)))
        N, H, V = lattices.kane_mele(L, L, seed=seed)
    lo, hi = lattices.gershgorin_bounds(N, *H)
    return N, H, V, (1.05 * lo, 1.05 * hi)


def request_stream(n_requests=200, seed=52, arrival_seed=51, n_min=1e4, n_max=2e5, m_min=128, m_max=512, r_max=16,
                   rate_hz=None):
    """Seeded request mix: 70 % DOS / 30 % Kubo-Bastin, square / honeycomb / Kane-Mele lattices,
    N log-uniform in [n_min, n_max], M uniform in [m_min, m_max] (rounded to 16), R in [1, r_max],
    precision FP64 or mixed; Poisson arrival gaps (exponential) from arrival_seed."""
    u = lattices.uniform(seed, 6 * n_requests).reshape(n_requests, 6)
    reqs = []
    for i in range(n_requests):
        kind = REQ_DOS if u[i, 0] < 0.7 else REQ_KUBO_BASTIN
        fam = ["square", "honeycomb", "kane_mele"][min(2, int(u[i, 1] * 3))]
        if kind == REQ_KUBO_BASTIN and fam == "square":
            fam = "honeycomb"  # Kubo needs a velocity operator
        N = float(np.exp(np.log(n_min) + u[i, 2] * (np.log(n_max) - np.log(n_min))))
        N = float(10 ** (np.round(np.log10(N) * 8) / 8))  # 8 sizes per decade: lattices are shared
        M = int(round((m_min + u[i, 3] * (m_max - m_min)) / 16) * 16)
        if kind == REQ_KUBO_BASTIN:
            M = max(m_min, M // 2)
        R = 1 + int(u[i, 4] * r_max)
        prec = PREC_FP64 if u[i, 5] < 0.5 else PREC_MIXED
        reqs.append(dict(kind=kind, family=fam, N=N, M=M, R=R, precision=prec))
    a = lattices.uniform(arrival_seed, n_requests)
    gaps = -np.log(1.0 - a)  # unit-rate exponential gaps, scaled by the caller
    return reqs, gaps


def sigma_points(M):
    """Energies of a Kubo-Bastin request's sigma(E): the smallest 256 * 2^j >= 2 M."""
    n = 256
    while n < 2 * M:
        n *= 2
    return n


def _prepare(reqs, session=None):
    """Device-resident operators per request (lattices shared by family and size), the seed of
    each request's random-phase states and H's rescaling (band width, centre)."""
    cache = {}
    prepared = []
    for i, r in enumerate(reqs):
        key = (r["family"], int(r["N"]))
        if key not in cache:
            N, H, V, (lo, hi) = _family(r["family"], r["N"], seed=31 + len(cache))
            Hg = Operator.from_csr(N, *H, session=session)
            Hg.rescale_to_chebyshev(hi - lo, (hi + lo) / 2)
            Vg = Operator.from_csr(N, *V, session=session) if V is not None else None
            cache[key] = (N, Hg, Vg, hi - lo, (hi + lo) / 2)
        N, Hg, Vg, bw, bc = cache[key]
        prepared.append((Hg, Vg, 1000 + i, bw, bc))
    return prepared


def run_serial(reqs, prepared, fp64_only=True, session=None):
    """The same stream one request at a time on the plain FP64 path: states made on the device
    from the request's seed, the solver's device entry point, the moments read back to the host.
    Pass a `session` bound to torch's current stream to keep its workspaces across calls."""
    import torch
    sess = session or Session(stream=torch.cuda.current_stream().cuda_stream)  # ordered with torch's copies
    t0 = time.perf_counter()
    lat = []
    for r, (Hg, Vg, seed, bw, bc) in zip(reqs, prepared):
        t = time.perf_counter()
        o = make_opts(precision=PREC_FP64 if fp64_only else r["precision"])
        N, R, M = Hg.n, r["R"], r["M"]
        st = torch.empty(2 * R * N, dtype=torch.float64, device="cuda")
        random_phase_states_dev(N, R, seed, st, session=sess)
        if r["kind"] == REQ_DOS:
            mu = torch.empty(2 * M, dtype=torch.float64, device="cuda")
            moments1d_dev(Hg, None, st, R, M, mu, opts=o, session=sess)
            mu.cpu()
        else:  # the moment table and sigma(E) from one recursion, as the server runs it
            nump = sigma_points(M)
            mu = torch.empty(2 * M * M, dtype=torch.float64, device="cuda")
            out = torch.empty(3 * nump, dtype=torch.float64, device="cuda")
            kubo_bastin_dev(Hg, Vg, Vg, st, R, M, nump, bw, bc, mu, out, opts=o, session=sess)
            mu.cpu()
            out.cpu()
        lat.append(1e3 * (time.perf_counter() - t))
    t_total = time.perf_counter() - t0
    if session is None:
        sess.close()
    return t_total, np.array(lat)


def run_stream(reqs, prepared, gaps, mean_gap_s, max_active=4, hbm_budget_bytes=0, device=0, server=None):
    """Replay the stream with arrival times cumsum(gaps) * mean_gap_s; returns (latencies ms, makespan s).
    A given `server` is reused (and stays open); otherwise one is created for the run."""
    srv = server if server is not None else Server(device, hbm_budget_bytes, max_active)
    arrivals = np.cumsum(gaps) * mean_gap_s
    tickets = []
    t0 = time.perf_counter()
    for i, (r, (Hg, Vg, seed, bw, bc)) in enumerate(zip(reqs, prepared)):
        now = time.perf_counter() - t0
        if arrivals[i] > now:
            time.sleep(arrivals[i] - now)
        if r["kind"] == REQ_KUBO_BASTIN:
            tickets.append(srv.submit(r["kind"], Hg, Vg, None, r["M"], r["precision"], R=r["R"], seed=seed,
                                      nump=sigma_points(r["M"]), band_width=bw, band_center=bc))
        else:
            tickets.append(srv.submit(r["kind"], Hg, None, None, r["M"], r["precision"], R=r["R"], seed=seed))
    srv.wait_all()
    makespan = time.perf_counter() - t0
    lat = []
    for t in tickets:
        status, ms = srv.poll(t)
        if status != 2:
            raise RuntimeError("request %d (%s) ended with status %d: %s"
                               % (t, reqs[tickets.index(t)], status, srv.error(t)))
        lat.append(ms)
        srv.release(t)
    if server is None:
        srv.close()
    return np.array(lat), makespan


def fifo_latencies(arrivals, service):
    """Latencies (same unit as the inputs) of a single FIFO server with the given service times."""
    t, lat = 0.0, []
    for a, s in zip(arrivals, service):
        t = max(t, a) + s
        lat.append(t - a)
    return np.array(lat)


def main(argv=None):
    """Serving benchmark: one JSON line with p50/p99 latency and throughput of the seeded stream
    through the server (also per precision), next to the same stream served one request at a
    time on the FP64 path.  Kubo-Bastin requests return their moment table and sigma(E)."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=400)
    ap.add_argument("--load", type=float, default=1.5,
                    help="offered load: arrival rate / serial FP64 service rate")
    ap.add_argument("--max-active", type=int, default=2)
    ap.add_argument("--n-max", type=float, default=1e6)
    ap.add_argument("--m-max", type=int, default=1024)
    ap.add_argument("--r-max", type=int, default=32)
    ap.add_argument("--minimal", action="store_true",
                    help="only the timed serial FP64 pass and the timed Poisson pass through the server (each "
                         "warmed up on the short warm-up requests), for streams too long for the full set of passes")
    a = ap.parse_args(argv)
    reqs, gaps = request_stream(a.requests, n_max=a.n_max, m_max=a.m_max, r_max=a.r_max)
    prepared = _prepare(reqs)
    # warm-up: every operator once in both precisions (FP32 value copies, library load)
    seen = set()
    warm_r, warm_p = [], []
    for r, p in zip(reqs, prepared):
        key = (id(p[0]), r["kind"])
        if key not in seen:
            seen.add(key)
            for prec in (PREC_FP64, PREC_MIXED):
                warm_r.append(dict(r, M=32, precision=prec))
                warm_p.append(p)
    import torch
    sess = Session(stream=torch.cuda.current_stream().cuda_stream)

    def serial(rs, ps, fp64_only):
        # the serial session returns its workspaces to the device pool after each pass, so
        # that the server (same pool) finds the memory its HBM budget was set from
        out = run_serial(rs, ps, fp64_only=fp64_only, session=sess)
        torch.cuda.synchronize()
        sess.trim()
        return out

    serial(warm_r, warm_p, False)
    if not a.minimal:
        # an untimed pass of the whole stream first (workspaces, the device pool); the serial
        # passes run before the server exists, since its pool keeps up to its budget cached
        serial(reqs, prepared, True)
    t_ser, svc = serial(reqs, prepared, True)
    t_mix = serial(reqs, prepared, False)[0] if not a.minimal else None
    sess.close()
    torch.cuda.empty_cache()
    srv = Server(0, 0, a.max_active)
    if a.minimal:
        run_stream(warm_r, warm_p, np.zeros(len(warm_r)), 0.0, server=srv)  # untimed: pinned blocks, pool
    else:
        run_stream(reqs, prepared, np.zeros_like(gaps), 0.0, server=srv)
    mean_gap = t_ser / len(reqs) / a.load
    arrivals = np.cumsum(gaps) * mean_gap
    lat_ser = 1e3 * fifo_latencies(arrivals, svc / 1e3)
    lat, makespan = run_stream(reqs, prepared, gaps, mean_gap, server=srv)
    if not a.minimal:
        lat_sat, makespan_sat = run_stream(reqs, prepared, np.zeros_like(gaps), 0.0, server=srv)
    retried = srv.retries()
    srv.close()
    q = lambda x, p: float(np.percentile(x, p)) if len(x) else None
    mixed = np.array([r["precision"] == PREC_MIXED for r in reqs])
    kubo = np.array([r["kind"] == REQ_KUBO_BASTIN for r in reqs])

    def split(x):
        return {"p50_ms": q(x, 50), "p99_ms": q(x, 99),
                "mixed": {"requests": int(mixed.sum()), "p50_ms": q(x[mixed], 50), "p99_ms": q(x[mixed], 99)},
                "fp64": {"requests": int((~mixed).sum()), "p50_ms": q(x[~mixed], 50), "p99_ms": q(x[~mixed], 99)},
                "kubo_bastin": {"p50_ms": q(x[kubo], 50), "p99_ms": q(x[kubo], 99)},
                "dos": {"p50_ms": q(x[~kubo], 50), "p99_ms": q(x[~kubo], 99)}}

    out = {
        "metric": "serving_stream", "requests": len(reqs), "offered_load": a.load,
        "mean_interarrival_ms": 1e3 * mean_gap, "max_active": a.max_active,
        "stream": {"n_range": [1e4, a.n_max], "m_range": [128, a.m_max], "r_max": a.r_max,
                   "dos_fraction": float((~kubo).mean()), "mixed_fraction": float(mixed.mean()),
                   "kubo_returns": "moment table and sigma(E) at the smallest 256*2^j >= 2M energies"},
        "server": dict(split(lat), requests_per_s=len(reqs) / makespan),
        "serial_fp64": dict(split(lat_ser), requests_per_s=len(reqs) / t_ser),
        "requests_rerun": {"on_the_cooperative_lane": retried[0], "alone_after_nomem": retried[1]},
    }
    if not a.minimal:
        out["serial_request_precision_requests_per_s"] = len(reqs) / t_mix
        out["server_saturated"] = dict(split(lat_sat), requests_per_s=len(reqs) / makespan_sat)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
