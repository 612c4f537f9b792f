"""Timing of the other workload families (one JSON line each), next to bench.py's
Kubo-Bastin graphene workload:

    python -m linqt_b200.workloads dos      # square L=256, 1 vector, M=1024, DOS (full size)
    python -m linqt_b200.workloads cubic    # cubic Anderson L=100 (N=1e6), 64 vectors, M=1024 (1 of 4 seeds)
    python -m linqt_b200.workloads spin     # Kane-Mele with spin, 64x64 cells, R=8, M=512, nump=1024
    python -m linqt_b200.workloads spin --moments 1024 --vectors 32 --reps 1   # the full moment and vector counts
    python -m linqt_b200.workloads layouts  # DOS recursion per sparse layout (CSR, SELL-C-sigma, autotuned)
    python -m linqt_b200.workloads realisations  # 4 disorder seeds in one recursion vs 4 separate solves
    python -m linqt_b200.workloads cubic_full    # cubic L=200 (N=8e6), 4 seeds x 64 vectors, M=4096 (full size)
    python -m linqt_b200.workloads lr_layouts    # L/R recursion of the 2D moments: CSR vs autotuned
    python -m linqt_b200.workloads cubic_width   # cubic L=200 DOS recursion GB/s: CSR vs autotuned, R = 64, 8
    python -m linqt_b200.workloads moments2d --cells 32 --moments 1024 --vectors 32   # one profiled 2D solve
    python -m linqt_b200.workloads recur1d --side 100 --vectors 64 --moments 16 --precision 0  # one 1D recursion
    python -m linqt_b200.workloads time_corr     # <V(t)V> of graphene 128x128, R=16, M=512, 40 time steps
    python -m linqt_b200.workloads supercell     # supercell CSR assembly (wannier2sparse) of two Wannier models
    python -m linqt_b200.workloads locality --side 200 --moments 128 --reps 3  # natural vs locality row order
    python -m linqt_b200.workloads lr_widths --cells 512 --vectors 16 --moments 64 --reps 2  # L/R recursion per width

Each line gives the device time per solve (CUDA events on the session stream, warm-up
first), Chebyshev steps*nnz/s, the recursion's algorithmic bytes per second, and for the
mixed-precision solve its error against FP64.  `spin` is the spin-transport case scaled
from 512x512 cells, M = 1024, R = 32 (2.8e14 flop of contraction, about 14 s per FP64 solve:
`spin --cells 512 --moments 1024 --vectors 32 --reps 1` runs the full size) to a size that runs
in a fraction of a second; `cubic` is one disorder seed of the four.
"""
import argparse
import json

import numpy as np

from . import lattices
from .core import PREC_FP64, PREC_MIXED, PREC_MIXED_FAST, Operator, Session, make_opts, kubo_bastin_dev, moments1d_dev


def _hbm_peak():
    """(GB/s, source): the copy bandwidth measured on this GPU model (MEASURED_PEAKS.json at
    the repository root), else the 6650 GB/s fallback."""
    import os
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p)).get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _timed(fn, reps, torch):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def _ops(N, H, extra=()):
    lo, hi = lattices.gershgorin_bounds(N, *H)
    bw, bc = 1.05 * (hi - lo), (hi + lo) / 2
    sess = Session()
    import torch
    sess.set_stream(torch.cuda.current_stream())
    Hg = Operator.from_csr(N, *H, session=sess)
    Hg.rescale_to_chebyshev(bw, bc)
    return sess, bw, bc, Hg, [Operator.from_csr(N, *X, session=sess) for X in extra]


def run_1d(name, N, H, R, M, reps, phase_seed):
    import torch
    sess, bw, bc, Hg, _ = _ops(N, H)
    st = lattices.random_phase_states(N, R, seed=phase_seed)
    st_dev = torch.from_numpy(st.view(np.float64).copy()).cuda()
    out = {}
    for prec in (PREC_FP64, PREC_MIXED):
        mu = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
        o = make_opts(precision=prec)
        ms = _timed(lambda: moments1d_dev(Hg, None, st_dev, R, M, mu, opts=o, session=sess), reps, torch)
        out[prec] = (ms, mu.cpu().numpy().view(np.complex128))
    nnz = Hg.nnz
    ms64, mu64 = out[PREC_FP64]
    msmx, mumx = out[PREC_MIXED]
    steps = M * R  # algorithmic recursion steps (columns x moments); the doubling identities do half
    Rc = 1 << (R - 1).bit_length()
    bytes_step = nnz * (16 + 4) + 4 * (N + 1) + 3 * 16 * N * Rc
    executed_steps = (M + 1) // 2
    return {
        "workload": name, "N": N, "nnz_full": nnz, "R": R, "M": M,
        "fp64": {"ms_per_solve": ms64, "steps_nnz_per_s": steps * nnz / (ms64 * 1e-3),
                 "recursion_GBps": executed_steps * bytes_step / (ms64 * 1e-3) / 1e9},
        "mixed": {"ms_per_solve": msmx, "steps_nnz_per_s": steps * nnz / (msmx * 1e-3),
                  "err_mu_vs_fp64": float(np.abs(mumx - mu64).max() / np.abs(mu64).max())},
    }


def run_spin(Lc, R, M, nump, reps, mixed_precisions=(PREC_MIXED,)):
    """Kane-Mele spin transport: the Kubo-Bastin solve (2D moments and the per-site FFT
    reconstruction of sigma(E)) and the 2D moments alone, FP64 and each of
    `mixed_precisions` (LINQT_PREC_MIXED: 4-digit INT8 contraction; LINQT_PREC_MIXED_FAST:
    3 digits, smaller digit planes and so wider vector chunks), layouts autotuned.
    sigma is also reconstructed from each precision's moment table by the Bastin energy sum
    (kuboBastinFromChebmom, all M moments kept), to state the error a moments-only mixed
    solve carries into sigma."""
    import torch
    from .core import bastin_from_moments, moments2d_dev
    N, H, J = lattices.kane_mele(Lc, Lc, seed=31)
    st = lattices.random_phase_states(N, R, seed=32)
    st_dev = torch.from_numpy(st.view(np.float64).copy()).cuda()
    res = {}
    for prec in (PREC_FP64,) + tuple(mixed_precisions):
        # a session (and operators) of its own per precision, so that neither is timed next
        # to the other's cached workspaces
        sess, bw, bc, Hg, (Jg,) = _ops(N, H, [J])
        mu = torch.zeros(2 * M * M, dtype=torch.float64, device="cuda")
        out = torch.zeros(3 * nump, dtype=torch.float64, device="cuda")
        o = make_opts(precision=prec, fmt=2)
        solve = lambda: kubo_bastin_dev(Hg, Jg, Jg, st_dev, R, M, nump, bw, bc, mu, out, opts=o, session=sess)
        ms = _timed(solve, reps, torch)
        sess.enable_timing(True)
        sess.phase_times(reset=True)
        for _ in range(reps):
            solve()
        torch.cuda.synchronize()
        ph, _ = sess.phase_times(reset=True)
        sess.enable_timing(False)
        mu_h = mu.cpu().numpy().view(np.complex128).reshape(M, M)
        s_fft = out.cpu().numpy()[nump:2 * nump]
        mu2 = torch.zeros(2 * M * M, dtype=torch.float64, device="cuda")
        ms2 = _timed(lambda: moments2d_dev(Hg, Jg, Jg, st_dev, R, M, mu2, opts=o, session=sess), reps, torch)
        E_m, s_mom = bastin_from_moments(mu_h, N, bw, bc, 1e-3, xbound=0.99, session=sess)
        res[prec] = dict(ms=ms, phases=[round(x / reps, 3) for x in ph], mu=mu_h, s_fft=s_fft, ms2=ms2, s_mom=s_mom,
                         tuned={":".join(k.split(":")[:3]): v for k, v in Hg.tuned().items()})
        nnz = Hg.nnz
        del mu, out, mu2, Hg, Jg
        sess.close()
        torch.cuda.synchronize()
    a = res[PREC_FP64]
    lo, hi = int(0.05 * nump), int(0.95 * nump)
    nd = len(a["s_mom"])
    lo2, hi2 = int(0.05 * nd), int(0.95 * nd)
    work = 2 * M * R * nnz  # algorithmic Chebyshev steps (L and R recursions) x nnz

    def side(r):
        return {"ms_per_solve": r["ms"], "phases_ms": r["phases"], "steps_nnz_per_s": work / (r["ms"] * 1e-3),
                "moments2d_ms": r["ms2"], "moments2d_steps_nnz_per_s": work / (r["ms2"] * 1e-3),
                "autotuned": r["tuned"]}

    out = {"workload": "spin_kane_mele_%dx%d" % (Lc, Lc), "N": N, "nnz_full": nnz, "R": R, "M": M, "nump": nump,
           "operator": "{s_z, V_x}/2", "fp64": side(a)}
    out["fp64"]["contraction_TFLOPs"] = 8.0 * M * M * N * R / (a["phases"][1] * 1e-3) / 1e12
    for prec in mixed_precisions:
        b = res[prec]
        key = {PREC_MIXED: "mixed", PREC_MIXED_FAST: "mixed_fast"}.get(prec, "precision_%d" % prec)
        out[key] = side(b)
        out[key].update({
            "speedup_solve": a["ms"] / b["ms"], "speedup_moments2d": a["ms2"] / b["ms2"],
            "err_mu_vs_fp64": float(np.abs(b["mu"] - a["mu"]).max() / np.abs(a["mu"]).max()),
            "err_sigma_fft_vs_fp64_interior90": float(np.abs(b["s_fft"][lo:hi] - a["s_fft"][lo:hi]).max()
                                                      / np.abs(a["s_fft"][lo:hi]).max()),
            "err_sigma_from_moments_vs_fp64_interior90": float(np.abs(b["s_mom"][lo2:hi2] - a["s_mom"][lo2:hi2]).max()
                                                               / np.abs(a["s_mom"][lo2:hi2]).max())})
    return out


def run_layouts(N, H, R, M, reps, name):
    """DOS recursion time per layout: CSR, SELL-C-sigma (C = 8, 32) and the autotuner's choice."""
    import torch
    sess, bw, bc, Hg, _ = _ops(N, H)
    st = lattices.random_phase_states(N, R, seed=45)
    st_dev = torch.from_numpy(st.view(np.float64).copy()).cuda()
    mu = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
    out = {"workload": name, "N": N, "R": R, "M": M}
    for label, fmt in (("csr", 0), ("sell32", 1), ("auto", 2)):
        o = make_opts(fmt=fmt)
        out[label + "_ms"] = _timed(lambda: moments1d_dev(Hg, None, st_dev, R, M, mu, opts=o, session=sess), reps,
                                    torch)
    return out


def run_realisations(L, S, Rs, M, reps):
    """S disorder seeds x Rs vectors: one stacked recursion against S separate solves."""
    import torch
    from .core import moments1d_realisations_dev
    sess = Session()
    sess.set_stream(torch.cuda.current_stream())
    ops, sts = [], []
    for r in range(S):
        N, H = lattices.cubic_lattice(L, 1.0, 2.0, 41 + r)
        Hg = Operator.from_csr(N, *H, session=sess)
        Hg.rescale_to_chebyshev(2 * 1.05 * 7.0, 0.0)
        ops.append(Hg)
        sts.append(lattices.random_phase_states(N, Rs, seed=45 + r))
    st_all = torch.from_numpy(np.concatenate(sts).view(np.float64).copy()).cuda()
    st_one = [torch.from_numpy(x.view(np.float64).copy()).cuda() for x in sts]
    out = {"workload": "dos_cubic_%d_%dseeds_x_%d" % (L, S, Rs), "N": ops[0].n, "M": M}
    for label, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        o = make_opts(precision=prec)
        mu = torch.zeros(2 * S * M, dtype=torch.float64, device="cuda")
        mu1 = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
        out[label + "_stacked_ms"] = _timed(
            lambda: moments1d_realisations_dev(ops, st_all, S * Rs, M, mu, opts=o, session=sess), reps, torch)
        out[label + "_separate_ms"] = _timed(
            lambda: [moments1d_dev(ops[r], None, st_one[r], Rs, M, mu1, opts=o, session=sess) for r in range(S)],
            reps, torch)
    return out


def run_cubic_full(L, S, Rs, M, mode=0):
    """Large DOS batching at full size: cubic Anderson L^3, S disorder seeds x Rs vectors in one
    persistent recursion (stacked realisations), FP64 and mixed.  The states come from the device
    generator (S*Rs*N complex values would be 33 GB on the host at L = 200).  Each precision is
    warmed up with a short solve (allocations, module loads, the stacked-or-separate choice of
    opts.realisations = mode) and then timed once."""
    import time
    import torch
    from .core import moments1d_realisations_dev, random_phase_states_dev
    sess = Session()
    sess.set_stream(torch.cuda.current_stream())
    ops = []
    t0 = time.time()
    for r in range(S):
        N, H = lattices.cubic_lattice(L, 1.0, 2.0, 41 + r)
        Hg = Operator.from_csr(N, *H, session=sess)
        Hg.rescale_to_chebyshev(2 * 1.05 * 7.0, 0.0)
        ops.append(Hg)
        del H
    setup_s = time.time() - t0
    R = S * Rs
    st = torch.empty(2 * R * N, dtype=torch.float64, device="cuda")
    random_phase_states_dev(N, R, 45, st, session=sess)
    nnz = ops[0].nnz
    steps = (M + 1) // 2  # recursion steps with the doubling identities
    out = {"workload": "dos_cubic_%d_%dseeds_x_%d" % (L, S, Rs), "N": N, "nnz_full": nnz, "R_total": R,
           "M": M, "realisations": ["autotuned", "stacked", "separate"][mode], "host_setup_s": round(setup_s, 1)}
    mus = {}
    # complex128 operators with FP64 and FP32 blocks, and complex64 operators with FP32 blocks
    for label, prec, esz, c64 in (("fp64", PREC_FP64, 16, 0), ("mixed", PREC_MIXED, 8, 0),
                                  ("mixed_c64", PREC_MIXED, 8, 1)):
        o = make_opts(precision=prec, fmt=2, realisations=mode, operator_precision=c64)
        mu = torch.zeros(2 * S * M, dtype=torch.float64, device="cuda")
        moments1d_realisations_dev(ops, st, R, 64, mu, opts=o, session=sess)  # warm-up
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        moments1d_realisations_dev(ops, st, R, M, mu, opts=o, session=sess)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        bytes_step = S * (nnz * ((8 if c64 else 16) + 4) + 4 * (N + 1)) + 3 * esz * N * R
        gbs = steps * bytes_step / (ms * 1e-3) / 1e9
        mus[label] = mu.cpu().numpy().view(np.complex128).reshape(S, M)
        peak, src = _hbm_peak()
        out[label] = {"ms_per_solve": ms, "steps_nnz_per_s": M * R * nnz / (ms * 1e-3),
                      "recursion_GBps": gbs, "hbm_frac": gbs / peak, "hbm_peak_GBps": peak, "hbm_peak_source": src,
                      "autotuned": {":".join(k.split(":")[:3]): v for k, v in ops[0].tuned().items()
                                    if (":f64" if prec == PREC_FP64 else ":f32") in k
                                    and ("c64" in k or k.startswith("1d64")) == bool(c64)}}
    for label in ("mixed", "mixed_c64"):
        e = np.abs(mus[label] - mus["fp64"]).max(axis=1) / np.abs(mus["fp64"]).max(axis=1)
        out[label]["err_mu_vs_fp64_per_seed"] = [float(x) for x in e]
    return out


def run_lr_layouts(name, N, H, V, R, M, reps):
    """Recursion phase of the 2D moments (L and R recursions with V fused) per precision,
    the operator's CSR (shape 0) against the autotuned layout / thread shape."""
    import torch
    from .core import moments2d_dev
    sess, bw, bc, Hg, (Vg,) = _ops(N, H, [V])
    st = torch.from_numpy(lattices.random_phase_states(N, R, seed=32).view(np.float64).copy()).cuda()
    mu = torch.zeros(2 * M * M, dtype=torch.float64, device="cuda")
    out = {"workload": "lr_" + name, "N": N, "R": R, "M": M}
    for lab, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        for fl, fmt in (("csr", 0), ("auto", 2)):
            o = make_opts(precision=prec, fmt=fmt)
            f = lambda: moments2d_dev(Hg, Vg, Vg, st, R, M, mu, opts=o, session=sess)
            f()
            f()
            torch.cuda.synchronize()
            sess.enable_timing(True)
            sess.phase_times(reset=True)
            for _ in range(reps):
                f()
            torch.cuda.synchronize()
            ph, _ = sess.phase_times(reset=True)
            sess.enable_timing(False)
            out[lab + "_" + fl + "_recursion_ms"] = ph[0] / reps
    return out


def run_lr_widths(Lc, R, M, widths, reps):
    """Recursion phase of the Kane-Mele spin 2D moments per precision and vector-block width
    (opts.block_width), layout autotuned: ms per block step and vector, and the autotuner's
    choice (the case the spin-transport workload's chunks run in)."""
    import torch
    from .core import moments2d_dev
    N, H, J = lattices.kane_mele(Lc, Lc, seed=31)
    sess, bw, bc, Hg, (Jg,) = _ops(N, H, [J])
    st = torch.from_numpy(lattices.random_phase_states(N, R, seed=32).view(np.float64).copy()).cuda()
    mu = torch.zeros(2 * M * M, dtype=torch.float64, device="cuda")
    rows = []
    for lab, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        for w in widths:
            o = make_opts(precision=prec, fmt=2, block_width=w)
            f = lambda: moments2d_dev(Hg, Jg, Jg, st, R, M, mu, opts=o, session=sess)
            f()
            f()
            torch.cuda.synchronize()
            sess.enable_timing(True)
            sess.phase_times(reset=True)
            for _ in range(reps):
                f()
            torch.cuda.synchronize()
            ph, _ = sess.phase_times(reset=True)
            sess.enable_timing(False)
            rec = ph[0] / reps
            choice = {k: v for k, v in Hg.tuned().items()
                      if k.startswith("lr:%d:%s:" % (w, "f64" if prec == PREC_FP64 else "f32"))}
            rows.append({"precision": lab, "block_width": w, "recursion_ms": round(rec, 3),
                         "us_per_step_and_vector": round(1e3 * rec / (M * R), 3), "choice": choice})
    return {"workload": "lr_widths_kane_mele_%dx%d" % (Lc, Lc), "N": N, "R": R, "M": M, "rows": rows}


def run_cubic_width(L, R, M, reps):
    """1D recursion on a large cubic lattice: algorithmic GB/s with the operator's CSR and
    with the autotuned layout, thread shape and block width."""
    import torch
    from .core import random_phase_states_dev
    N, H = lattices.cubic_lattice(L, 1.0, 2.0, 41)
    sess = Session()
    sess.set_stream(torch.cuda.current_stream())
    Hg = Operator.from_csr(N, *H, session=sess)
    Hg.rescale_to_chebyshev(2 * 1.05 * 7.0, 0.0)
    del H
    st = torch.empty(2 * R * N, dtype=torch.float64, device="cuda")
    random_phase_states_dev(N, R, 45, st, session=sess)
    mu = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
    out = {"workload": "dos_cubic_%d" % L, "N": N, "R": R, "M": M}
    for lab, prec, esz in (("fp64", PREC_FP64, 16), ("mixed", PREC_MIXED, 8)):
        for fl, fmt in (("csr", 0), ("auto", 2)):
            o = make_opts(precision=prec, fmt=fmt)
            ms = _timed(lambda: moments1d_dev(Hg, None, st, R, M, mu, opts=o, session=sess), reps, torch)
            by = Hg.nnz * 20 + 4 * (N + 1) + 3 * esz * N * R
            out[lab + "_" + fl + "_GBps"] = (M + 1) // 2 * by / (ms * 1e-3) / 1e9
    return out


def run_recur1d_once(L, R, M, prec, fmt=0):
    """One warm-up and one timed 1D DOS recursion on the cubic Anderson lattice L^3 (the
    case the 1D recursion kernel is profiled on: one persistent launch per solve)."""
    import torch
    from .core import random_phase_states_dev
    N, H = lattices.cubic_lattice(L, 1.0, 2.0, 41)
    sess = Session()
    sess.set_stream(torch.cuda.current_stream())
    Hg = Operator.from_csr(N, *H, session=sess)
    Hg.rescale_to_chebyshev(2 * 1.05 * 7.0, 0.0)
    del H
    st = torch.empty(2 * R * N, dtype=torch.float64, device="cuda")
    random_phase_states_dev(N, R, 45, st, session=sess)
    mu = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
    o = make_opts(precision=prec, fmt=fmt, block_width=R)
    ms = _timed(lambda: moments1d_dev(Hg, None, st, R, M, mu, opts=o, session=sess), 1, torch)
    esz = 16 if prec == PREC_FP64 else 8
    by = Hg.nnz * 20 + 4 * (N + 1) + 3 * esz * N * R
    return {"workload": "recur1d_cubic_%d" % L, "N": N, "R": R, "M": M, "precision": prec, "format": fmt,
            "ms_per_solve": ms, "recursion_GBps": (M + 1) // 2 * by / (ms * 1e-3) / 1e9,
            "bytes_per_step": by}


def run_locality(L, widths, M, reps):
    """The 1D DOS recursion on the cubic Anderson lattice L^3 with the rows visited in their
    natural order (CSR), in the locality order (FORMAT_LOCAL) and as autotuned, per block width,
    precision of the blocks and of the operator values (complex128, or complex64 with FP32
    blocks), one block of R vectors, CUDA events; the locality order is built and the autotuner
    runs in the untimed first call."""
    import torch
    from .core import FORMAT_AUTO, FORMAT_CSR, FORMAT_LOCAL, random_phase_states_dev
    N, H = lattices.cubic_lattice(L, 1.0, 2.0, 41)
    sess = Session()
    sess.set_stream(torch.cuda.current_stream())
    Hg = Operator.from_csr(N, *H, session=sess)
    Hg.rescale_to_chebyshev(2 * 1.05 * 7.0, 0.0)
    del H
    peak, src = _hbm_peak()
    rows = []
    for R in widths:
        st = torch.empty(2 * R * N, dtype=torch.float64, device="cuda")
        random_phase_states_dev(N, R, 45, st, session=sess)
        mu = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
        for prec, c64 in ((PREC_FP64, 0), (PREC_MIXED, 0), (PREC_MIXED, 1)):
            esz = 16 if prec == PREC_FP64 else 8
            by = Hg.nnz * (12 if c64 else 20) + 4 * (N + 1) + 3 * esz * N * R
            res = {"R": R, "blocks": "fp64" if prec == PREC_FP64 else "fp32", "operator": "c64" if c64 else "c128"}
            ref = None
            for name, fmt in (("csr", FORMAT_CSR), ("local", FORMAT_LOCAL), ("auto", FORMAT_AUTO)):
                o = make_opts(precision=prec, fmt=fmt, block_width=R, operator_precision=c64)
                moments1d_dev(Hg, None, st, R, M, mu, opts=o, session=sess)
                ms = _timed(lambda: moments1d_dev(Hg, None, st, R, M, mu, opts=o, session=sess), reps, torch)
                gbs = (M + 1) // 2 * by / (ms * 1e-3) / 1e9
                m = mu.cpu().numpy().view(np.complex128)
                if ref is None:
                    ref = m
                res[name] = {"ms": round(ms, 3), "GBps": round(gbs, 1), "hbm_frac": round(gbs / peak, 3),
                             "rel_diff_vs_csr": float(np.abs(m - ref).max() / np.abs(ref).max())}
            res["auto"]["choice"] = {k: v for k, v in Hg.tuned().items() if (":%d:" % R) in k and
                                     (":f64:" if prec == PREC_FP64 else ":f32:") in k and
                                     k.startswith("1d64:" if c64 else "1d:")}
            rows.append(res)
        del st
        torch.cuda.empty_cache()
    return {"workload": "locality_cubic_%d" % L, "N": N, "M": M,
            "bytes_per_step": "nnz*(20 or 12 with complex64 values) + 4(N+1) + 3*esz*N*R",
            "hbm_peak_GBps": peak, "hbm_peak_source": src, "rows": rows}


def run_moments2d_once(Lc, R, M, prec):
    """One warm-up and one timed Kane-Mele spin 2D-moment solve with per-phase times (the
    case the contraction kernels are profiled on)."""
    import torch
    from .core import moments2d_dev
    N, H, J = lattices.kane_mele(Lc, Lc, seed=31)
    sess, bw, bc, Hg, (Jg,) = _ops(N, H, [J])
    st = torch.from_numpy(lattices.random_phase_states(N, R, seed=32).view(np.float64).copy()).cuda()
    mu = torch.zeros(2 * M * M, dtype=torch.float64, device="cuda")
    o = make_opts(precision=prec)
    f = lambda: moments2d_dev(Hg, Jg, Jg, st, R, M, mu, opts=o, session=sess)
    f()
    torch.cuda.synchronize()
    sess.enable_timing(True)
    sess.phase_times(reset=True)
    f()
    torch.cuda.synchronize()
    ph, ln = sess.phase_times(reset=True)
    return {"workload": "moments2d_kane_mele_%dx%d" % (Lc, Lc), "N": N, "R": R, "M": M, "precision": prec,
            "phases_ms": ph, "launches": ln}


def run_time_corr(Lc, R, M, NT, dt, reps):
    """Time-domain correlations <V(t) V> of graphene (TimeDependentCorrelations): per time step a
    1D recursion of M steps and two evolution series of K steps each."""
    import torch
    from .core import moments_td_dev, random_phase_states_dev
    N, H, V = lattices.honeycomb(Lc, Lc, t=-2.7, W=1.0, seed=21)
    sess, bw, bc, Hg, (Vg,) = _ops(N, H, [V])
    st = torch.empty(2 * R * N, dtype=torch.float64, device="cuda")
    random_phase_states_dev(N, R, 22, st, session=sess)
    mu = torch.zeros(2 * M * NT, dtype=torch.float64, device="cuda")
    ms = _timed(lambda: moments_td_dev(Hg, Vg, Vg, st, R, M, NT, dt, bw, bc, mu, session=sess), reps, torch)
    x = dt * (0.5 * bw) / 0.6582119624
    K = 0
    from math import fabs
    from scipy.special import jv
    while True:  # the series length the library uses (terms until |J_k(x)| <= 1e-10)
        K += 1
        if not fabs(jv(K, x)) > 1e-10:
            break
    steps = NT * M + 2 * (NT - 1) * K
    return {"workload": "time_corr_graphene_%dx%d" % (Lc, Lc), "N": N, "nnz_full": Hg.nnz, "R": R, "M": M, "NT": NT,
            "dt_fs": dt, "series_terms": K, "ms_per_solve": ms, "ms_per_time_step": ms / NT,
            "steps_nnz_per_s": steps * R * Hg.nnz / (ms * 1e-3)}


def run_supercell(orbitals, reach, L, op, reps):
    """The operator builder on the device: the upper-triangle CSR of `op` for a synthetic
    Wannier model on an L x L x 1 supercell, written into HBM-resident buffers."""
    import os
    import tempfile
    import torch
    from .core import TBModel
    d = tempfile.mkdtemp(prefix="linqt_w2s_")
    label = os.path.join(d, "m")
    lattices.wannier_model(label, orbitals, reach, seed=7)
    sess = Session(0)
    sess.set_stream(torch.cuda.current_stream())
    m = TBModel.load(label)
    n, nnz = m.csr_size(op, (L, L, 1), session=sess)
    rp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    cl = torch.empty(nnz, dtype=torch.int32, device="cuda")
    vl = torch.empty(2 * nnz, dtype=torch.float64, device="cuda")
    ms = _timed(lambda: m.supercell_csr_dev(op, (L, L, 1), rp, cl, vl, nnz, session=sess), reps, torch)
    out_bytes = 20 * nnz + 4 * (n + 1)
    return {"workload": "supercell_wannier%d_r%d_%dx%d_%s" % (orbitals, reach, L, L, op), "N": n, "nnz_upper": nnz,
            "hoppings_per_cell": m.info()[1], "ms_per_build": ms, "entries_per_s": nnz / (ms * 1e-3),
            "output_GBps": out_bytes / (ms * 1e-3) / 1e9}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["dos", "cubic", "cubic_full", "spin", "layouts", "realisations",
                                         "lr_layouts", "cubic_width", "moments2d", "recur1d", "time_corr", "supercell",
                                         "locality", "lr_widths"])
    ap.add_argument("--precision", type=int, default=PREC_MIXED, help="moments2d: LINQT_PREC_* value")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--cells", type=int, default=64, help="spin: Kane-Mele cells per side")
    ap.add_argument("--moments", type=int, default=512, help="spin: M")
    ap.add_argument("--vectors", type=int, default=8, help="spin: R")
    ap.add_argument("--realisations", type=int, default=0, help="cubic_full: 0 autotuned, 1 stacked, 2 separate")
    ap.add_argument("--side", type=int, default=100, help="recur1d: cubic lattice side L")
    ap.add_argument("--mixed", default="1", help="spin: comma-separated mixed precisions beside FP64 (1 = 4-digit "
                                                 "INT8 contraction, 4 = 3-digit)")
    ap.add_argument("--format", type=int, default=0, help="recur1d: LINQT_FORMAT_* value")
    ap.add_argument("--widths", default="8,64,256", help="locality: comma-separated block widths")
    a = ap.parse_args(argv)
    if a.workload == "dos":
        N, H = lattices.square_lattice(256, 1.0, 1.0, 11)
        r = run_1d("dos_square_256", N, H, 1, 1024, a.reps, 12)
    elif a.workload == "cubic":
        N, H = lattices.cubic_lattice(100, 1.0, 2.0, 41)
        r = run_1d("dos_cubic_100_seed41", N, H, 64, 1024, a.reps, 45)
    elif a.workload == "lr_layouts":
        N, H, J = lattices.kane_mele(64, 64, seed=31)
        print(json.dumps(run_lr_layouts("kane_mele_64", N, H, J, 32, 1024, a.reps)))
        N, H, V = lattices.honeycomb(128, 128, t=-2.7, W=1.0, seed=21)
        r = run_lr_layouts("graphene_128", N, H, V, 8, 512, a.reps)
    elif a.workload == "cubic_width":
        print(json.dumps(run_cubic_width(200, 64, 64, a.reps)))
        r = run_cubic_width(200, 8, 64, a.reps)
    elif a.workload == "supercell":
        print(json.dumps(run_supercell(18, 3, 128, "HAM", a.reps)))
        print(json.dumps(run_supercell(18, 3, 128, "VXSY", a.reps)))
        r = run_supercell(4, 1, 2048, "HAM", a.reps)
    elif a.workload == "time_corr":
        r = run_time_corr(128, 16, 512, 40, 1.0, a.reps)
    elif a.workload == "lr_widths":
        r = run_lr_widths(a.cells, a.vectors, a.moments, (2, 4, 8, 16), a.reps)
    elif a.workload == "locality":
        r = run_locality(a.side, tuple(int(x) for x in a.widths.split(",")), a.moments, a.reps)
    elif a.workload == "recur1d":
        r = run_recur1d_once(a.side, a.vectors, a.moments, a.precision, a.format)
    elif a.workload == "moments2d":
        r = run_moments2d_once(a.cells, a.vectors, a.moments, a.precision)
    elif a.workload == "cubic_full":
        r = run_cubic_full(200, 4, 64, 4096, a.realisations)
    elif a.workload == "realisations":
        rs = [run_realisations(100, 4, 64, 1024, a.reps), run_realisations(40, 4, 8, 1024, a.reps)]
        for r in rs:
            print(json.dumps(r))
        return
    elif a.workload == "layouts":
        N, H = lattices.cubic_lattice(100, 1.0, 2.0, 41)
        rs = [run_layouts(N, H, R, 256, a.reps, "dos_cubic_100") for R in (1, 4, 64)]
        N, H, _ = lattices.kane_mele(256, 256, seed=31)
        rs += [run_layouts(N, H, R, 256, a.reps, "dos_kane_mele_256") for R in (1, 4)]
        for r in rs:
            print(json.dumps(r))
        return
    else:
        r = run_spin(a.cells, a.vectors, a.moments, max(1024, a.moments), a.reps,
                     tuple(int(x) for x in a.mixed.split(",")))
    print(json.dumps(r))


if __name__ == "__main__":
    main()
