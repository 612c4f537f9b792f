"""Python host API over the C ABI.

Mirrors the reference operations on the hot path:

    Operator.from_csr / Operator.rescale / Operator.multiply   SparseMatrixType (include/sparse_matrix.hpp)
    moments1d                                                  chebyshev::SpectralMoments
    moments1d_nonorth                                          chebyshev::SpectralMoments_nonOrth
    moments2d                                                  chebyshev::CorrelationExpansionMoments
    kubo_fft                                                   chebyshev::Kubo_solver_FFT::compute
    dos_from_moments                                           spectralFunctionFromChebmom_FFTgrid
    spectral_function_from_moments                             spectralFunctionFromChebmom{,_FFTgrid}
    bastin_from_moments                                        kuboBastinFromChebmom

Host arrays are numpy; *_dev functions take device pointers (ints) or torch CUDA
tensors and enqueue on the session stream.
"""
import ctypes

import numpy as np

from ._lib import Opts, check, load

PREC_FP64, PREC_MIXED, PREC_FP32, PREC_MIXED_TF32, PREC_MIXED_FAST = 0, 1, 2, 3, 4
KUBO_GREENWOOD, KUBO_BASTIN = 0, 1
STORAGE_HERMITIAN_UPPER, STORAGE_GENERAL = 0, 1
OP_C128, OP_C64 = 0, 1  # opts.operator_precision: complex128 or complex64 operator values (1D recursions)
FORMAT_CSR, FORMAT_SELL, FORMAT_AUTO, FORMAT_LOCAL = 0, 1, 2, 3  # opts.format


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _c128(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


def _ptr(x):
    """Device pointer of a torch tensor or an int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


def make_opts(precision=PREC_FP64, fmt=0, block_width=0, doubling=0, step_launches=0, use_graphs=0,
              realisations=0, operator_precision=OP_C128, thread_shape=0):
    """Solver options (linqt_opts).  doubling: 0 auto, 1 force, 2 off.  step_launches: 1 = one launch per
    recursion step instead of the persistent cooperative kernel.  use_graphs: 1 = *_dev solves replayed
    from CUDA graphs after their first call.  realisations: 0 autotuned, 1 stacked in one launch,
    2 one solve per realisation."""
    o = Opts()
    o.precision, o.format, o.block_width, o.doubling, o.step_launches = (precision, fmt, block_width, doubling,
                                                                         step_launches)
    o.use_graphs = use_graphs
    o.realisations = realisations
    o.operator_precision = operator_precision
    o.thread_shape = thread_shape
    return o


class Session:
    """A CUDA stream plus cached device workspaces on one GPU."""

    def __init__(self, device=0, stream=None):
        h = ctypes.c_void_p()
        check(load().linqt_session_create(device, ctypes.byref(h)))
        self.h = h
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if getattr(self, "h", None):
            check(load().linqt_session_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        """Adopt an external CUDA stream (an int handle or a torch.cuda.Stream)."""
        ptr = stream if isinstance(stream, int) else stream.cuda_stream
        check(load().linqt_session_set_stream(self.h, ctypes.c_void_p(ptr)))

    def stream(self):
        p = ctypes.c_void_p()
        check(load().linqt_session_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def synchronize(self):
        check(load().linqt_session_synchronize(self.h))

    def trim(self):
        check(load().linqt_session_trim(self.h))

    def enable_timing(self, on=True):
        check(load().linqt_session_enable_timing(self.h, 1 if on else 0))

    def graph_stats(self):
        """(instantiated graphs, solves launched from graphs) under opts.use_graphs."""
        g, r = ctypes.c_int(), ctypes.c_long()
        check(load().linqt_session_graph_stats(self.h, ctypes.byref(g), ctypes.byref(r)))
        return g.value, r.value

    def set_sm_share(self, share):
        """Persistent kernels of this session use at most `share` of the device's co-resident
        CTAs and run on its stream, next to other sessions' (see linqt_session_set_sm_share)."""
        check(load().linqt_session_set_sm_share(self.h, share))

    def inject_barrier_timeout(self, extra_arrivals=1, spin_limit=1024):
        """Test hook: make this session's grid barriers wait for CTAs never launched (the next
        solve then fails with LINQT_ERR_TIMEOUT); (0, 0) restores them."""
        check(load().linqt_session_inject_barrier_timeout(self.h, extra_arrivals, spin_limit))

    def phase_times(self, reset=False):
        """(ms[4], launches[4]) for recursion, contraction, FFT, other."""
        ms = (ctypes.c_double * 4)()
        ln = (ctypes.c_long * 4)()
        check(load().linqt_session_phase_times(self.h, ms, ln, 1 if reset else 0))
        return list(ms), list(ln)


def _sh(session):
    return None if session is None else session.h


class Operator:
    """A sparse operator resident on the GPU (SparseMatrixType)."""

    def __init__(self, handle, session=None):
        self.h = handle
        self.session = session

    @classmethod
    def from_csr(cls, n, rowptr, col, val, storage=STORAGE_HERMITIAN_UPPER, session=None):
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        v = _c128(val).view(np.float64) if np.iscomplexobj(val) else np.ascontiguousarray(val, dtype=np.float64)
        if len(rowptr) != n + 1:
            raise ValueError("rowptr must have n+1 entries")
        h = ctypes.c_void_p()
        check(load().linqt_csr_create(_sh(session), n, _ip(rowptr), _ip(col), _dp(v), storage, ctypes.byref(h)))
        return cls(h, session)

    @classmethod
    def from_file(cls, path, session=None):
        """Read a LinQT CSR file (src/sparse_matrix.cpp:3-50)."""
        from .formats import read_csr
        n, rp, cl, vl = read_csr(path)
        return cls.from_csr(n, rp, cl, vl, session=session)

    def close(self):
        if getattr(self, "h", None):
            check(load().linqt_op_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        n = ctypes.c_int()
        nnz = ctypes.c_long()
        check(load().linqt_op_info(self.h, ctypes.byref(n), ctypes.byref(nnz)))
        return n.value, nnz.value

    def tuned(self):
        """The autotuner's cached decisions for this operator: {key: choice}."""
        ln = ctypes.c_long()
        check(load().linqt_op_tuned(self.h, None, 0, ctypes.byref(ln)))
        buf = ctypes.create_string_buffer(ln.value + 1)
        check(load().linqt_op_tuned(self.h, buf, ln.value + 1, ctypes.byref(ln)))
        out = {}
        for line in buf.value.decode().splitlines():
            k, _, v = line.partition(" ")
            out[k] = v
        return out

    @property
    def n(self):
        return self.info()[0]

    @property
    def nnz(self):
        return self.info()[1]

    def rescale(self, a, b):
        """H <- a*H + b*I (SparseMatrixType::Rescale)."""
        av = np.array([complex(a).real, complex(a).imag])
        bv = np.array([complex(b).real, complex(b).imag])
        check(load().linqt_op_rescale(self.h, _dp(av), _dp(bv)))
        return self

    def rescale_to_chebyshev(self, band_width, band_center):
        """Moments::Rescale2ChebyshevDomain: H <- H/a - (c/a) I, a = band_width/2."""
        a = band_width / 2.0
        return self.rescale(1.0 / a, -band_center / a)

    def multiply(self, x, a=1.0, b=0.0, y=None, session=None):
        """y <- a*H*x + b*y for one vector (N,) or a column block (N, ncols) (column-major semantics)."""
        x = _c128(x)
        single = x.ndim == 1
        X = x.reshape(-1, 1) if single else x
        n, ncols = X.shape
        # the C ABI takes ncols column-major vectors: transpose to (ncols, n) contiguous
        # (copies: with one column the transpose is already contiguous and would alias the caller's arrays)
        xt = np.array(X.T, order="C", copy=True)
        yt = np.zeros_like(xt) if y is None else np.array(_c128(y).reshape(n, ncols).T, order="C", copy=True)
        av = np.array([complex(a).real, complex(a).imag])
        bv = np.array([complex(b).real, complex(b).imag])
        check(load().linqt_op_multiply(_sh(session or self.session), self.h, _dp(av), _dp(xt.view(np.float64)),
                                       _dp(bv), _dp(yt.view(np.float64)), ncols))
        out = yt.T
        return out.reshape(-1) if single else np.ascontiguousarray(out)

    def spectral_bounds(self, session=None):
        lo, hi = ctypes.c_double(), ctypes.c_double()
        check(load().linqt_spectral_bounds(_sh(session or self.session), self.h, ctypes.byref(lo), ctypes.byref(hi)))
        return lo.value, hi.value


def _oph(op):
    return None if op is None else op.h


def moments1d(H, op, states, M, opts=None, session=None):
    """mu[M] of chebyshev::SpectralMoments over the R states (rows of `states`)."""
    st = np.atleast_2d(_c128(states))
    R = st.shape[0]
    mu = np.zeros(M, np.complex128)
    o = opts or make_opts()
    check(load().linqt_moments1d(_sh(session), H.h, _oph(op), _dp(st.view(np.float64)), R, M, ctypes.byref(o),
                                 _dp(mu.view(np.float64))))
    return mu


def moments1d_nonorth(H, op, S, states, M, tol=1e-4, maxit=2000, opts=None, session=None):
    """chebyshev::SpectralMoments_nonOrth: mu[M] in a non-orthogonal basis with overlap S (an
    Operator; build it with storage=STORAGE_GENERAL from the CSR file's arrays to reproduce
    the reference, which solves with the stored triangle).  Returns (mu, BiCGSTAB iterations
    summed over all solves)."""
    st = np.atleast_2d(_c128(states))
    R = st.shape[0]
    mu = np.zeros(M, np.complex128)
    its = ctypes.c_long()
    o = opts or make_opts()
    check(load().linqt_moments1d_nonorth(_sh(session), H.h, _oph(op), S.h, _dp(st.view(np.float64)), R, M, tol,
                                         maxit, ctypes.byref(o), _dp(mu.view(np.float64)), ctypes.byref(its)))
    return mu, its.value


def moments1d_nonorth_dev(H, op, S, states_dev, R, M, mu_dev, tol=1e-4, maxit=2000, opts=None, session=None,
                          iterations=False):
    """Device-pointer form; with iterations=True it synchronises and returns the iteration count."""
    its = ctypes.c_long()
    o = opts or make_opts()
    check(load().linqt_moments1d_nonorth_dev(_sh(session), H.h, _oph(op), S.h, ctypes.c_void_p(_ptr(states_dev)), R,
                                             M, tol, maxit, ctypes.byref(o), ctypes.c_void_p(_ptr(mu_dev)),
                                             ctypes.byref(its) if iterations else None))
    return its.value if iterations else None


def random_phase_states_dev(N, R, seed, out_dev, session=None):
    """R random-phase states (R x N complex128, device) from the seeded Philox generator;
    equal to lattices.random_phase_states(N, R, seed) up to the last bit of sin/cos."""
    check(load().linqt_random_phase_states_dev(_sh(session), N, R, seed, ctypes.c_void_p(_ptr(out_dev))))


def _handles(Hs):
    return (ctypes.c_void_p * len(Hs))(*[H.h.value if isinstance(H.h, ctypes.c_void_p) else H.h for H in Hs])


def moments1d_realisations(Hs, states, M, opts=None, session=None):
    """mu[S, M]: SpectralMoments of S Hamiltonians with one sparsity pattern (disorder
    realisations), the R/S consecutive rows of `states` per realisation, in one recursion."""
    st = np.atleast_2d(_c128(states))
    R, S = st.shape[0], len(Hs)
    mu = np.zeros((S, M), np.complex128)
    o = opts or make_opts()
    check(load().linqt_moments1d_realisations(_sh(session), _handles(Hs), S, _dp(st.view(np.float64)), R, M,
                                              ctypes.byref(o), _dp(mu.view(np.float64))))
    return mu


def moments1d_realisations_dev(Hs, states_dev, R, M, mu_dev, opts=None, session=None):
    o = opts or make_opts()
    check(load().linqt_moments1d_realisations_dev(_sh(session), _handles(Hs), len(Hs), ctypes.c_void_p(_ptr(states_dev)),
                                                  R, M, ctypes.byref(o), ctypes.c_void_p(_ptr(mu_dev))))


def moments1d_dev(H, op, states_dev, R, M, mu_dev, opts=None, session=None):
    o = opts or make_opts()
    check(load().linqt_moments1d_dev(_sh(session), H.h, _oph(op), ctypes.c_void_p(_ptr(states_dev)), R, M,
                                     ctypes.byref(o), ctypes.c_void_p(_ptr(mu_dev))))


def moments1d_noalloc(H, states_dev, R, M, mu_dev, stream=0):
    """1D moments (identity operator, FP64) with no device allocation: scratch lives in a
    fixed static device array (see linqt_moments1d_noalloc in include/linqt_gpu.h)."""
    check(load().linqt_moments1d_noalloc(H.h, ctypes.c_void_p(_ptr(states_dev)), R, M, ctypes.c_void_p(_ptr(mu_dev)),
                                         ctypes.c_void_p(stream)))


def moments_td(H, opl, opr, states, M, NT, dt, band_width, band_center, opts=None, session=None):
    """TimeDependentCorrelations: mu[m, n] (M x NT) at times n*dt (fs); H rescaled with
    band_width / band_center (eV)."""
    st = _c128(np.atleast_2d(states))
    R = st.shape[0]
    mu = np.zeros((M, NT), np.complex128)
    o = opts or make_opts()
    check(load().linqt_moments_td(_sh(session), H.h, _oph(opl), _oph(opr), _dp(st.view(np.float64)), R, M, NT, dt,
                                  band_width, band_center, ctypes.byref(o), _dp(mu.view(np.float64))))
    return mu


def time_correlation_from_moments(mu, N, band_width, band_center, dt, broad_meV, energy, session=None):
    """timeCorrelationsFromChebmom: (t, C(t)) from a TD moment table mu[M, NT]."""
    m = _c128(mu)
    M, NT = m.shape
    t, c = np.zeros(NT), np.zeros(NT)
    used = ctypes.c_int()
    check(load().linqt_time_correlation_from_moments(_sh(session), _dp(m.view(np.float64)), M, NT, N, band_width,
                                                     band_center, dt, broad_meV, energy, _dp(t), _dp(c),
                                                     ctypes.byref(used)))
    return t, c


def moments_td_dev(H, opl, opr, states_dev, R, M, NT, dt, band_width, band_center, mu_dev, opts=None, session=None):
    o = opts or make_opts()
    check(load().linqt_moments_td_dev(_sh(session), H.h, _oph(opl), _oph(opr), ctypes.c_void_p(_ptr(states_dev)), R, M,
                                      NT, dt, band_width, band_center, ctypes.byref(o), ctypes.c_void_p(_ptr(mu_dev))))


def moments2d(H, opl, opr, states, M, opts=None, session=None):
    """mu[M, M] of chebyshev::CorrelationExpansionMoments (row index follows OPL)."""
    st = np.atleast_2d(_c128(states))
    R = st.shape[0]
    mu = np.zeros((M, M), np.complex128)
    o = opts or make_opts()
    check(load().linqt_moments2d(_sh(session), H.h, _oph(opl), _oph(opr), _dp(st.view(np.float64)), R, M,
                                 ctypes.byref(o), _dp(mu.view(np.float64))))
    return mu


def moments2d_dev(H, opl, opr, states_dev, R, M, mu_dev, opts=None, session=None):
    o = opts or make_opts()
    check(load().linqt_moments2d_dev(_sh(session), H.h, _oph(opl), _oph(opr), ctypes.c_void_p(_ptr(states_dev)), R,
                                     M, ctypes.byref(o), ctypes.c_void_p(_ptr(mu_dev))))


def kubo_fft(H, opl, opr, states, M, nump, formula, band_width, band_center, opts=None, session=None):
    """(E, sigma, integrand) of Kubo_solver_FFT with one section, nump >= M."""
    st = np.atleast_2d(_c128(states))
    R = st.shape[0]
    E, s, integ = np.zeros(nump), np.zeros(nump), np.zeros(nump)
    o = opts or make_opts()
    check(load().linqt_kubo_fft(_sh(session), H.h, _oph(opl), _oph(opr), _dp(st.view(np.float64)), R, M, nump,
                                formula, band_width, band_center, ctypes.byref(o), _dp(E), _dp(s), _dp(integ)))
    return E, s, integ


def kubo_fft_dev(H, opl, opr, states_dev, R, M, nump, formula, band_width, band_center, out_dev, opts=None,
                 session=None):
    o = opts or make_opts()
    check(load().linqt_kubo_fft_dev(_sh(session), H.h, _oph(opl), _oph(opr), ctypes.c_void_p(_ptr(states_dev)), R, M,
                                    nump, formula, band_width, band_center, ctypes.byref(o),
                                    ctypes.c_void_p(_ptr(out_dev))))


def kubo_bastin(H, opl, opr, states, M, nump, band_width, band_center, want_mu=True, want_fft=True, opts=None,
                session=None):
    """One Kubo-Bastin solve: (mu[M, M] or None, (E, sigma, integrand) or None)."""
    st = np.atleast_2d(_c128(states))
    R = st.shape[0]
    mu = np.zeros((M, M), np.complex128) if want_mu else None
    E, s, integ = (np.zeros(nump), np.zeros(nump), np.zeros(nump)) if want_fft else (None, None, None)
    o = opts or make_opts()
    nul = ctypes.POINTER(ctypes.c_double)()
    check(load().linqt_kubo_bastin(_sh(session), H.h, _oph(opl), _oph(opr), _dp(st.view(np.float64)), R, M, nump,
                                   band_width, band_center, ctypes.byref(o),
                                   _dp(mu.view(np.float64)) if want_mu else nul,
                                   _dp(E) if want_fft else nul, _dp(s) if want_fft else nul,
                                   _dp(integ) if want_fft else nul))
    return mu, ((E, s, integ) if want_fft else None)


def kubo_bastin_host_ptr(H, opl, opr, states_ptr, R, M, nump, band_width, band_center, mu_ptr, E_ptr, sigma_ptr,
                         opts=None, session=None):
    """Same as kubo_bastin with raw host pointers (e.g. pinned torch tensors)."""
    o = opts or make_opts()
    P = ctypes.POINTER(ctypes.c_double)
    check(load().linqt_kubo_bastin(_sh(session), H.h, _oph(opl), _oph(opr), ctypes.cast(states_ptr, P), R, M, nump,
                                   band_width, band_center, ctypes.byref(o), ctypes.cast(mu_ptr, P),
                                   ctypes.cast(E_ptr, P), ctypes.cast(sigma_ptr, P), P()))


def kubo_bastin_dev(H, opl, opr, states_dev, R, M, nump, band_width, band_center, mu_dev, out_dev, opts=None,
                    session=None):
    o = opts or make_opts()
    check(load().linqt_kubo_bastin_dev(_sh(session), H.h, _oph(opl), _oph(opr), ctypes.c_void_p(_ptr(states_dev)), R,
                                       M, nump, band_width, band_center, ctypes.byref(o),
                                       ctypes.c_void_p(_ptr(mu_dev)), ctypes.c_void_p(_ptr(out_dev))))


def dos_from_moments(mu, N, band_width, band_center, broad_meV, session=None):
    """Jackson kernel + DOS on the Chebyshev grid (spectralFunctionFromChebmom_FFTgrid)."""
    m = _c128(mu)
    M = len(m)
    E, d = np.zeros(M), np.zeros(M)
    n = ctypes.c_int()
    check(load().linqt_dos_from_moments(_sh(session), _dp(m.view(np.float64)), M, N, band_width, band_center,
                                        broad_meV, _dp(E), _dp(d), ctypes.byref(n)))
    return E[: n.value], d[: n.value]


def spectral_function_from_moments(mu, N, band_width, band_center, broad_meV, grid=0, num_div=0, session=None):
    """Jackson kernel + spectral function: grid GRID_UNIFORM (spectralFunctionFromChebmom, 30 M'
    points in [-1, 1], end points non-finite) or GRID_CHEBYSHEV (the _FFTgrid variant, M' points,
    absolute values)."""
    m = _c128(mu)
    M = len(m)
    n_max = num_div if num_div > 0 else (30 * M if grid == GRID_UNIFORM else M)  # M' <= M
    E, d = np.zeros(n_max), np.zeros(n_max)
    n = ctypes.c_int()
    check(load().linqt_spectral_function_from_moments(_sh(session), _dp(m.view(np.float64)), M, N, band_width,
                                                      band_center, broad_meV, grid, num_div, _dp(E), _dp(d),
                                                      ctypes.byref(n)))
    return E[: n.value], d[: n.value]


def bastin_from_moments(mu, N, band_width, band_center, broad_meV, xbound=0.99, num_div=0, session=None):
    """Jackson kernel + Kubo-Bastin conductivity (kuboBastinFromChebmom)."""
    m = _c128(mu)
    M0, M1 = m.shape
    nd = num_div if num_div > 0 else 30 * max(M0, M1)
    E, s = np.zeros(nd), np.zeros(nd)
    n = ctypes.c_int()
    check(load().linqt_bastin_from_moments(_sh(session), _dp(m.view(np.float64)), M0, M1, N, band_width,
                                           band_center, broad_meV, xbound, num_div, _dp(E), _dp(s), ctypes.byref(n)))
    return E[: n.value], s[: n.value]


SUM_VARIANTS = {"bastin": 0, "greenwood": 1, "bastin_I": 2, "bastin_II": 3, "bastin_sea": 4, "bastin_surf": 5}
GRID_UNIFORM, GRID_CHEBYSHEV, GRID_CHEBYSHEV_ASCENDING = 0, 1, 2


def kubo_from_moments(mu, N, band_width, band_center, broad_meV, variant="bastin", grid=GRID_UNIFORM, xbound=1.0,
                      num_div=0, session=None):
    """(E, column) of LinQT's energy-sum post-processor `variant` (kubo*FromChebmom*) on a 2D table,
    Jackson kernel included; see linqt_kubo_from_moments in include/linqt_gpu.h."""
    m = np.ascontiguousarray(mu, dtype=np.complex128)
    M0, M1 = m.shape
    cap = num_div if num_div > 0 else 30 * max(M0, M1)
    E, out = np.zeros(cap), np.zeros(cap)
    n = ctypes.c_int()
    check(load().linqt_kubo_from_moments(_sh(session), _dp(m.view(np.float64)), M0, M1, N, band_width, band_center,
                                         broad_meV, SUM_VARIANTS[variant], grid, xbound, num_div, _dp(E), _dp(out),
                                         ctypes.byref(n)))
    return E[: n.value], out[: n.value]


def jackson1d(mu, band_width, broad_meV):
    m = _c128(mu).copy()
    n = ctypes.c_int()
    check(load().linqt_jackson1d(_dp(m.view(np.float64)), len(m), band_width, broad_meV, ctypes.byref(n)))
    return m[: n.value]


def jackson2d(mu, band_width, b0, b1):
    m = _c128(mu).copy()
    M0, M1 = m.shape
    a, b = ctypes.c_int(), ctypes.c_int()
    check(load().linqt_jackson2d(_dp(m.view(np.float64)), M0, M1, band_width, b0, b1, ctypes.byref(a),
                                 ctypes.byref(b)))
    return m.reshape(-1)[: a.value * b.value].reshape(a.value, b.value)


def locality_order(rowptr, col, part_rows=8192):
    """The locality order behind FORMAT_LOCAL (host only): order[pos] = row."""
    rp = np.ascontiguousarray(rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(col, dtype=np.int32)
    n = len(rp) - 1
    out = np.empty(max(n, 0), dtype=np.int32)
    check(load().linqt_locality_order(n, _ip(rp), _ip(ci), part_rows, _ip(out)))
    return out


# --- operator builder (LinQT's utilities/wannier2sparse) ---------------------------------------
W2S_OPERATORS = ["VX", "VY", "VZ", "VXSX", "VXSY", "VXSZ", "VYSX", "VYSY", "VYSZ", "VZSX", "VZSY", "VZSZ",
                 "SX", "SY", "SZ", "TX", "TY", "TZ"]


class TBModel:
    """A Wannier90 tight-binding model (LABEL.xyz, LABEL.uc, LABEL_hr.dat) and the supercell
    operators wannier2sparse builds from it, assembled on the GPU (linqt_supercell_*)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def load(cls, label):
        h = ctypes.c_void_p()
        check(load().linqt_tbmodel_load(label.encode(), ctypes.byref(h)))
        return cls(h)

    def close(self):
        if getattr(self, "h", None):
            check(load().linqt_tbmodel_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        """(orbitals per cell, hoppings kept from the _hr.dat file)."""
        n, k = ctypes.c_int(), ctypes.c_long()
        check(load().linqt_tbmodel_info(self.h, ctypes.byref(n), ctypes.byref(k)))
        return n.value, k.value

    @staticmethod
    def _dims(cell_dim):
        d = np.ascontiguousarray(cell_dim, dtype=np.int32)
        if d.shape != (3,):
            raise ValueError("cell_dim must hold 3 integers")
        return d

    def csr_size(self, op, cell_dim, session=None):
        """(n, nnz) of the upper-triangle CSR of `op` on the supercell."""
        d = self._dims(cell_dim)
        n, nnz = ctypes.c_int(), ctypes.c_long()
        check(load().linqt_supercell_csr(_sh(session), self.h, op.encode(), _ip(d), ctypes.byref(n),
                                         ctypes.byref(nnz), None, None, None, 0))
        return n.value, nnz.value

    def supercell_csr(self, op, cell_dim, session=None):
        """(n, rowptr, col, val complex128): the matrix of LABEL.op.CSR as wannier2sparse writes it."""
        d = self._dims(cell_dim)
        n, nnz = self.csr_size(op, cell_dim, session)
        rp = np.zeros(n + 1, dtype=np.int32)
        cl = np.zeros(max(nnz, 1), dtype=np.int32)
        vl = np.zeros(max(nnz, 1), dtype=np.complex128)
        n2, nnz2 = ctypes.c_int(), ctypes.c_long()
        check(load().linqt_supercell_csr(_sh(session), self.h, op.encode(), _ip(d), ctypes.byref(n2),
                                         ctypes.byref(nnz2), _ip(rp), _ip(cl), _dp(vl.view(np.float64)), len(cl)))
        return n2.value, rp, cl[: nnz2.value], vl[: nnz2.value]

    def supercell_csr_dev(self, op, cell_dim, rowptr_dev, col_dev, val_dev, capacity, session=None):
        """Fill device buffers (torch tensors or pointers) on the session stream; returns (n, nnz)."""
        d = self._dims(cell_dim)
        n, nnz = ctypes.c_int(), ctypes.c_long()
        check(load().linqt_supercell_csr_dev(_sh(session), self.h, op.encode(), _ip(d), ctypes.byref(n),
                                             ctypes.byref(nnz), _ptr(rowptr_dev), _ptr(col_dev), _ptr(val_dev),
                                             capacity))
        return n.value, nnz.value

    def write_csr(self, op, cell_dim, path, session=None):
        """Write LABEL.op.CSR (the bytes wannier2sparse writes)."""
        d = self._dims(cell_dim)
        check(load().linqt_supercell_write_csr(_sh(session), self.h, op.encode(), _ip(d), path.encode()))

    def operator(self, op, cell_dim, session=None):
        """The supercell operator as a device Operator (Hermitian-upper, like the file)."""
        d = self._dims(cell_dim)
        h = ctypes.c_void_p()
        check(load().linqt_supercell_operator(_sh(session), self.h, op.encode(), _ip(d), ctypes.byref(h)))
        return Operator(h, session)
