"""Python handle on the oracles (TEST INFRASTRUCTURE ONLY).

Two checkers live under oracle/:

* ``liblinqt_oracle.so`` -- the plain-C restatement of LinQT's hot path
  (linqt_oracle.c), loaded here through ctypes;
* ``_ref/`` -- the reference's own sources compiled unmodified against stand-in
  MKL/FFTW/Eigen headers, driven here through its CLI programs and through
  ``ref_harness`` (a timing harness that calls the reference solvers in-process).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module.  The product package (linqt_b200) never does.
"""
import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblinqt_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build():
    """Compile the oracles (make -C oracle); the _ref part needs the reference checkout."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle library missing: run `make -C oracle`")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.lo_op_from_upper.restype = vp
        L.lo_op_from_upper.argtypes = [ctypes.c_int, ip, ip, dp]
        L.lo_op_free.argtypes = [vp]
        L.lo_op_dim.restype = ctypes.c_int
        L.lo_op_dim.argtypes = [vp]
        L.lo_op_nnz.restype = ctypes.c_long
        L.lo_op_nnz.argtypes = [vp]
        L.lo_op_rescale.argtypes = [vp, ctypes.c_double, ctypes.c_double]
        L.lo_op_mv.argtypes = [vp, dp, dp, dp, dp]
        L.lo_op_export.argtypes = [vp, ip, ip, dp]
        L.lo_moments1d.argtypes = [vp, vp, dp, ctypes.c_int, ctypes.c_int, dp]
        L.lo_moments2d.argtypes = [vp, vp, vp, dp, ctypes.c_int, ctypes.c_int, dp]
        L.lo_time_correlation.restype = ctypes.c_int
        L.lo_time_correlation.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp]
        L.lo_moments_td.argtypes = [vp, vp, vp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, dp]
        L.lo_jackson1d.argtypes = [dp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.lo_jackson2d.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ip, ip]
        L.lo_dos_fftgrid.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp]
        L.lo_moments1d_nonorth.argtypes = [vp, vp, ip, ip, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_int, dp, ctypes.POINTER(ctypes.c_long)]
        L.lo_spectral_function.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int, ctypes.c_int, dp, dp]
        L.lo_bastin_from_moments.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp]
        L.lo_kubo_from_moments.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp]
        L.lo_kubo_fft.argtypes = [vp, vp, vp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _cplx_as_f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).view(np.float64)


class Op:
    """A Hermitian operator held by the C oracle (built from an upper-stored CSR)."""

    def __init__(self, rowptr, col, val):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = _cplx_as_f64(val) if np.iscomplexobj(val) else np.ascontiguousarray(val, dtype=np.float64)
        n = len(self.rowptr) - 1
        self.h = lib().lo_op_from_upper(n, _ip(self.rowptr), _ip(self.col), _dp(self.val))
        if not self.h:
            raise ValueError("invalid CSR")

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.lo_op_free(self.h)
            self.h = None

    @property
    def n(self):
        return lib().lo_op_dim(self.h)

    @property
    def nnz(self):
        return lib().lo_op_nnz(self.h)

    def rescale(self, scale, shift):
        lib().lo_op_rescale(self.h, scale, shift)
        return self

    def mv(self, x, a=1.0, b=0.0, y=None):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros_like(x) if y is None else np.ascontiguousarray(y, dtype=np.complex128).copy()
        av = np.array([complex(a).real, complex(a).imag])
        bv = np.array([complex(b).real, complex(b).imag])
        lib().lo_op_mv(self.h, _dp(av), _dp(x.view(np.float64)), _dp(bv), _dp(y.view(np.float64)))
        return y

    def export(self):
        n, nnz = self.n, self.nnz
        rp = np.zeros(n + 1, np.int32)
        cl = np.zeros(nnz, np.int32)
        vl = np.zeros(2 * nnz, np.float64)
        lib().lo_op_export(self.h, _ip(rp), _ip(cl), _dp(vl))
        return rp, cl, vl.view(np.complex128)


def _h(op):
    return None if op is None else op.h


def moments1d(H, op, states, M):
    st = np.ascontiguousarray(states, dtype=np.complex128)
    R = st.shape[0]
    mu = np.zeros(M, np.complex128)
    rc = lib().lo_moments1d(H.h, _h(op), _dp(st.view(np.float64)), R, M, _dp(mu.view(np.float64)))
    if rc:
        raise RuntimeError("lo_moments1d failed: %d" % rc)
    return mu


def moments1d_nonorth(H, op, S, states, M, tol=1e-4, maxit=2000):
    """SpectralMoments_nonOrth: S = (rowptr, col, val) as stored in its CSR file.
    Returns (mu, BiCGSTAB iterations summed over all solves)."""
    st = np.ascontiguousarray(states, dtype=np.complex128)
    R = st.shape[0]
    rp = np.ascontiguousarray(S[0], dtype=np.int32)
    cl = np.ascontiguousarray(S[1], dtype=np.int32)
    vl = _cplx_as_f64(S[2]) if np.iscomplexobj(S[2]) else np.ascontiguousarray(S[2], dtype=np.float64)
    mu = np.zeros(M, np.complex128)
    its = ctypes.c_long()
    rc = lib().lo_moments1d_nonorth(H.h, _h(op), _ip(rp), _ip(cl), _dp(vl), _dp(st.view(np.float64)), R, M, tol, maxit,
                                    _dp(mu.view(np.float64)), ctypes.byref(its))
    if rc:
        raise RuntimeError("lo_moments1d_nonorth failed: %d" % rc)
    return mu, its.value


def moments_td(H, opl, opr, states, M, NT, dt, band_width, band_center):
    """TimeDependentCorrelations: mu[m, n] (M x NT) for time steps n*dt."""
    st = np.ascontiguousarray(states, dtype=np.complex128)
    R = st.shape[0]
    mu = np.zeros((M, NT), np.complex128)
    rc = lib().lo_moments_td(H.h, _h(opl), _h(opr), _dp(st.view(np.float64)), R, M, NT, ctypes.c_double(dt),
                             ctypes.c_double(band_width), ctypes.c_double(band_center), _dp(mu.view(np.float64)))
    if rc:
        raise RuntimeError("lo_moments_td failed: %d" % rc)
    return mu


def time_correlation(mu, N, band_width, band_center, dt, broad_meV, energy):
    """timeCorrelationsFromChebmom: (t, C(t)) from a TD moment table mu[M, NT]."""
    m = np.ascontiguousarray(mu, dtype=np.complex128)
    M, NT = m.shape
    t, c = np.zeros(NT), np.zeros(NT)
    rc = lib().lo_time_correlation(_dp(m.view(np.float64)), M, NT, N, band_width, band_center, dt, broad_meV, energy,
                                   _dp(t), _dp(c))
    if rc < 0:
        raise RuntimeError("lo_time_correlation failed: %d" % rc)
    return t, c


def moments2d(H, opl, opr, states, M):
    st = np.ascontiguousarray(states, dtype=np.complex128)
    R = st.shape[0]
    mu = np.zeros((M, M), np.complex128)
    rc = lib().lo_moments2d(H.h, _h(opl), _h(opr), _dp(st.view(np.float64)), R, M, _dp(mu.view(np.float64)))
    if rc:
        raise RuntimeError("lo_moments2d failed: %d" % rc)
    return mu


def jackson1d(mu, band_width, broad_meV):
    m = np.ascontiguousarray(mu, dtype=np.complex128).copy()
    Mt = lib().lo_jackson1d(_dp(m.view(np.float64)), len(m), band_width, broad_meV)
    return m[:Mt]


def jackson2d(mu, band_width, b0, b1):
    m = np.ascontiguousarray(mu, dtype=np.complex128).copy()
    M0, M1 = m.shape
    a0, a1 = ctypes.c_int(), ctypes.c_int()
    lib().lo_jackson2d(_dp(m.view(np.float64)), M0, M1, band_width, b0, b1, ctypes.byref(a0), ctypes.byref(a1))
    return m.reshape(-1)[: a0.value * a1.value].reshape(a0.value, a1.value)


def dos_fftgrid(mu, N, band_width, band_center):
    m = np.ascontiguousarray(mu, dtype=np.complex128)
    M = len(m)
    E, d = np.zeros(M), np.zeros(M)
    lib().lo_dos_fftgrid(_dp(m.view(np.float64)), M, N, band_width, band_center, _dp(E), _dp(d))
    return E, d


def spectral_function(mu, N, band_width, band_center, grid=0, num_div=None):
    """spectralFunctionFromChebmom (grid 0, num_div = 30 M) or its _FFTgrid variant (grid 1,
    num_div = M) on Jackson-damped moments."""
    m = np.ascontiguousarray(mu, dtype=np.complex128)
    M = len(m)
    n = num_div or (30 * M if grid == 0 else M)
    E, d = np.zeros(n), np.zeros(n)
    with np.errstate(all="ignore"):
        lib().lo_spectral_function(_dp(m.view(np.float64)), M, N, band_width, band_center, grid, n, _dp(E), _dp(d))
    return E, d


def bastin_from_moments(mu, N, band_width, band_center, xbound=0.99, num_div=None):
    m = np.ascontiguousarray(mu, dtype=np.complex128)
    M0, M1 = m.shape
    if num_div is None:
        num_div = 30 * max(M0, M1)
    E, s = np.zeros(num_div - 1), np.zeros(num_div - 1)
    lib().lo_bastin_from_moments(_dp(m.view(np.float64)), M0, M1, N, band_width, band_center, xbound, num_div,
                                 _dp(E), _dp(s))
    return E, s


# variants and grids of lo_kubo_from_moments
FROM_MOM = {"bastin": 0, "greenwood": 1, "bastin_I": 2, "bastin_II": 3, "bastin_sea": 4, "bastin_surf": 5}
GRID_UNIFORM, GRID_CHEBYSHEV, GRID_CHEBYSHEV_ASCENDING = 0, 1, 2


def kubo_from_moments(mu, N, band_width, band_center, variant, grid=GRID_UNIFORM, xbound=1.0, num_div=None):
    """(E, column) of LinQT's post-processor `variant` on a Jackson-damped table."""
    m = np.ascontiguousarray(mu, dtype=np.complex128)
    M0, M1 = m.shape
    if num_div is None:
        num_div = 30 * max(M0, M1) if grid == GRID_UNIFORM else max(M0, M1)
    E, out = np.zeros(num_div - 1), np.zeros(num_div - 1)
    rc = lib().lo_kubo_from_moments(FROM_MOM[variant], grid, _dp(m.view(np.float64)), M0, M1, N, band_width,
                                    band_center, xbound, num_div, _dp(E), _dp(out))
    if rc:
        raise RuntimeError("lo_kubo_from_moments failed: %d" % rc)
    return E, out


def kubo_fft(H, opl, opr, states, M, nump, formula, N, band_width, band_center):
    st = np.ascontiguousarray(states, dtype=np.complex128)
    R = st.shape[0]
    E, s, integ = np.zeros(nump), np.zeros(nump), np.zeros(nump)
    fin = np.zeros(2 * nump, np.complex128)
    rc = lib().lo_kubo_fft(H.h, _h(opl), _h(opr), _dp(st.view(np.float64)), R, M, nump, formula, N, band_width,
                           band_center, _dp(E), _dp(s), _dp(integ), _dp(fin.view(np.float64)))
    if rc:
        raise RuntimeError("lo_kubo_fft failed: %d" % rc)
    return E, s, integ, fin


# ---------------------------------------------------------------------------
# The reference's own build (oracle/_ref)
# ---------------------------------------------------------------------------

def ref_available():
    return os.path.exists(os.path.join(REF_DIR, "ref_harness"))


def write_csr(path, n, rowptr, col, val):
    """Write a CSR in the reference's text format (src/sparse_matrix.cpp:3-50)."""
    val = np.asarray(val, dtype=np.complex128)
    with open(path, "w") as f:
        f.write("%d %d\n" % (n, len(col)))
        f.write(" ".join("%.17g %.17g" % (v.real, v.imag) for v in val) + "\n")
        f.write(" ".join(str(int(c)) for c in col) + "\n")
        f.write(" ".join(str(int(r)) for r in rowptr) + "\n")


def write_vector_states(path, states):
    """Write a `vector` state file (include/quantum_states.hpp:155-183)."""
    st = np.asarray(states, dtype=np.complex128)
    R, N = st.shape
    with open(path, "w") as f:
        f.write("vector\n%d %d\n" % (R, N))
        for r in range(R):
            f.write("\n".join("%.17g %.17g" % (v.real, v.imag) for v in st[r]) + "\n")


def run_ref_harness(args, workdir, threads=None, timeout=3600):
    """Run oracle/_ref/ref_harness in workdir; returns its JSON result."""
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    p = subprocess.run([os.path.join(REF_DIR, "ref_harness")] + [str(a) for a in args], cwd=workdir, env=env,
                       capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError("ref_harness failed (%d): %s" % (p.returncode, p.stderr[-2000:]))
    for line in reversed(p.stdout.splitlines()):
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError("ref_harness printed no result")


def ref_workdir():
    return tempfile.mkdtemp(prefix="linqt_ref_")
