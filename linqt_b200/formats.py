"""LinQT file formats (byte-compatible writers, tolerant readers).

    CSR operator     src/sparse_matrix.cpp:3-50          "dim nnz" / nnz "re im" / nnz cols / dim+1 row ptrs
    .chebmom1D       src/chebyshev_moments1D.cpp:19-51, 91-103
    .chebmom2D       src/chebyshev_moments2D.cpp:16-68   (two spaces before BandCenter, trailing space
                                                         after the moment counts)
    state files      include/quantum_states.hpp:135-228 ("vector" / "local")

Numbers are written like std::ostream with precision(digits10 = 15), i.e. "%.15g".
"""
import numpy as np


def _g(x):
    return "%.15g" % x


def read_csr(path):
    tok = open(path).read().split()
    dim, nnz = int(tok[0]), int(tok[1])
    v = np.array(tok[2:2 + 2 * nnz], dtype=np.float64)
    col = np.array(tok[2 + 2 * nnz:2 + 3 * nnz], dtype=np.int32)
    rp = np.array(tok[2 + 3 * nnz:2 + 3 * nnz + dim + 1], dtype=np.int32)
    if len(v) != 2 * nnz or len(col) != nnz or len(rp) != dim + 1:
        raise ValueError("truncated CSR file: %s" % path)
    return dim, rp, col, v[0::2] + 1j * v[1::2]


def write_csr(path, n, rowptr, col, val):
    """Values are written with 17 significant digits (lossless for doubles)."""
    val = np.asarray(val, dtype=np.complex128)
    with open(path, "w") as f:
        f.write("%d %d\n" % (n, len(col)))
        f.write(" ".join("%.17g %.17g" % (z.real, z.imag) for z in val) + " \n")
        f.write(" ".join(str(int(c)) for c in col) + " \n")
        f.write(" ".join(str(int(r)) for r in rowptr) + " \n")


def write_chebmom1d(path, system_size, band_width, band_center, mu):
    mu = np.asarray(mu, dtype=np.complex128)
    with open(path, "w") as f:
        f.write("%d %s %s\n" % (system_size, _g(band_width), _g(band_center)))
        f.write("%d\n" % len(mu))
        for z in mu:
            f.write("%s %s\n" % (_g(z.real), _g(z.imag)))


def read_chebmom1d(path):
    if ".chebmom1D" not in path:
        raise ValueError("not a .chebmom1D file: %s" % path)
    tok = open(path).read().split()
    n, bw, bc, M = int(tok[0]), float(tok[1]), float(tok[2]), int(tok[3])
    v = np.array(tok[4:4 + 2 * M], dtype=np.float64)
    if len(v) != 2 * M:
        raise ValueError("truncated .chebmom1D file: %s" % path)
    return n, bw, bc, v[0::2] + 1j * v[1::2]


def write_chebmom2d(path, system_size, band_width, band_center, mu):
    mu = np.asarray(mu, dtype=np.complex128)
    m0, m1 = mu.shape
    with open(path, "w") as f:
        f.write("%d %s  %s\n" % (system_size, _g(band_width), _g(band_center)))
        f.write("%d %d \n" % (m0, m1))
        for z in mu.reshape(-1):
            f.write("%s %s\n" % (_g(z.real), _g(z.imag)))


def read_chebmom2d(path):
    if ".chebmom2D" not in path:
        raise ValueError("not a .chebmom2D file: %s" % path)
    tok = open(path).read().split()
    n, bw, bc = int(tok[0]), float(tok[1]), float(tok[2])
    m0, m1 = int(tok[3]), int(tok[4])
    v = np.array(tok[5:5 + 2 * m0 * m1], dtype=np.float64)
    return n, bw, bc, (v[0::2] + 1j * v[1::2]).reshape(m0, m1)


def write_chebmomtd(path, system_size, band_width, band_center, dt, mu):
    """MomentsTD::saveIn (src/chebyshev_momentsTD.cpp:86-99): header `N bw bc NT dt`, then
    `M NT`, then mu(m, n) row-major, one `re im` per line, 15 digits."""
    mu = np.asarray(mu, dtype=np.complex128)
    m, nt = mu.shape
    with open(path, "w") as f:
        f.write("%d %s %s %d %s \n" % (system_size, _g(band_width), _g(band_center), nt, _g(dt)))
        f.write("%d %d \n" % (m, nt))
        for z in mu.reshape(-1):
            f.write("%s %s\n" % (_g(z.real), _g(z.imag)))


def read_chebmomtd(path):
    """(N, band_width, band_center, dt, mu[M, NT]) of a .chebmomTD file."""
    if ".chebmomTD" not in path:
        raise ValueError("not a .chebmomTD file: %s" % path)
    tok = open(path).read().split()
    n, bw, bc, nt, dt = int(tok[0]), float(tok[1]), float(tok[2]), int(tok[3]), float(tok[4])
    m, nt2 = int(tok[5]), int(tok[6])
    v = np.array(tok[7:7 + 2 * m * nt2], dtype=np.float64)
    return n, bw, bc, dt, (v[0::2] + 1j * v[1::2]).reshape(m, nt2)


def write_vector_states(path, states):
    st = np.atleast_2d(np.asarray(states, dtype=np.complex128))
    R, N = st.shape
    with open(path, "w") as f:
        f.write("vector\n%d %d\n" % (R, N))
        for r in range(R):
            f.write("".join("%s %s\n" % (repr(float(z.real)), repr(float(z.imag))) for z in st[r]))


def read_state_file(path, dim=None):
    """States of a LinQT state file as an (R, N) array; `local` files need dim."""
    tok = open(path).read().split()
    kind = tok[0]
    if kind == "vector":
        R, N = int(tok[1]), int(tok[2])
        v = np.array(tok[3:3 + 2 * R * N], dtype=np.float64)
        if len(v) != 2 * R * N:
            raise ValueError("truncated vector state file: %s" % path)
        return (v[0::2] + 1j * v[1::2]).reshape(R, N)
    if kind == "local":
        R = int(tok[1])
        if dim is None:
            raise ValueError("local states need the system dimension")
        if len(tok) < 2 + R:
            raise ValueError("truncated local state file: %s" % path)
        st = np.zeros((R, dim), np.complex128)
        for r in range(R):
            st[r, int(tok[2 + r])] = 1.0
        return st
    raise ValueError("unknown state kind %r" % kind)


def default_state(dim):
    """LinQT's default "random" state: a unit vector at dim/2 (include/quantum_states.hpp:85-93)."""
    st = np.zeros((1, dim), np.complex128)
    st[0, dim // 2] = 1.0
    return st
