"""Seeded synthetic tight-binding operators and random-phase states.

These stand in for the operators LinQT reads from operators/<LABEL>.<OP>.CSR
(written by its wannier2sparse tool): every builder returns the upper triangle
(col >= row, diagonal included, rows sorted by column) of a Hermitian matrix, as
utilities/wannier2sparse/src/hopping_list.cpp:253 writes it.  Velocity operators
follow utilities/wannier2sparse/src/tbmodel.cpp:92-126:  V_x = i (x_i - x_j) H_ij
with minimum-image bond vectors.

Random numbers come from Philox4x32-10 (Salmon et al., "Parallel random numbers:
as easy as 1, 2, 3", SC'11), restated here in numpy: key = (seed lo, seed hi),
counter = (index lo, index hi, stream, 0); a double u = (x >> 11) * 2^-53 from the
first two output words x = (w0 << 32) | w1.
"""
import numpy as np

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = 0x9E3779B9, 0xBB67AE85
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32 with 10 rounds on uint32 counter arrays (returned as uint64 arrays)."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint64) & _MASK for c in (c0, c1, c2, c3))
    k0, k1 = int(k0) & 0xFFFFFFFF, int(k1) & 0xFFFFFFFF
    for _ in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0
        k0 = (k0 + _W0) & 0xFFFFFFFF
        k1 = (k1 + _W1) & 0xFFFFFFFF
    return c0, c1, c2, c3


def uniform(seed, n, stream=0, offset=0):
    """n doubles in [0, 1) for counters offset .. offset+n-1."""
    idx = np.arange(offset, offset + n, dtype=np.uint64)
    w0, w1, _, _ = philox4x32_10(idx & _MASK, idx >> np.uint64(32), np.full(n, stream, np.uint64),
                                 np.zeros(n, np.uint64), seed & 0xFFFFFFFF, seed >> 32)
    x = (w0 << np.uint64(32)) | w1
    return (x >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def random_phase_states(N, R, seed):
    """R states r_i = exp(i phi_i)/sqrt(N), phi uniform in [0, 2 pi) (cf. qstates::FillWithRandomPhase,
    include/quantum_states.hpp:231-252, which LinQT never calls)."""
    u = uniform(seed, N * R).reshape(R, N)
    return np.exp(2j * np.pi * u) / np.sqrt(N)


def disorder(N, W, seed):
    """Anderson on-site energies W*(u - 1/2)."""
    return W * (uniform(seed, N) - 0.5)


def upper_csr(n, rows, cols, vals):
    """Upper-triangle CSR (col >= row) of the Hermitian matrix with H[r, c] = v for the given
    entries; an entry below the diagonal is stored as its conjugate at (c, r).  Duplicates are summed."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.complex128)
    low = cols < rows
    r = np.where(low, cols, rows)
    c = np.where(low, rows, cols)
    v = np.where(low, np.conj(vals), vals)
    key = r * n + c
    order = np.argsort(key, kind="stable")
    key, v = key[order], v[order]
    uk, start = np.unique(key, return_index=True)
    vs = np.add.reduceat(v, start) if len(v) else v
    r, c = uk // n, uk % n
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, r + 1, 1)
    rowptr = np.cumsum(rowptr)
    return rowptr.astype(np.int32), c.astype(np.int32), vs


def hermitian_dense(n, rowptr, col, val):
    """Dense Hermitian matrix of an upper-stored CSR (tests only; small n)."""
    H = np.zeros((n, n), np.complex128)
    for i in range(n):
        for k in range(rowptr[i], rowptr[i + 1]):
            j = col[k]
            if j < i:
                continue
            H[i, j] = val[k]
            if j != i:
                H[j, i] = np.conj(val[k])
    return H


def square_lattice(L, t=1.0, W=1.0, seed=11):
    """2D square lattice L x L, periodic, hopping t, Anderson disorder W (5 non-zeros per row)."""
    N = L * L
    x, y = np.meshgrid(np.arange(L), np.arange(L), indexing="ij")
    i = (x + L * y).ravel()
    jx = (((x + 1) % L) + L * y).ravel()
    jy = (x + L * ((y + 1) % L)).ravel()
    eps = disorder(N, W, seed)
    rows = np.concatenate([np.arange(N), i, i])
    cols = np.concatenate([np.arange(N), jx, jy])
    vals = np.concatenate([eps, np.full(N, t), np.full(N, t)]).astype(np.complex128)
    return N, upper_csr(N, rows, cols, vals)


def cubic_lattice(L, t=1.0, W=2.0, seed=41):
    """3D cubic lattice L^3, periodic, 7-point stencil."""
    N = L ** 3
    g = np.arange(N)
    x, y, z = g % L, (g // L) % L, g // (L * L)
    idx = lambda a, b, c: (a % L) + L * ((b % L) + L * (c % L))
    eps = disorder(N, W, seed)
    rows = np.concatenate([g, g, g, g])
    cols = np.concatenate([g, idx(x + 1, y, z), idx(x, y + 1, z), idx(x, y, z + 1)])
    vals = np.concatenate([eps, np.full(3 * N, t)]).astype(np.complex128)
    return N, upper_csr(N, rows, cols, vals)


def _honeycomb_geometry(Lx, Ly, a):
    """Site positions and NN bonds (A -> B) of a periodic honeycomb, armchair along x:
    NN vectors d1 = (a, 0), d2 = (-a/2, sqrt(3) a/2), d3 = (-a/2, -sqrt(3) a/2)."""
    d = np.array([[a, 0.0], [-a / 2, np.sqrt(3) * a / 2], [-a / 2, -np.sqrt(3) * a / 2]])
    a1, a2 = d[0] - d[1], d[0] - d[2]
    ci, cj = np.meshgrid(np.arange(Lx), np.arange(Ly), indexing="ij")
    ci, cj = ci.ravel(), cj.ravel()
    cell = ci + Lx * cj
    A, B = 2 * cell, 2 * cell + 1
    cellid = lambda i, j: (i % Lx) + Lx * (j % Ly)
    # A(i,j) - B(i,j) [d1], A(i,j) - B(i-1,j) [d2], A(i,j) - B(i,j-1) [d3]
    nb = [(A, 2 * cellid(ci, cj) + 1, d[0]), (A, 2 * cellid(ci - 1, cj) + 1, d[1]),
          (A, 2 * cellid(ci, cj - 1) + 1, d[2])]
    return A, B, ci, cj, cellid, a1, a2, d, nb


def honeycomb(Lx, Ly, t=-2.7, W=1.0, seed=21, a=1.42):
    """Graphene (2 sites per cell), hopping t, Anderson disorder W; returns (N, H, V_x)."""
    A, B, ci, cj, cellid, a1, a2, d, nb = _honeycomb_geometry(Lx, Ly, a)
    N = 2 * Lx * Ly
    eps = disorder(N, W, seed)
    rows, cols, hv, vv = [np.arange(N)], [np.arange(N)], [eps.astype(np.complex128)], [np.zeros(N, np.complex128)]
    for src, dst, dv in nb:
        rows.append(src)
        cols.append(dst)
        hv.append(np.full(len(src), t, np.complex128))
        # V_x = i (x_src - x_dst) H = -i d_x H
        vv.append(np.full(len(src), -1j * dv[0] * t, np.complex128))
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    H = upper_csr(N, rows, cols, np.concatenate(hv))
    V = _drop_zeros(upper_csr(N, rows, cols, np.concatenate(vv)))
    return N, H, V


def _drop_zeros(csr):
    rp, c, v = csr
    n = len(rp) - 1
    keep = v != 0
    counts = np.add.reduceat(keep.astype(np.int64), rp[:-1]) if len(v) else np.zeros(n, np.int64)
    counts = np.where(np.diff(rp) > 0, counts, 0)
    rp2 = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return rp2, c[keep], v[keep]


def kane_mele(Lx, Ly, t=1.0, lam_so=0.06, lam_r=0.05, W=0.5, seed=31, a=1.0):
    """Kane-Mele honeycomb with spin (4 orbitals per cell: A-up, A-dn, B-up, B-dn).

    H = t sum_<ij> c+_i c_j + i lam_so sum_<<ij>> nu_ij c+_i s_z c_j + i lam_r sum_<ij> c+_i (s x d_ij)_z c_j
        + sum_i eps_i c+_i c_i
    with nu_ij = sign((d_ik x d_kj)_z) through the common neighbour k and d_ij the unit NN vector.
    Returns (N, H, J) with J = {s_z, V_x}/2 the spin-velocity operator."""
    A, B, ci, cj, cellid, a1, a2, d, nb = _honeycomb_geometry(Lx, Ly, a)
    ns = 2 * Lx * Ly  # spatial sites
    N = 2 * ns
    sx = np.array([[0, 1], [1, 0]], np.complex128)
    sy = np.array([[0, -1j], [1j, 0]], np.complex128)
    sz = np.array([[1, 0], [0, -1]], np.complex128)
    eps = disorder(N, W, seed)
    bonds = []  # (src spatial, dst spatial, displacement, 2x2 hopping)
    for src, dst, dv in nb:
        u = dv / np.linalg.norm(dv)
        hr = 1j * lam_r * (sx * u[1] - sy * u[0])
        bonds.append((src, dst, dv, t * np.eye(2) + hr))
    # NNN: A(R) -> A(R + e) and B(R) -> B(R + e) for e in {a1, a2, a2 - a1}
    Bsite = lambda i, j: 2 * cellid(i, j) + 1
    for (di, dj), e in (((1, 0), a1), ((0, 1), a2), ((-1, 1), a2 - a1)):
        for sub in (0, 1):
            src = 2 * cellid(ci, cj) + sub
            dst = 2 * cellid(ci + di, cj + dj) + sub
            # common neighbour k: R + d_k = R + e + d_m for NN vectors d_k, d_m of this sublattice
            nbr = d if sub == 0 else -d
            k = None
            for dk in nbr:
                for dm in nbr:
                    if np.allclose(dk, e + dm):
                        k = (dk, e - dk)
            d1v, d2v = k
            nu = np.sign(d1v[0] * d2v[1] - d1v[1] * d2v[0])
            bonds.append((src, dst, e, 1j * lam_so * nu * sz))
    rows, cols, hv, jv = [np.arange(N)], [np.arange(N)], [eps.astype(np.complex128)], [np.zeros(N, np.complex128)]
    for src, dst, dv, h in bonds:
        for s1 in range(2):
            for s2 in range(2):
                if h[s1, s2] == 0:
                    continue
                rows.append(2 * src + s1)
                cols.append(2 * dst + s2)
                hv.append(np.full(len(src), h[s1, s2]))
                v = -1j * dv[0] * h[s1, s2]  # V_x = i (x_src - x_dst) H
                jv.append(np.full(len(src), v * (sz[s1, s1] + sz[s2, s2]) / 2))
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    H = upper_csr(N, rows, cols, np.concatenate(hv))
    J = _drop_zeros(upper_csr(N, rows, cols, np.concatenate(jv)))
    return N, H, J


def overlap_matrix(N, H, s=0.08, seed=13):
    """Upper-triangle CSR of an overlap matrix S = I + (off-diagonal entries on H's bonds) for a
    non-orthogonal basis: S_ij = s e^{i theta_ij} with theta_ij uniform in [0, 2 pi) (Philox,
    seed), on every bond (i < j) of H's upper triangle.  Positive definite when s times the
    bonds per row stays below 1."""
    rp, col, _ = H
    rows = np.repeat(np.arange(N), np.diff(rp))
    off = col > rows
    r, c = rows[off], col[off].astype(np.int64)
    th = 2 * np.pi * uniform(seed, len(r))
    vals = np.concatenate([np.ones(N), s * np.exp(1j * th)])
    return upper_csr(N, np.concatenate([np.arange(N), r]), np.concatenate([np.arange(N), c]), vals)


def gershgorin_bounds(n, rowptr, col, val):
    """Gershgorin interval of the Hermitian matrix stored as upper CSR (host, for tests)."""
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    diag = np.zeros(n)
    rad = np.zeros(n)
    on = col == rows
    np.add.at(diag, rows[on], val[on].real)
    off = ~on
    np.add.at(rad, rows[off], np.abs(val[off]))
    np.add.at(rad, col[off], np.abs(val[off]))
    return float((diag - rad).min()), float((diag + rad).max())


def wannier_model(label, orbitals=18, reach=3, seed=7, three_d=False):
    """Write a synthetic Wannier90 model LABEL_hr.dat / LABEL.xyz / LABEL.uc and return its
    number of hopping lines.  `orbitals` spinful orbitals (spin-down block second, labels
    _s+_ / _s-_) on a hexagonal cell; a hopping between every orbital pair for every cell
    vector with |R_i| <= reach (R_z = 0 unless three_d), magnitudes decaying as exp(-|R|),
    Hermitian (t(-R) = t(R)^H) and printed with 6 decimals as Wannier90 does."""
    rng = np.random.default_rng(seed)
    rz = reach if three_d else 0
    Rs = [(x, y, z) for x in range(-reach, reach + 1) for y in range(-reach, reach + 1) for z in range(-rz, rz + 1)]
    A = {R: (rng.normal(size=(orbitals, orbitals)) + 1j * rng.normal(size=(orbitals, orbitals)))
         * np.exp(-np.sqrt(R[0] ** 2 + R[1] ** 2 + R[2] ** 2)) for R in Rs}
    lines = []
    for R in Rs:
        mR = (-R[0], -R[1], -R[2])
        t = 0.5 * (A[R] + A[mR].conj().T)
        for n in range(orbitals):
            for m in range(orbitals):
                v = t[m, n]
                lines.append("%5d%5d%5d%5d%5d%12.6f%12.6f" % (R[0], R[1], R[2], m + 1, n + 1, v.real, v.imag))
    deg = ["    1" * min(15, len(Rs) - i) for i in range(0, len(Rs), 15)]
    with open(label + "_hr.dat", "w") as f:
        f.write(" synthetic model (seed %d)\n%12d\n%12d\n%s\n%s\n" % (seed, orbitals, len(Rs), "\n".join(deg),
                                                                     "\n".join(lines)))
    with open(label + ".uc", "w") as f:
        f.write(" 2.46 0.0 0.0\n 1.23 2.130422 0.0\n 0.0 0.0 %s\n" % ("2.46" if three_d else "20.0"))
    pos = rng.uniform(0.0, 1.0, size=(orbitals // 2, 3)) * np.array([2.0, 1.7, 0.5])
    with open(label + ".xyz", "w") as f:
        f.write("%d\n" % orbitals)
        for s in ("+", "-"):
            for i, p in enumerate(pos):
                f.write("o%d_s%s_ %.8f %.8f %.8f\n" % (i, s, *p))
    return len(lines)
