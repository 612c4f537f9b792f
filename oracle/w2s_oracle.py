"""CPU restatement of LinQT's operator builder, utilities/wannier2sparse (TEST INFRASTRUCTURE ONLY).

wannier2sparse turns a Wannier90 tight-binding model (LABEL_hr.dat, LABEL.xyz, LABEL.uc)
into the upper-triangle CSR text files the KPM solvers read (LABEL.HAM.CSR and one file
per requested operator: velocities, spin densities, spin currents, torques, spinorial
LABEL.OP files), for a supercell of Dim0 x Dim1 x Dim2 unit cells.  This module follows
the reference step by step, with plain Python data structures standing in for its
std::multimap<string, hopping> and Eigen triplets:

  * parsing        utilities/wannier2sparse/src/wannier_parser.cpp:45-117
  * hopping filter src/hopping_list.cpp:114-155 (|t| / mean|t| > 1e-10, file order)
  * list order     include/hopping_list.hpp:163-171, 226 (multimap keyed by the tag
                   "cx cy cz e0 e1 ": string order, equal tags in insertion order)
  * operators      src/tbmodel.cpp:38-440 (currents :92-126, spin currents :162-212,
                   spin/torque densities :129-159, 362-440, .OP files :331-354)
  * supercell      src/hopping_list.cpp:158-224 (every hopping copied to every cell
                   shift, cell indices wrapped, edges offset by the cell index * WBB)
  * CSR writer     src/hopping_list.cpp:227-285 (|v| / mean|v| > 1e-10 and
                   col >= row; Eigen setFromTriplets sums duplicates in triplet order and
                   sorts each row by column; values printed with 6 significant digits)

Complex arithmetic is written out as libstdc++'s std::complex<double> does it for finite
values (complex * complex = (ac - bd, ad + bc); complex * double and double * complex scale
both parts), so results are bitwise those of the reference built with g++.

Pinned by tests/test_w2s_oracle.py against the example operators LinQT ships
(examples/utilities/wannier2sparse/linear_chain/operators, 100 x 100 cells: identical
bytes), against the unit-test files of utilities/wannier2sparse/test that the sources in
the tree reproduce, and against the reference tool compiled from its own sources
(oracle/_ref/wannier2sparse, built by oracle/Makefile).

Only tests/ and bench.py's CPU-baseline leg import this module.
"""
import math
import os

import numpy as np

AVAIL_OPS = ["VX", "VY", "VZ", "VXSX", "VXSY", "VXSZ", "VYSX", "VYSY", "VYSZ", "VZSX", "VZSY", "VZSZ",
             "SX", "SY", "SZ", "TX", "TY", "TZ"]  # include/operator_utils.hpp:31-35


# --- std::complex<double> arithmetic (finite values) ---------------------------------------
def cmul(a, b):
    return (a[0] * b[0] - a[1] * b[1], a[0] * b[1] + a[1] * b[0])


def cscale(k, a):
    return (k * a[0], k * a[1])


def cadd(a, b):
    return (a[0] + b[0], a[1] + b[1])


def csub(a, b):
    return (a[0] - b[0], a[1] - b[1])


def cneg(a):
    return (-a[0], -a[1])


def cconj(a):
    return (a[0], -a[1])


def cexp(z):
    """glibc cexp for a finite argument with a zero real part: (cos y, sin y), and y itself
    as the imaginary part when y is zero (keeps its sign)."""
    assert z[0] == 0.0
    if z[1] == 0.0:
        return (1.0, z[1])
    return (math.cos(z[1]), math.sin(z[1]))


def cnorm(a):
    return a[0] * a[0] + a[1] * a[1]


I_UNIT = (0.0, 1.0)
MINUS_I = cneg(I_UNIT)


# --- model files -----------------------------------------------------------------------------
class Model:
    def __init__(self, num_wann, hoppings, lat, orbitals):
        self.num_wann = num_wann
        self.hoppings = hoppings  # [(cell(3), (e0, e1), value(re, im))], multimap order
        self.lat = lat            # 3 lattice vectors (rows)
        self.orbitals = orbitals  # [(label, (x, y, z))]


def tag(cell, edge):
    return "".join("%d " % x for x in tuple(cell) + tuple(edge))


def multimap_order(entries):
    """entries in insertion order -> iteration order of multimap<string, .> keyed by tag."""
    return [e for _, e in sorted(((tag(e[0], e[1]), i), e) for i, e in enumerate(entries))]


def _above(norm, avg):
    """norm / avg > 1e-10 with IEEE semantics (0 / 0 and x / NaN compare false)."""
    if avg != avg or avg == 0.0:
        return avg == 0.0 and norm > 0.0
    return norm / avg > 1e-10


def read_hr(path):
    """wannier_parser.cpp:45-84 and hopping_list.cpp:114-155.  Blank lines are skipped."""
    with open(path) as f:
        lines = f.read().split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    num_wann = int(lines[1].split()[0])
    nrpts = int(lines[2].split()[0])
    body = [ln for ln in lines[3 + 1 + nrpts // 15:] if ln.strip()]
    parsed = []
    for ln in body:
        t = ln.split()
        cell = (int(t[0]), int(t[1]), int(t[2]))
        edge = (int(t[3]) - 1, int(t[4]) - 1)
        parsed.append((cell, edge, (float(t[5]), float(t[6]))))
    avg = 0.0
    for _, _, v in parsed:
        avg += math.sqrt(cnorm(v))
    avg = avg / len(parsed) if parsed else math.nan
    kept = [p for p in parsed if _above(math.sqrt(cnorm(p[2])), avg)]
    return num_wann, multimap_order(kept)


def read_model(label):
    with open(label + ".xyz") as f:
        tok = f.read().split()
    n = int(tok[0])
    orbitals = [(tok[1 + 4 * i], tuple(float(x) for x in tok[2 + 4 * i:5 + 4 * i])) for i in range(n)]
    with open(label + ".uc") as f:
        u = [float(x) for x in f.read().split()[:9]]
    lat = [u[0:3], u[3:6], u[6:9]]
    num_wann, hops = read_hr(label + "_hr.dat")
    if len(orbitals) != num_wann:
        raise ValueError("%s.xyz lists %d orbitals, %s_hr.dat %d" % (label, len(orbitals), label, num_wann))
    return Model(num_wann, hops, lat, orbitals)


def volume(uc):  # tbmodel.cpp:492-498
    return abs((uc[0][1] * uc[1][2] - uc[1][1] * uc[0][2]) * uc[2][0]
               + (uc[0][2] * uc[1][0] - uc[0][0] * uc[1][2]) * uc[2][1]
               + (uc[0][0] * uc[1][1] - uc[0][1] * uc[1][0]) * uc[2][2])


# --- unit-cell operators -----------------------------------------------------------------------
def currents(m, d):
    """tbmodel.cpp:92-126: t -> t * (0, -dx_d), dx = pos[e1] - pos[e0] + R . lat."""
    av_length = math.pow(volume(m.lat), 1.0 / 3.0)
    out = []
    for cell, edge, v in m.hoppings:
        p1, p0 = m.orbitals[edge[1]][1], m.orbitals[edge[0]][1]
        diff = [p1[i] + (-p0[i]) for i in range(3)]
        for i in range(3):
            c = 0.0
            for j in range(3):
                c += cell[j] * m.lat[j][i]
            diff[i] += c
        s = (0.0, -diff[d]) if abs(diff[d]) / av_length > 1e-10 else (0.0, 0.0)
        out.append((cell, edge, cmul(v, s)))
    return out  # same tags, same order


def density(m, op):
    """tbmodel.cpp:64-90: every (i, j) of the unit cell, zeros included."""
    n = len(m.orbitals)
    return multimap_order([((0, 0, 0), (i, j), op[i][j]) for i in range(n) for j in range(n)])


def spinorial(m, elems):
    """tbmodel.cpp:362-380: a 2x2 spin matrix (row major) on every orbital's spin pair."""
    tot = len(m.orbitals)
    od = tot // 2
    op = [[(0.0, 0.0)] * tot for _ in range(tot)]
    for io in range(od):
        for si in range(2):
            for sj in range(2):
                op[si * od + io][sj * od + io] = elems[si * 2 + sj]
    return op


def spin_matrix_elems(theta, phi):  # tbmodel.cpp:144-148
    return [(math.cos(theta), 0.0), cscale(-math.sin(theta), cexp(cscale(phi, MINUS_I))),
            cscale(math.sin(theta), cexp(cscale(phi, I_UNIT))), (-math.cos(theta), 0.0)]


def torque_matrix(m, theta, phi):
    """tbmodel.cpp:393-440, the on-site exchange field of every orbital pair."""
    tot = len(m.orbitals)
    od = tot // 2
    H00 = [[(0.0, 0.0)] * tot for _ in range(tot)]
    for cell, edge, v in multimap_order([h for h in m.hoppings if h[0] == (0, 0, 0)]):
        H00[edge[0]][edge[1]] = cadd(H00[edge[0]][edge[1]], v)
    Tu = [[(0.0, 0.0)] * tot for _ in range(tot)]
    for io in range(od):
        i, j = io, od + io
        J00 = cscale(0.5, csub(H00[i][i], H00[j][j]))
        J01 = cscale(0.5, cadd(H00[i][j], cconj(H00[j][i])))
        J = [J01[0], -J01[1], J00[0]]
        st, ct, sp, cp = math.sin(theta), math.cos(theta), math.sin(phi), math.cos(phi)
        Tu[i][i] = (1.0 * st * (J[1] * cp - J[0] * sp), 0.0)
        Tu[j][j] = (-1.0 * st * (J[1] * cp - J[0] * sp), 0.0)
        a = cscale(J[0], MINUS_I)
        a = (a[0] - J[1], a[1])
        a = cscale(ct, a)
        b = cscale(cp, I_UNIT)
        b = (b[0] + sp, b[1])
        b = cscale(J[2] * st, b)
        Tu[i][j] = cadd(a, b)
        Tu[j][i] = cconj(Tu[i][j])
    return Tu


ANGLES = {"X": (0.5 * math.pi, 0.0 * math.pi), "Y": (0.5 * math.pi, 0.5 * math.pi), "Z": (0.0 * math.pi, 0.0 * math.pi)}


def spin_currents(m, d, theta, phi):
    """tbmodel.cpp:162-212."""
    ns = len(m.orbitals) // 2
    out = []

    def chg(edge, s):
        return (edge[0] % ns + s[0] * ns, edge[1] % ns + s[1] * ns)

    for cell, edge, v in currents(m, d):
        is0, is1 = edge[0] // ns, edge[1] // ns
        sz = 1.0 - 2.0 * is0
        if is0 == is1:
            s_uu = sz * math.cos(theta)
            s_ud = cscale(0.5 * math.sin(theta), cexp(cscale(phi, MINUS_I)))
            if s_uu * s_uu > 1e-5:
                out.append((cell, chg(edge, (is0, is0)), cmul(v, (s_uu, 0.0))))
            if cnorm(s_ud) > 1e-5:
                out.append((cell, chg(edge, (0, 1)), cmul(v, s_ud)))
                out.append((cell, chg(edge, (1, 0)), cmul(v, cconj(s_ud))))
        else:
            s_uu = cscale(0.5 * math.sin(theta), cexp(cscale(phi, cscale(sz, I_UNIT))))
            if cnorm(s_uu) > 1e-5:
                out.append((cell, chg(edge, (0, 0)), cmul(v, s_uu)))
                out.append((cell, chg(edge, (1, 1)), cmul(v, s_uu)))
    return multimap_order(out)


def operator_list(m, op, workdir="."):
    """tbmodel.cpp:310-359 (WannierOperator)."""
    if op == "HAM":
        return list(m.hoppings)
    dirs = {"X": 0, "Y": 1, "Z": 2}
    if op in AVAIL_OPS[0:3]:
        return currents(m, dirs[op[1]])
    if op in AVAIL_OPS[3:12]:
        return spin_currents(m, dirs[op[1]], *ANGLES[op[-1]])
    if op in AVAIL_OPS[12:15]:
        return density(m, spinorial(m, spin_matrix_elems(*ANGLES[op[-1]])))
    if op in AVAIL_OPS[15:18]:
        return density(m, torque_matrix(m, *ANGLES[op[-1]]))
    path = os.path.join(workdir, op + ".OP")
    if os.path.exists(path):
        with open(path) as f:
            tok = f.read().split()
        elems = [(float(tok[1 + 2 * k]), float(tok[2 + 2 * k])) for k in range(4)]
        return density(m, spinorial(m, elems))
    raise ValueError("unknown operator %r" % op)


# --- supercell and CSR -------------------------------------------------------------------------
def index_aliasing(c, b):  # include/hopping_list_util.hpp:12-16 (C++ % truncates)
    def m(x, n):
        return int(math.fmod(x + n, n))
    return (m(c[2], b[2]) * b[1] + m(c[1], b[1])) * b[0] + m(c[0], b[0])


def supercell_csr(m, op, dims, workdir="."):
    """hopping_list.cpp:158-285: returns (n, rowptr, col, val complex128) of the file."""
    uc = operator_list(m, op, workdir)
    wbb = m.num_wann
    entries = []  # (supercell tag, insertion index, e0, e1, value)
    k = 0
    for cell, edge, v in uc:
        for sz in range(dims[2]):
            for sy in range(dims[1]):
                for sx in range(dims[0]):
                    sh = (sx, sy, sz)
                    c = tuple(int(math.fmod(cell[i] + sh[i] + dims[i], dims[i])) for i in range(3))
                    e0 = edge[0] + index_aliasing(sh, dims) * wbb
                    e1 = edge[1] + index_aliasing(c, dims) * wbb
                    entries.append((tag((0, 0, 0), (e0, e1)), k, e0, e1, v))
                    k += 1
    entries.sort(key=lambda e: (e[0], e[1]))
    n = wbb * dims[0] * dims[1] * dims[2]
    avg = 0.0
    for e in entries:
        avg += math.sqrt(cnorm(e[4]))
    avg = avg / len(entries) if entries else math.nan
    rows = [dict() for _ in range(n)]
    for _, _, e0, e1, v in entries:
        if _above(math.sqrt(cnorm(v)), avg) and e1 >= e0:
            r = rows[e0]
            r[e1] = cadd(r[e1], v) if e1 in r else v
    rowptr = np.zeros(n + 1, dtype=np.int64)
    cols, vals = [], []
    for i in range(n):
        for c in sorted(rows[i]):
            cols.append(c)
            vals.append(complex(*rows[i][c]))
        rowptr[i + 1] = len(cols)
    return n, rowptr, np.array(cols, dtype=np.int64), np.array(vals, dtype=np.complex128)


def format_csr(n, rowptr, col, val):
    """The text hopping_list.cpp:260-282 writes (ostream defaults: %g with 6 digits)."""
    parts = ["%d %d\n" % (n, len(col))]
    parts.append("".join("%g %g " % (v.real, v.imag) for v in val) + "\n")
    parts.append("".join("%d " % c for c in col) + "\n")
    parts.append("".join("%d " % p for p in rowptr) + "\n")
    return "".join(parts)
