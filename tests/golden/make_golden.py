"""Regenerate tests/golden/linear_chain.npz from the reference's shipped example.

The reference ships one end-to-end example with results
(examples/utilities/wannier2sparse/linear_chain/ in adamecius/linqt):

  operators/linear_chain.{HAM,VX}.CSR              upper-triangle CSR operators, N = 20000
  NonLEqOpVX-VXlinear_chainKPM_M{100x100,300x300}.chebmom2D
                                                   2D Kubo-Bastin moment tables written by
                                                   inline_compute-kpm-nonEqOp (default state
                                                   = unit vector at N/2, one state)
  KuboBastin_kernel_...M{100x100,300x300}JACKSON.dat
                                                   sigma(E) written by kuboBastinFromChebmom

This script parses those text files (the formats of src/sparse_matrix.cpp:3-50,
src/chebyshev_moments2D.cpp:16-68) and stores them as one compressed numpy
archive so that the tests need no access to the reference checkout.

Usage:  python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_csr(path):
    tok = open(path).read().split()
    dim, nnz = int(tok[0]), int(tok[1])
    vals = np.array(tok[2:2 + 2 * nnz], dtype=np.float64)
    cols = np.array(tok[2 + 2 * nnz:2 + 3 * nnz], dtype=np.int32)
    rows = np.array(tok[2 + 3 * nnz:2 + 3 * nnz + dim + 1], dtype=np.int32)
    return rows, cols, vals


def read_chebmom2d(path):
    tok = open(path).read().split()
    n, bw, bc = int(tok[0]), float(tok[1]), float(tok[2])
    m0, m1 = int(tok[3]), int(tok[4])
    v = np.array(tok[5:5 + 2 * m0 * m1], dtype=np.float64)
    return np.array([n, bw, bc]), v.reshape(m0, m1, 2)


def read_dat(path):
    return np.loadtxt(path)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LINQT_REF")
    if not ref:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT  (or set LINQT_REF)")
    d = os.path.join(ref, "examples/utilities/wannier2sparse/linear_chain")
    out = {}
    for op in ("HAM", "VX"):
        r, c, v = read_csr(os.path.join(d, "operators", "linear_chain.%s.CSR" % op))
        out[op + "_rowptr"], out[op + "_col"], out[op + "_val"] = r, c, v
    for m in (100, 300):
        hdr, mu = read_chebmom2d(os.path.join(d, "NonLEqOpVX-VXlinear_chainKPM_M%dx%d.chebmom2D" % (m, m)))
        out["mu%d_header" % m], out["mu%d" % m] = hdr, mu
        dat = read_dat(os.path.join(d, "KuboBastin_kernel_NonLEqOpVX-VXlinear_chainKPM_M%dx%dJACKSON.dat" % (m, m)))
        out["bastin%d" % m] = dat
    np.savez_compressed(os.path.join(HERE, "linear_chain.npz"), **out)


if __name__ == "__main__":
    main()
