"""The supercell operators assembled on the GPU (linqt_supercell_*) against the operator-builder
oracle (oracle/w2s_oracle.py) and the reference tool's own files.

  * every (model, supercell, operator) of tests/golden/w2s_ref.json: the arrays equal the
    oracle's bit for bit and the written file equals the reference tool's byte for byte;
  * random models (duplicates, hoppings longer than the supercell, 3D): bit for bit;
  * large supercells, where the oracle is too slow: the same matrix built independently by
    scipy from the replicated hopping list (no entry has two contributions there, so the
    sums are exact either way);
  * the drop-in: linqt_b200/w2s/_bin/wannier2sparse writes the reference tool's files;
  * the device operator: the 2D moments of the example linear chain built from its Wannier
    files on the GPU equal the table LinQT ships (NonLEqOpVX-VXlinear_chainKPM_M100x100).
"""
import json
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import linqt_b200 as lq

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)
import w2s_oracle as w  # noqa: E402
from test_w2s_oracle import LABELS, W2S, random_model  # noqa: E402

CLI = os.path.join(ROOT, "linqt_b200", "w2s", "_bin", "wannier2sparse")


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "w2s_ref.json")) as f:
        return json.load(f)


def same_arrays(got, want):
    n, rp, cl, vl = got
    n2, rp2, cl2, vl2 = want
    assert n == n2
    assert np.array_equal(rp, rp2) and np.array_equal(cl, cl2)
    # bitwise, signed zeros included
    assert np.array_equal(vl.view(np.uint64), np.asarray(vl2, dtype=np.complex128).view(np.uint64))


def test_reference_cases_bitwise(golden, tmp_path, monkeypatch):
    count = 0
    for key, files in golden["ref"].items():
        case, cell = key.split("/")
        dims = tuple(int(x) for x in cell.split("x"))
        monkeypatch.chdir(os.path.join(W2S, case))  # NAME.OP files are looked up here
        label = os.path.join(W2S, case, LABELS[case])
        m, o = lq.TBModel.load(label), w.read_model(label)
        for op, txt in files.items():
            same_arrays(m.supercell_csr(op, dims), w.supercell_csr(o, op, dims))
            out = str(tmp_path / ("%s.%s.CSR" % (case, op)))
            m.write_csr(op, dims, out)
            assert open(out).read() == txt, (key, op)
            count += 1
    assert count > 300


@pytest.mark.parametrize("seed", range(10))
def test_random_models_bitwise(tmp_path, seed):
    label, dims = random_model(str(tmp_path), seed)
    m, o = lq.TBModel.load(label), w.read_model(label)
    for op in ["HAM", "VX", "VY", "VZ", "VXSX", "VYSY", "VZSZ", "SX", "SY", "SZ", "TX", "TZ"]:
        same_arrays(m.supercell_csr(op, dims), w.supercell_csr(o, op, dims))
        assert m.csr_size(op, dims) == (dims[0] * dims[1] * dims[2] * o.num_wann, len(w.supercell_csr(o, op, dims)[2]))


def scipy_upper(o, op, dims):
    """The supercell matrix from the replicated unit-cell list by scipy (duplicates summed)."""
    import scipy.sparse as sp
    uc = w.operator_list(o, op)
    wbb = o.num_wann
    D = np.array(dims)
    cells = np.stack(np.meshgrid(np.arange(D[0]), np.arange(D[1]), np.arange(D[2]), indexing="ij"), -1).reshape(-1, 3)
    idx = lambda c: (c[:, 2] * D[1] + c[:, 1]) * D[0] + c[:, 0]  # noqa: E731
    norms = np.array([np.hypot(*v) for _, _, v in uc])
    mean = norms.mean() if len(norms) else 0.0
    keep = norms > 1e-10 * mean if mean > 0 else np.zeros(len(norms), dtype=bool)
    n = wbb * len(cells)
    rows, cols, vals = [np.zeros(0, np.int64)], [np.zeros(0, np.int64)], [np.zeros(0, np.complex128)]
    for (cell, (e0, e1), v), k in zip(uc, keep):
        if not k:
            continue
        tgt = np.mod(cells + np.array(cell), D)
        rows.append(idx(cells) * wbb + e0)
        cols.append(idx(tgt) * wbb + e1)
        vals.append(np.full(len(cells), complex(*v)))
    r, c, v = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    up = c >= r
    A = sp.csr_matrix((v[up], (r[up], c[up])), shape=(n, n))
    A.sort_indices()
    return n, A.indptr, A.indices, A.data


@pytest.mark.parametrize("case,dims", [("graphene_MoTe2", (300, 200, 1)), ("graphene_M_x", (1000, 700, 1)),
                                       ("linear_chain_multi", (4000, 3, 5))])
def test_large_supercells_against_scipy(case, dims):
    label = os.path.join(W2S, case, LABELS[case])
    m, o = lq.TBModel.load(label), w.read_model(label)
    for op in ["HAM", "VX", "VYSX"]:
        got = m.supercell_csr(op, dims)
        n, rp, cl, vl = scipy_upper(o, op, dims)
        assert got[0] == n and np.array_equal(got[1], rp) and np.array_equal(got[2], cl)
        assert np.array_equal(got[3], vl), op


def test_device_buffers_and_errors():
    import torch
    label = os.path.join(W2S, "graphene_M_z", LABELS["graphene_M_z"])
    m = lq.TBModel.load(label)
    dims = (37, 23, 1)
    n, rp, cl, vl = m.supercell_csr("VXSY", dims)
    s = lq.Session(0)
    r_d = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    c_d = torch.zeros(len(cl), dtype=torch.int32, device="cuda")
    v_d = torch.zeros(2 * len(cl), dtype=torch.float64, device="cuda")
    assert m.supercell_csr_dev("VXSY", dims, r_d, c_d, v_d, len(cl), session=s) == (n, len(cl))
    s.synchronize()
    assert np.array_equal(r_d.cpu().numpy(), rp) and np.array_equal(c_d.cpu().numpy(), cl)
    assert np.array_equal(v_d.cpu().numpy().view(np.complex128), vl)
    with pytest.raises(lq.LinqtError) as e:
        m.supercell_csr_dev("VXSY", dims, r_d, c_d, v_d, len(cl) - 1, session=s)
    assert e.value.code == -1 and "capacity" in str(e.value)
    for op, d in (("VQ", dims), ("HAM", (0, 1, 1)), ("HAM", (70000, 70000, 1))):
        with pytest.raises(lq.LinqtError) as e:
            m.supercell_csr(op, d)
        assert e.value.code == -1


@pytest.mark.skipif(not os.path.exists(CLI), reason="wannier2sparse command line not built")
def test_command_line_writes_the_reference_files(golden, tmp_path):
    for key in ("graphene_M_x/2x3x1", "linear_chain_multi/5x1x1", "graphene_MoTe2/5x7x1"):
        case, cell = key.split("/")
        d = tmp_path / key.replace("/", "_")
        shutil.copytree(os.path.join(W2S, case), str(d))
        ops = [op for op in golden["ref"][key] if op != "HAM"]
        ops = ["all"] + [op for op in ops if op not in w.AVAIL_OPS]
        p = subprocess.run([CLI, LABELS[case]] + cell.split("x") + ops, cwd=str(d), capture_output=True, text=True)
        assert p.returncode == 0, p.stderr
        for op, txt in golden["ref"][key].items():
            assert open(str(d / ("%s.%s.CSR" % (LABELS[case], op)))).read() == txt, (key, op)


def test_device_operator_reproduces_shipped_moments():
    """Wannier files -> GPU supercell operators -> GPU 2D moments = the published table."""
    g = np.load(os.path.join(HERE, "golden", "linear_chain.npz"))
    m = lq.TBModel.load(os.path.join(W2S, "linear_chain_example", "linear_chain"))
    H = m.operator("HAM", (100, 100, 1))
    V = m.operator("VX", (100, 100, 1))
    # the same operators as the ones read from the shipped files
    for op, X in (("HAM", H), ("VX", V)):
        F = lq.Operator.from_csr(20000, g[op + "_rowptr"], g[op + "_col"],
                                 g[op + "_val"][0::2] + 1j * g[op + "_val"][1::2])
        assert F.info() == X.info()
    assert H.info() == (20000, 40000)
    bw, bc = 10.0, 0.0  # BOUNDS -5 5
    H.rescale_to_chebyshev(bw, bc)
    st = np.zeros((1, 20000), dtype=np.complex128)
    st[0, 10000] = 1.0  # the reference's default state: a delta at N/2
    mu = lq.moments2d(H, V, V, st, 100)
    want = g["mu100"][..., 0] + 1j * g["mu100"][..., 1]
    assert np.abs(mu - want).max() <= 1e-13 * np.abs(want).max()
