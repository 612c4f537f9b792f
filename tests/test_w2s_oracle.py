"""The operator-builder oracle (oracle/w2s_oracle.py, LinQT's utilities/wannier2sparse restated)
pinned against the reference's own outputs, plus the host side of the library's model loader.

Pins:
  * the example operators LinQT ships, examples/utilities/wannier2sparse/linear_chain/
    operators/linear_chain.{HAM,VX}.CSR (a 100 x 100 x 1 supercell of the 2-orbital chain;
    kept in tests/golden/linear_chain.npz): identical arrays and identical text;
  * the unit-test files of utilities/wannier2sparse/test that the tree's sources reproduce
    (tests/golden/w2s_ref.json "shipped"), byte for byte;
  * every file the reference tool compiled from its own sources writes for 19 (model,
    supercell) cases x all operators (w2s_ref.json "ref", made by make_w2s_golden.py);
  * live, when oracle/_ref/wannier2sparse is built: random models against that tool.
"""
import json
import os
import random
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import w2s_oracle as w  # noqa: E402

GOLD = os.path.join(HERE, "golden")
W2S = os.path.join(GOLD, "w2s")
LABELS = {"linear_chain_example": "linear_chain", "linear_chain_multi": "linear_chain",
          "linear_chain_local": "linear_chain", "graphene_M_x": "graphene+rashba+M_x",
          "graphene_M_y": "graphene+rashba+M_y", "graphene_M_z": "graphene+rashba+M_z",
          "graphene_MoTe2": "graphene+MoTe2-SC5x7"}
REF_TOOL = os.path.join(ROOT, "oracle", "_ref", "wannier2sparse")


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(GOLD, "w2s_ref.json")) as f:
        return json.load(f)


def model(case):
    return w.read_model(os.path.join(W2S, case, LABELS[case]))


def test_example_operators_shipped_with_linqt():
    g = np.load(os.path.join(GOLD, "linear_chain.npz"))
    m = model("linear_chain_example")
    for op in ("HAM", "VX"):
        n, rp, cl, vl = w.supercell_csr(m, op, (100, 100, 1))
        assert n == 20000
        assert np.array_equal(rp, g[op + "_rowptr"]) and np.array_equal(cl, g[op + "_col"])
        want = g[op + "_val"][0::2] + 1j * g[op + "_val"][1::2]
        assert np.array_equal(vl, want)


def test_shipped_unit_test_files(golden):
    assert len(golden["shipped"]) >= 40
    for path, txt in golden["shipped"].items():
        case = path.split("/")[0]
        op = os.path.basename(path).split(".")[1]
        assert w.format_csr(*w.supercell_csr(model(case), op, (1, 1, 1))) == txt, path


def test_files_from_other_versions_of_the_tool_are_listed(golden):
    """The files the tree's sources do not reproduce: SX/SY carry the opposite sign of
    sin(theta) in every set, linear_chain_local's velocities lack the explicit zeros Eigen
    keeps, and linear_chain_multi's top-level velocities come from yet another version."""
    other = golden["shipped_other_version"]
    ops = sorted({os.path.basename(p).split(".")[1] for p in other})
    assert ops == ["SX", "SY", "VX", "VXSX", "VXSY", "VXSZ"]
    sx = other["linear_chain_multi/old_case/linear_chain.SX.CSR"].split("\n")[1].split()
    n, rp, cl, vl = w.supercell_csr(model("linear_chain_multi"), "SX", (1, 1, 1))
    assert float(sx[0]) == -vl[0].real == 1.0


def test_reference_tool_outputs(golden):
    count = 0
    for key, files in golden["ref"].items():
        case, cell = key.split("/")
        dims = tuple(int(x) for x in cell.split("x"))
        m = model(case)
        for op, txt in files.items():
            got = w.format_csr(*w.supercell_csr(m, op, dims, workdir=os.path.join(W2S, case)))
            assert got == txt, (key, op)
            count += 1
    assert count > 300


def random_model(d, seed):
    """A spinful model with hoppings up to 3 cells away (3D when seed is odd), duplicates
    and zeros included, on a skewed cell."""
    rnd = random.Random(seed)
    W = rnd.choice([2, 4, 6])
    rng = rnd.choice([1, 2, 3])
    three_d = seed % 2 == 1
    lines = []
    for _ in range(rnd.randint(5, 60)):
        R = (rnd.randint(-rng, rng), rnd.randint(-rng, rng), rnd.randint(-rng, rng) if three_d else 0)
        lines.append("%d %d %d %d %d %.6f %.6f" % (R + (rnd.randint(1, W), rnd.randint(1, W), rnd.uniform(-2, 2),
                                                        rnd.choice([0.0, rnd.uniform(-1, 1)]))))
    lines.append(lines[0])
    with open(os.path.join(d, "m_hr.dat"), "w") as f:
        f.write("random model\n%d\n1\n    1\n%s\n" % (W, "\n".join(lines)))
    with open(os.path.join(d, "m.uc"), "w") as f:
        f.write("1.0 0.1 0.0\n-0.3 0.9 0.0\n0.0 0.2 1.5\n")
    with open(os.path.join(d, "m.xyz"), "w") as f:
        f.write("%d\n" % W)
        for i in range(W):
            f.write("o%d_s%s_ %.3f %.3f %.3f\n" % (i, "+" if i < W // 2 else "-", rnd.random(), rnd.random(),
                                                  rnd.random()))
    dims = (rnd.randint(1, 6), rnd.randint(1, 4), rnd.randint(1, 3) if three_d else 1)
    return os.path.join(d, "m"), dims


@pytest.mark.skipif(not os.path.exists(REF_TOOL), reason="oracle/_ref/wannier2sparse not built")
@pytest.mark.parametrize("seed", range(6))
def test_random_models_against_reference_tool(tmp_path, seed):
    label, dims = random_model(str(tmp_path), seed)
    ops = ["VX", "VZ", "VXSY", "VYSZ", "SX", "TY"]
    subprocess.run([REF_TOOL, "m"] + [str(x) for x in dims] + ops, cwd=tmp_path, check=True,
                   stdout=subprocess.DEVNULL)
    m = w.read_model(label)
    for op in ["HAM"] + ops:
        want = open(os.path.join(tmp_path, "m.%s.CSR" % op)).read()
        assert w.format_csr(*w.supercell_csr(m, op, dims)) == want, op


# --- the library's model loader (host code, no GPU needed) ------------------------------------
def test_library_reads_models_like_the_oracle():
    import linqt_b200 as lq
    for case in LABELS:
        m = lq.TBModel.load(os.path.join(W2S, case, LABELS[case]))
        o = model(case)
        assert m.info() == (o.num_wann, len(o.hoppings))


def test_library_model_errors(tmp_path):
    import linqt_b200 as lq
    with pytest.raises(lq.LinqtError) as e:
        lq.TBModel.load(str(tmp_path / "missing"))
    assert e.value.code == -1
    src = os.path.join(W2S, "linear_chain_local", "linear_chain")
    for ext in (".uc", ".xyz", "_hr.dat"):
        with open(src + ext) as f, open(str(tmp_path / ("m" + ext)), "w") as g:
            g.write(f.read())
    with open(str(tmp_path / "m.stdis"), "w") as f:
        f.write("uniform\n0 0 0\n1 1\n-1 0 1 0\n0.5\n")
    with pytest.raises(lq.LinqtError) as e:
        lq.TBModel.load(str(tmp_path / "m"))
    assert e.value.code == -4 and "stdis" in str(e.value)
    os.remove(str(tmp_path / "m.stdis"))
    with open(str(tmp_path / "m_hr.dat"), "a") as f:
        f.write("0 0 0 1 x 1.0 0.0\n")
    with pytest.raises(lq.LinqtError) as e:
        lq.TBModel.load(str(tmp_path / "m"))
    assert e.value.code == -1 and "malformed" in str(e.value)
