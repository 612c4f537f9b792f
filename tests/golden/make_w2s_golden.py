"""Regenerate the operator-builder fixtures (tests/golden/w2s/ and tests/golden/w2s_ref.json).

    python tests/golden/make_w2s_golden.py [REFERENCE_CHECKOUT]

Inputs: the Wannier models LinQT ships (utilities/wannier2sparse/test/{linear_chain_multi,
linear_chain_local,graphene_sot}, examples/utilities/wannier2sparse/{linear_chain,
graphene/unit_cell}) are copied to tests/golden/w2s/<case>/, plus one spinorial operator
file (MYOP.OP) written here.

Outputs, in w2s_ref.json:
  "ref"     the CSR text files written by the reference tool compiled from its own sources
            (oracle/_ref/wannier2sparse, `make -C oracle`), per case, supercell and operator;
  "shipped" the unit-test CSR files of utilities/wannier2sparse/test that the sources in the
            tree reproduce byte for byte, and "shipped_other_version" the ones they do not
            (files written by other versions of the tool: spin densities SX/SY with the
            opposite sign of sin(theta); linear_chain_local's velocities without the
            explicit zeros Eigen keeps; linear_chain_multi's top-level velocities).
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LINQT_REF")
if not REF:
    sys.exit("usage: python tests/golden/make_w2s_golden.py REFERENCE_CHECKOUT  (or set LINQT_REF)")
TOOL = os.path.join(ROOT, "oracle", "_ref", "wannier2sparse")
OUT = os.path.join(HERE, "w2s")

ALL = ["VX", "VY", "VZ", "VXSX", "VXSY", "VXSZ", "VYSX", "VYSY", "VYSZ", "VZSX", "VZSY", "VZSZ",
       "SX", "SY", "SZ", "TX", "TY", "TZ"]
T = os.path.join(REF, "utilities", "wannier2sparse", "test")
E = os.path.join(REF, "examples", "utilities", "wannier2sparse")
CASES = {
    # case: (source dir, label, [supercells], operators)
    "linear_chain_example": (os.path.join(E, "linear_chain"), "linear_chain", [(20, 1, 1), (7, 3, 2)], ["VX", "VY"]),
    "linear_chain_multi": (os.path.join(T, "linear_chain_multi"), "linear_chain", [(1, 1, 1), (3, 1, 1), (5, 1, 1),
                                                                                    (9, 2, 1), (3, 2, 2)], ALL),
    "linear_chain_local": (os.path.join(T, "linear_chain_local"), "linear_chain", [(1, 1, 1), (2, 1, 1), (4, 1, 3)],
                           ALL),
    "graphene_M_x": (os.path.join(T, "graphene_sot"), "graphene+rashba+M_x", [(1, 1, 1), (2, 3, 1), (4, 4, 1)],
                     ALL + ["MYOP"]),
    "graphene_M_y": (os.path.join(T, "graphene_sot"), "graphene+rashba+M_y", [(3, 2, 1)], ALL),
    "graphene_M_z": (os.path.join(T, "graphene_sot"), "graphene+rashba+M_z", [(2, 2, 1), (5, 1, 1)], ALL),
    "graphene_MoTe2": (os.path.join(E, "graphene", "unit_cell"), "graphene+MoTe2-SC5x7", [(1, 1, 1), (3, 2, 1),
                                                                                         (5, 7, 1)], ALL),
}
MYOP = "spinorial\n0.25 0.5\n-1.5 0.125\n2.0 -0.75\n0.5 0.0\n"


def main():
    if not os.path.exists(TOOL):
        sys.exit("build the reference tool first: make -C oracle")
    golden = {"ref": {}, "shipped": {}, "shipped_other_version": {}}
    for case, (src, label, cells, ops) in CASES.items():
        dst = os.path.join(OUT, case)
        os.makedirs(dst, exist_ok=True)
        for ext in (".uc", ".xyz", "_hr.dat"):
            shutil.copy(os.path.join(src, label + ext), os.path.join(dst, label + ext))
        if "MYOP" in ops:
            with open(os.path.join(dst, "MYOP.OP"), "w") as f:
                f.write(MYOP)
        for cell in cells:
            with tempfile.TemporaryDirectory() as tmp:
                for fn in os.listdir(dst):
                    shutil.copy(os.path.join(dst, fn), tmp)
                subprocess.run([TOOL, label] + [str(c) for c in cell] + ops, cwd=tmp, check=True,
                               stdout=subprocess.DEVNULL)
                key = "%s/%dx%dx%d" % (case, *cell)
                golden["ref"][key] = {op: open(os.path.join(tmp, "%s.%s.CSR" % (label, op))).read()
                                      for op in ["HAM"] + ops}
    for case, sub in (("linear_chain_multi", "old_case"), ("linear_chain_multi", ""), ("linear_chain_local", ""),
                      ("linear_chain_local", "old")):
        d = os.path.join(T, case, sub)
        made = golden["ref"]["%s/1x1x1" % case]
        for fn in sorted(os.listdir(d)):
            if fn.endswith(".CSR"):
                op = fn.split(".")[1]
                txt = open(os.path.join(d, fn)).read()
                bucket = "shipped" if made[op] == txt else "shipped_other_version"
                golden[bucket][os.path.join(case, sub, fn)] = txt
    with open(os.path.join(HERE, "w2s_ref.json"), "w") as f:
        json.dump(golden, f, indent=0, sort_keys=True)
    print({k: len(v) for k, v in golden.items()})


if __name__ == "__main__":
    main()
