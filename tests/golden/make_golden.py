"""Regenerate the golden fixtures of tests/golden/ from the reference (run where the reference sources are present):

  python tests/golden/make_golden.py [<reference source tree>]

* ve_example_data.npy — the 99-particle x 31-column fixture of the reference's SPH kernel tests
  (sph/test/example_data.txt, read by sph/test/ve.cpp:69-77), as float64.
* ve_known_answers.json — every EXPECT_NEAR(value, expected, tolerance) of sph/test/ve.cpp, by test name.
* sedov12_ref.npz, noh14_ref.npz — outputs of the reference's own CPU step (oracle/_ref/libsphref.so, FP64 types)
  for the synthetic Sedov 12^3 and Noh 14^3 workloads: initial-sync keys/order/tree, the first force computation
  (neighbour counts and lists, every chain field, scalars) and the state after the first integration.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

COLUMNS = ("x", "y", "z", "vx", "vy", "vz", "h", "c", "c11", "c12", "c13", "c22", "c23", "c33", "p", "gradh", "rho0",
           "sumwhrho0", "sumwh", "dvxdx", "dvxdy", "dvxdz", "dvydx", "dvydy", "dvydz", "dvzdx", "dvzdy", "dvzdz",
           "alpha", "u", "divv")

FIELDS = ("xm", "kx", "gradh", "prho", "c", "c11", "c12", "c13", "c22", "c23", "c33", "divv", "curlv", "alpha", "ax",
          "ay", "az", "du", "h", "nc")
STATE = ("x", "y", "z", "h", "temp", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha")


def ve_fixture(ref_root):
    data = np.loadtxt(os.path.join(ref_root, "sph", "test", "example_data.txt"))
    assert data.shape == (99, len(COLUMNS)), data.shape
    np.save(os.path.join(HERE, "ve_example_data.npy"), data)
    src = open(os.path.join(ref_root, "sph", "test", "ve.cpp")).read()
    answers = {}
    for m in re.finditer(r"TEST_F\(SphKernelTests,\s*(\w+)\)\s*\{(.*?)\n\}", src, flags=re.S):
        name, body = m.group(1), m.group(2)
        blocks = re.split(r"\{ // test", body)
        entries = []
        for k, blk in enumerate(blocks):
            for e in re.finditer(r"EXPECT_NEAR\(([^,]+),\s*([^,]+),\s*([^)]+)\);", blk):
                entries.append({"block": k, "quantity": e.group(1).strip(), "expected": e.group(2).strip(),
                                "tol": e.group(3).strip()})
            for e in re.finditer(r"EXPECT_EQ\(([^,]+),\s*([^)]+)\);", blk):
                entries.append({"block": k, "quantity": e.group(1).strip(), "expected": e.group(2).strip(),
                                "tol": "0"})
        answers[name] = entries
    with open(os.path.join(HERE, "ve_known_answers.json"), "w") as f:
        json.dump(answers, f, indent=1)


def reference_run(ic, path):
    from oracle import refsim
    r = refsim.RefSim(ic)
    out = {"init_keys": r.keys(), "init_id": r.get("id").astype(np.uint64)}
    lv, cnt, lay = r.tree()
    out.update(init_leaves=lv, init_counts=cnt, init_layout=lay)
    r.compute_forces()
    out["keys"] = r.keys()
    out["id"] = r.get("id").astype(np.uint64)
    lv, cnt, lay = r.tree()
    out.update(leaves=lv, counts=cnt, layout=lay)
    for f in FIELDS:
        out["f_" + f] = r.get(f)
    nb = r.neighbors()
    nc = out["f_nc"].astype(np.int64)
    out["nbr"] = np.concatenate([nb[i, :min(nc[i] - 1, nb.shape[1])] for i in range(r.n)]).astype(np.uint32)
    sc = r.scalars()
    out["scalars_forces"] = np.array([sc[k] for k in refsim.SCALAR_NAMES])
    r.integrate()
    for f in STATE:
        out["s_" + f] = r.get(f)
    sc = r.scalars()
    out["scalars_integrate"] = np.array([sc[k] for k in refsim.SCALAR_NAMES])
    np.savez_compressed(path, **out)


def reference_root() -> str:
    """$SPHEXA_REFERENCE, else the directory "reference" beside this repository."""
    return os.environ.get("SPHEXA_REFERENCE", os.path.abspath(os.path.join(ROOT, "..", "reference")))


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else reference_root()
    ve_fixture(ref_root)
    from sphexa_b200 import ic as icm
    reference_run(icm.sedov(12), os.path.join(HERE, "sedov12_ref.npz"))
    reference_run(icm.noh(14), os.path.join(HERE, "noh14_ref.npz"))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
