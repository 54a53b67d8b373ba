"""The oracle reproduces the reference's own outputs (tests/golden, made by
running the reference kernels through oracle/_ref) bit for bit."""
import glob
import os

import numpy
import pytest

import oracle as O
from helpers import VEC3, bits_equal, diff_report

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# the Navier-Stokes fixture has no C restatement to check: it is compared with
# the reference's host build (test_oracle_reference.py) and the device solver
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "*.bin"))
               if not os.path.basename(p).startswith("ns_"))


@pytest.fixture(scope="module", autouse=True)
def built():
    O.build(ref=False)


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_golden(case):
    gold = numpy.load(os.path.join(HERE, case + ".npz"))
    steps = sorted({int(k.split("@")[1]) for k in gold.files})
    fields = sorted({k.split("@")[0] for k in gold.files})
    orc = O.Oracle(os.path.join(HERE, case + ".bin"), fluid=case.startswith("darcy"))
    done = 0
    for s in steps:
        assert orc.step(s - done) == 0, orc.error()
        done = s
        for f in fields:
            a = orc.get(f)
            if f in VEC3:
                a = a[:, :3]
            b = gold[f"{f}@{s}"]
            if f == "darcy_nijac_last":
                a = a.astype(numpy.int64)
                b = b.astype(numpy.int64)
            assert bits_equal(a, b), f"step {s}: " + diff_report(f, a, b)
    orc.close()


def test_golden_cases_have_contacts():
    for case in CASES:
        gold = numpy.load(os.path.join(HERE, case + ".npz"))
        if case in ("dense_model1", "darcy_consolidation"):
            continue
        n = gold["x@1"].shape[0]
        assert (gold["contacts@20"] != n).sum() > 50, case
