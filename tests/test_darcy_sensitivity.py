"""How far last-bit differences of the math library move the Darcy solve.

The engine computes the reference's pow calls (sphere volumes, Kozeny-Carman
permeabilities) with CUDA's pow, the oracle with glibc's; they may differ in
the last bit.  The probe variant of the oracle (liboracle_powprod.so, pow
replaced by products) makes differences of that size on purpose.  On the
40 x 40 x 80 benchmark grid the pressure then moves by ~1e-9 of its maximum
after one solve of ~870 iterations: the stop rule (a relative change of 1e-8
per iteration) ends the Jacobi loop far from its fixed point, where small
changes of the coefficients show.  The GPU parity tests bound their errors by
this probe (tests/test_gpu_darcy.py)."""
import numpy

from sphere_b200 import binfile

import oracle as O
from test_gpu_darcy import PAIRS, grid_case


def errors(a, b):
    out = {}
    for name, _ in PAIRS:
        x, y = numpy.asarray(a.get(name), dtype=float), numpy.asarray(b.get(name), dtype=float)
        out[name] = float(numpy.abs(x - y).max()) / max(float(numpy.abs(y).max()), 1e-300)
    return out


def test_last_bit_changes_of_pow_move_the_pressure_by_about_1e9(tmp_path):
    O.build(ref=False)
    d = grid_case(61)
    path = str(tmp_path / "grid.bin")
    binfile.write_bin(d, path)
    orc = O.Oracle(path, fluid=True)
    probe = O.Oracle(path, fluid=True, lib_path=O.POWPROD_SO)
    worst = {}
    for _ in range(2):
        assert orc.step(1) == 0 and probe.step(1) == 0
        assert int(orc.get("darcy_nijac_last")[0]) == int(probe.get("darcy_nijac_last")[0])
        for f, e in errors(probe, orc).items():
            worst[f] = max(worst.get(f, 0.0), e)
    # the coefficients differ in the last bits only ...
    assert worst["darcy_phi"] < 1e-14 and worst["darcy_k"] < 1e-13
    # ... and the solve carries that to ~1e-9 of the pressure
    assert 1e-11 < worst["darcy_p"] < 1e-8
