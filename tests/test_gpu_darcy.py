"""The engine's Darcy solver (cfd_solver 1) against the CPU oracle.

The oracle is pinned bit-exact against the reference's own Darcy kernels
(tests/test_oracle_reference.py).  The device solver keeps the reference's
operation order, but `pow` (sphere volumes, Kozeny-Carman permeabilities)
comes from CUDA's math library on the device and glibc's on the host, which
may differ in the last bit; the coupled DEM state then drifts by rounding.
So the pressure, porosity, permeability and velocity fields and the DEM
state are compared to a relative tolerance of 1e-9 of each field's largest
magnitude, while the Jacobi iteration counts must match exactly.
"""
import os

import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-9
PAIRS = (("darcy_p", "darcy_p"), ("darcy_phi", "darcy_phi"), ("darcy_dphi", "darcy_dphi"),
         ("darcy_k", "darcy_k"), ("darcy_v", "darcy_v"), ("darcy_f_p", "darcy_f_p"),
         ("x", "x"), ("vel", "vel"), ("force", "force"))


def darcy_case(seed, periodic=1, bottom_no_flow=True, top_wall=True, ndem=1, n=300,
               maxiter=2000, flux_bottom=None, p_mod=None):
    d = configs.settling_lattice(n=n, seed=seed, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    d.periodic = periodic
    if top_wall:
        configs.add_top_wall(d, 10e3)
        d.w_x[0] -= 0.002
    configs.init_fluid_darcy(d, mu=1.797e-6, k_c=3.5e-13, tolerance=1e-8, maxiter=maxiter,
                             bottom_no_flow=bottom_no_flow, ndem=ndem)
    if flux_bottom is not None:
        d.bc_bot = 4
        d.bc_bot_flux = flux_bottom
    if p_mod is not None:
        d.p_mod_A, d.p_mod_f = p_mod
    return d


def compare(eng, orc):
    bad = {}
    for a_name, b_name in PAIRS:
        a = numpy.asarray(eng.get(a_name), dtype=float)
        b = numpy.asarray(orc.get(b_name), dtype=float)
        if a_name in ("x", "vel", "force", "darcy_f_p"):
            a, b = a.reshape(-1, 4)[:, :3], b.reshape(-1, 4)[:, :3]
        a, b = a.ravel(), b.ravel()
        if a.shape != b.shape:
            bad[a_name] = f"shape {a.shape} vs {b.shape}"
            continue
        scale = max(float(numpy.abs(b).max()), 1e-300)
        err = float(numpy.abs(a - b).max()) / scale
        if not err <= RTOL:
            bad[a_name] = f"relative max error {err:.3e}"
    it_e = int(eng.get("darcy_iters")[0])
    it_o = int(orc.get("darcy_nijac_last")[0])
    if it_e != it_o:
        bad["iterations"] = f"{it_e} vs {it_o}"
    return bad


CASES = {
    "neumann_bottom": dict(),
    "dirichlet_bottom": dict(bottom_no_flow=False),
    "periodic_x": dict(periodic=2),
    "no_wall": dict(top_wall=False),
    "ndem2": dict(ndem=2),
    "flux_bottom": dict(flux_bottom=2e-6),
    "top_modulation": dict(p_mod=(2e3, 5.0)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_darcy_parity(tmp_path, name):
    from sphere_b200.engine import Engine
    d = darcy_case(51, **CASES[name])
    path = str(tmp_path / "darcy.bin")
    binfile.write_bin(d, path)
    orc = O.Oracle(path, fluid=True)
    eng = Engine(path, fluid=True, precision="faithful")
    for k in range(6):
        assert eng.step(1) == 0
        assert orc.step(1) == 0, orc.error()
        bad = compare(eng, orc)
        assert not bad, f"after step {k + 1}: {bad}"
    assert int(orc.get("darcy_nijac_last")[0]) > 10
    assert int(eng.get("darcy_iters_total")[0]) == int(orc.get("darcy_nijac_total")[0])
    exact = int(eng.get("darcy_iters_exact")[0])
    assert 0 <= exact <= int(eng.get("darcy_iters")[0])
    eng.close()


def test_darcy_golden_fixture():
    """The committed consolidation fixture (outputs of the reference's own
    Darcy kernels built for the host, steps 1-3) reproduced by the device
    solver."""
    from sphere_b200.engine import Engine
    here = os.path.join(os.path.dirname(__file__), "golden")
    gold = numpy.load(os.path.join(here, "darcy_consolidation.npz"))
    eng = Engine(os.path.join(here, "darcy_consolidation.bin"), fluid=True, precision="faithful")
    for step in (1, 2, 3):
        assert eng.step(1) == 0
        for key in gold.files:
            name, at = key.split("@")
            if int(at) != step:
                continue
            b = numpy.asarray(gold[key], dtype=float)
            if name == "darcy_nijac_last":
                assert int(eng.get("darcy_iters")[0]) == int(b.ravel()[0]), step
                continue
            a = numpy.asarray(eng.get(name), dtype=float)
            if name in ("x", "vel", "force", "darcy_f_p"):
                a = a.reshape(-1, 4)[:, :3]
                b = b.reshape(len(a), -1)[:, :3]
            a, b = a.ravel(), b.ravel()
            scale = max(float(numpy.abs(b).max()), 1e-300)
            assert float(numpy.abs(a - b).max()) <= RTOL * scale, (key, step)
    eng.close()


def test_darcy_noconv_warning(tmp_path):
    """A solve that reaches maxiter returns the 'did not converge' warning
    (the reference prints an error and continues) and still matches the
    oracle."""
    from sphere_b200.engine import Engine
    d = darcy_case(52, maxiter=7)
    path = str(tmp_path / "noconv.bin")
    binfile.write_bin(d, path)
    orc = O.Oracle(path, fluid=True)
    eng = Engine(path, fluid=True)
    assert eng.step(1) == 0           # iteration 0 is checked and converges at once
    assert orc.step(1) == 0
    rc = eng.step(1)
    assert orc.step(1) == 0
    assert rc == 1
    assert int(eng.get("darcy_iters")[0]) == 6
    bad = compare(eng, orc)
    assert not bad, bad
    eng.close()


def test_darcy_run_files(tmp_path):
    """run() writes output files, the status file and the conv log."""
    from sphere_b200.engine import Engine
    d = darcy_case(53)
    dt = float(d.time_dt)
    d.time_total = 12 * dt
    d.time_file_dt = 5 * dt
    path = str(tmp_path / "flow.bin")
    binfile.write_bin(d, path)
    out = tmp_path / "out"
    out.mkdir()
    eng = Engine(path, fluid=True, output_dir=str(out))
    assert eng.run() == 0
    eng.close()
    names = sorted(os.listdir(out))
    assert "flow.output00000.bin" in names and "flow.output00002.bin" in names
    assert "flow-conv.log" in names and "flow.status.dat" in names
    lines = (out / "flow-conv.log").read_text().split("\n")
    first = lines[0].split("\t")
    assert first[0] == "1"
    orc = O.Oracle(path, fluid=True)
    assert orc.step(1) == 0
    assert int(first[1]) == int(orc.get("darcy_nijac_last")[0])
    last = binfile.read_bin(str(out / "flow.output00002.bin"), fluid=True)
    assert last.fluid and last.p_f.shape == tuple(int(v) for v in d.num)
