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


def field_errors(eng, orc):
    """Largest |engine - oracle| of each field over the field's largest
    magnitude."""
    errs = {}
    for a_name, b_name in PAIRS:
        a = numpy.asarray(eng.get(a_name), dtype=float)
        b = numpy.asarray(orc.get(b_name), dtype=float)
        if a_name in ("x", "vel", "force", "darcy_f_p"):
            a, b = a.reshape(-1, 4)[:, :3], b.reshape(-1, 4)[:, :3]
        scale = max(float(numpy.abs(b).max()), 1e-300)
        errs[a_name] = float(numpy.abs(a.ravel() - b.ravel()).max()) / scale
    return errs


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
    worst = {}
    for k in range(6):
        assert eng.step(1) == 0
        assert orc.step(1) == 0, orc.error()
        bad = compare(eng, orc)
        assert not bad, f"after step {k + 1}: {bad}"
        for f, e in field_errors(eng, orc).items():
            worst[f] = max(worst.get(f, 0.0), e)
    print(f"\n{name}: worst relative error per field: "
          + ", ".join(f"{f} {e:.2e}" for f, e in sorted(worst.items())))
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


def grid_case(seed, n=3000, maxiter=200000):
    """A few thousand spheres on the 40 x 40 x 80 fluid grid of the
    consolidation workload: 128,000 cells, so the Jacobi launch spans 500
    blocks of 256 cells and each block waits only for the ~13 blocks within
    one z layer of its cells (nb_lo > 0 and nb_hi < G - 1 for most blocks)."""
    d = configs.settling_lattice(n=n, seed=seed, nx=20, ny=20, nz=8, spacing=0.0462, steps=40)
    dx = 2.1 * 0.011
    d.num = numpy.array([40, 40, 80], dtype=numpy.uint32)
    d.L = d.num.astype(numpy.float64) * dx
    configs.add_top_wall(d, 10e3)
    # the workload's permeability prefactor, compressibility and tolerance; a
    # water viscosity keeps the loose packing's (porosity 0.9) pressure
    # diffusion within the explicit step's stability limit at the DEM dt
    configs.init_fluid_darcy(d, mu=8.9e-4, rho_f=1000.0, k_c=3.5e-13, beta_f=4.5e-10,
                             tolerance=1e-8, maxiter=maxiter, bottom_no_flow=True)
    return d


GRID_CASES = {
    "reference_stop": dict(),
    "exact_stop": dict(exact=True),
    "maxiter_mid_ring": dict(maxiter=137),
}

# Beyond RTOL, a field may differ from the oracle by at most SENS_FACTOR
# times what the oracle itself moves when its pow calls are replaced by
# products (oracle/liboracle_powprod.so): last-bit changes of the sphere
# volumes and permeabilities, the size of the difference between CUDA's pow
# and glibc's.  On this grid the non-converged Jacobi solve (the stop rule is
# a relative change of 1e-8 per iteration) carries such changes into the
# pressure at ~1e-9 of its maximum, where the 7 x 7 x 7 cases stay near 1e-11.
SENS_FACTOR = 10.0


@pytest.mark.parametrize("name", list(GRID_CASES))
def test_darcy_parity_benchmark_grid(tmp_path, name):
    """The neighbour-subset waits, the one-iteration-late stop decision and
    the residual ring of the Jacobi kernel at the benchmark grid size:
    identical iteration counts and fields within the bound above over three
    fluid steps.  maxiter 137 ends the solve at a check that is not a
    multiple of 10, after the 64-slot residual ring has wrapped twice."""
    from sphere_b200.engine import Engine
    opt = dict(GRID_CASES[name])
    exact = opt.pop("exact", False)
    d = grid_case(61, **opt)
    path = str(tmp_path / "grid.bin")
    binfile.write_bin(d, path)
    orc = O.Oracle(path, fluid=True)
    probe = O.Oracle(path, fluid=True, lib_path=O.POWPROD_SO)
    if exact:
        for o in (orc, probe):
            o.set("darcy_exact_stop", numpy.array([1], dtype=numpy.int32))
    eng = Engine(path, fluid=True, precision="faithful", darcy_exact_stop=exact)
    iters = []
    worst, worst_sens = {}, {}
    for k in range(3):
        rc_e = eng.step(1)
        assert orc.step(1) == 0, orc.error()
        assert probe.step(1) == 0, probe.error()
        it_o = int(orc.get("darcy_nijac_last")[0])
        iters.append(it_o)
        assert int(eng.get("darcy_iters")[0]) == it_o, f"step {k + 1}"
        assert rc_e == (1 if it_o + 1 == d.maxiter and it_o > 0 else 0), (k, rc_e, it_o)
        errs = field_errors(eng, orc)
        sens = field_errors(probe, orc)
        for f, e in errs.items():
            worst[f] = max(worst.get(f, 0.0), e)
            worst_sens[f] = max(worst_sens.get(f, 0.0), sens[f])
        bad = {f: (e, sens[f]) for f, e in errs.items() if not e <= max(RTOL, SENS_FACTOR * sens[f])}
        assert not bad, f"after step {k + 1}: (error, probe) {bad}"
    print(f"\n{name}: iterations {iters}; worst relative error per field (probe): "
          + ", ".join(f"{f} {e:.2e} ({worst_sens[f]:.2e})" for f, e in sorted(worst.items())))
    assert max(iters) >= 40, iters
    if "maxiter" in opt:
        assert max(iters) == opt["maxiter"] - 1
    if exact:
        assert any(i % 10 for i in iters), iters
    eng.close()
