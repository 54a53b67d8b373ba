"""The engine's Navier-Stokes solver (cfd_solver 0) against the reference's
own Navier-Stokes kernels built for the host (oracle/_ref, driven through
the stage order of DEM::startTime, device.cu:1213-1898) and against the
committed fixture made from them (tests/golden/ns_settling.*).

The device code keeps the reference's operation order with FMA contraction
off, but the drag law's pow/exp/log10 come from CUDA's math library on the
device and glibc's on the host, which may differ in the last bit, and the
coupled state then drifts by rounding.  Fields are therefore compared to a
relative tolerance of 1e-9 of each field's largest magnitude; the Jacobi
iteration counts must match exactly.
"""
import os

import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-9
# (engine field, reference field)
PAIRS = (("darcy_p", "ns_p"), ("darcy_phi", "ns_phi"), ("darcy_dphi", "ns_dphi"),
         ("darcy_v", "ns_v"), ("ns_v_face", "ns_v_face"), ("ns_epsilon", "ns_epsilon"),
         ("ns_norm", "ns_norm"), ("ns_f_d", "ns_f_d"), ("darcy_f_p", "ns_f_p"),
         ("ns_f_v", "ns_f_v"), ("ns_f_sum", "ns_f_sum"), ("x", "x"), ("vel", "vel"),
         ("force", "force"))
_PART = {"x", "vel", "force", "darcy_f_p", "ns_f_d", "ns_f_v", "ns_f_sum"}


def ns_case(seed, periodic=1, top_wall=False, ndem=1, n=300, maxiter=2000, beta=0.0,
            bc_bot=0, bc_top=0, p_mod=None, mu=8.9e-4, hydrostatic=True, lattice=(7, 7, 7),
            tall=1):
    d = configs.settling_lattice(n=n, seed=seed, nx=lattice[0], ny=lattice[1], nz=lattice[2],
                                 spacing=0.0195, steps=40)
    if tall > 1:
        # the same cells, `tall` times as many layers (fluid above the packing)
        d.L = numpy.array([d.L[0], d.L[1], d.L[2] * tall])
        d.num = numpy.array([d.num[0], d.num[1], d.num[2] * tall], dtype=numpy.uint32)
    d.periodic = periodic
    if top_wall:
        configs.add_top_wall(d, 10e3)
        d.w_x[0] -= 0.002
    configs.init_fluid_ns(d, mu=mu, hydrostatic=hydrostatic, tolerance=1e-6, maxiter=maxiter,
                          ndem=ndem, beta=beta, bc_bot=bc_bot, bc_top=bc_top)
    if p_mod is not None:
        d.p_mod_A, d.p_mod_f = p_mod
    return d


def compare(eng, get_ref, it_ref):
    bad = {}
    for a_name, b_name in PAIRS:
        a = numpy.asarray(eng.get(a_name), dtype=float)
        b = numpy.asarray(get_ref(b_name), dtype=float)
        if a_name in _PART:
            a, b = a.reshape(-1, 4)[:, :3], b.reshape(len(a), -1)[:, :3]
        a, b = a.ravel(), b.ravel()
        if a.shape != b.shape:
            bad[a_name] = f"shape {a.shape} vs {b.shape}"
            continue
        scale = max(float(numpy.abs(b).max()), 1e-300)
        err = float(numpy.abs(a - b).max()) / scale
        if not err <= RTOL:
            bad[a_name] = f"relative max error {err:.3e}"
    it_e = int(eng.get("darcy_iters")[0])
    if it_e != it_ref:
        bad["iterations"] = f"{it_e} vs {it_ref}"
    return bad


CASES = {
    "dirichlet": dict(),
    "top_wall": dict(top_wall=True),
    "neumann_bottom": dict(bc_bot=1),
    "noslip_bottom": dict(bc_bot=2),
    "neumann_top": dict(bc_top=1),
    "periodic_x": dict(periodic=2),
    "pressure_projection": dict(beta=0.5),
    "ndem2": dict(ndem=2),
    "top_modulation": dict(p_mod=(200.0, 5.0)),
    "inviscid": dict(mu=0.0),
    # an 11 x 11 x 22 grid: the Jacobi launch spans several blocks that
    # wait for their z neighbours (or, with the periodic z ghosts of
    # bc_bot 2, for all blocks)
    "multiblock": dict(n=1500, lattice=(12, 12, 11), tall=2),
    "multiblock_wall": dict(n=1500, lattice=(12, 12, 11), tall=2, top_wall=True),
    "multiblock_zwrap": dict(n=1500, lattice=(12, 12, 11), tall=2, bc_bot=2),
}


@pytest.mark.skipif(not O.ref_available(), reason="the reference's host build (oracle/_ref) is absent")
@pytest.mark.parametrize("name", list(CASES))
def test_ns_parity(tmp_path, name):
    from sphere_b200.engine import Engine
    d = ns_case(61, **CASES[name])
    path = str(tmp_path / "ns.bin")
    binfile.write_bin(d, path)
    ref = O.Reference(path, fluid=True)
    eng = Engine(path, fluid=True, precision="faithful")
    for k in range(5):
        assert eng.step(1) in (0, 1)
        assert ref.step(1) == 0
        bad = compare(eng, ref.get, int(ref.get("ns_nijac_last")[0]))
        assert not bad, f"after step {k + 1}: {bad}"
    assert int(eng.get("darcy_iters_total")[0]) == int(ref.get("ns_nijac_total")[0])
    eng.close()
    ref.close()


def test_ns_golden_fixture():
    """The committed settling fixture (the reference's own kernels built for
    the host, steps 1-3) reproduced by the device solver."""
    from sphere_b200.engine import Engine
    here = os.path.join(os.path.dirname(__file__), "golden")
    gold = numpy.load(os.path.join(here, "ns_settling.npz"))
    eng = Engine(os.path.join(here, "ns_settling.bin"), fluid=True, precision="faithful")
    for step in (1, 2, 3):
        assert eng.step(1) == 0
        it = int(gold[f"ns_nijac_last@{step}"].ravel()[0])
        bad = compare(eng, lambda f: gold[f"{f}@{step}"], it)
        assert not bad, (step, bad)
    eng.close()


def test_ns_file_roundtrip(tmp_path):
    """A written output carries the solver's fields in the reference's layout
    (bottom condition first, which its reader takes as the top one), and the
    reference writes the same bytes after the same steps."""
    from sphere_b200.engine import Engine
    d = ns_case(62, bc_bot=1, bc_top=0)
    path = str(tmp_path / "ns.bin")
    binfile.write_bin(d, path)
    eng = Engine(path, fluid=True, precision="faithful")
    assert eng.step(2) == 0
    out = str(tmp_path / "out.bin")
    eng.write_bin(out)
    eng.close()
    back = binfile.read_bin(out, fluid=True)
    assert back.cfd_solver == 0
    assert (back.bc_top, back.bc_bot) == (1, 0)
    if O.ref_available():
        ref = O.Reference(path, fluid=True)
        ref.step(2)
        rout = str(tmp_path / "ref.bin")
        ref.write_bin(rout)
        ref.close()
        a = binfile.read_bin(rout, fluid=True)
        for name in ("p_f", "phi", "dphi", "v_f", "f_d", "f_p", "f_v", "f_sum"):
            x, y = numpy.asarray(getattr(back, name)), numpy.asarray(getattr(a, name))
            scale = max(float(numpy.abs(y).max()), 1e-300)
            assert float(numpy.abs(x - y).max()) <= RTOL * scale, name


def test_ns_run_files(tmp_path):
    """run() checks the reference's stability criteria, writes the output
    files, the status file and the conv log (its first line: step 1 and the
    reference's iteration count)."""
    from sphere_b200.engine import Engine
    d = ns_case(63, top_wall=True)
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
    first = (out / "flow-conv.log").read_text().split("\n")[0].split("\t")
    assert first[0] == "1"
    gold = binfile.read_bin(str(out / "flow.output00002.bin"), fluid=True)
    assert gold.cfd_solver == 0 and numpy.isfinite(gold.p_f).all()
    if O.ref_available():
        ref = O.Reference(path, fluid=True)
        assert ref.step(1) == 0
        assert int(first[1]) == int(ref.get("ns_nijac_last")[0])
        ref.close()


def test_ns_run_rejects_unstable_time_step(tmp_path):
    """The reference exits when mu dt / dmin^2 > 0.5 before writing a file;
    the engine's run() returns SPH_ERR_INPUT there (raised by the wrapper)."""
    from sphere_b200.engine import Engine
    d = ns_case(64, mu=1500.0)
    dt = float(d.time_dt)
    d.time_total = 6 * dt
    d.time_file_dt = 5 * dt
    path = str(tmp_path / "flow.bin")
    binfile.write_bin(d, path)
    out = tmp_path / "out"
    out.mkdir()
    from sphere_b200.engine import EngineError
    eng = Engine(path, fluid=True, output_dir=str(out))
    with pytest.raises(EngineError, match="diffusive term"):
        eng.run()
    eng.close()
    assert not (out / "flow.output00001.bin").exists()


def test_ns_smoothing_runs(tmp_path):
    """gamma > 0 smooths the pressure change after each converged solve
    (read before write here; the reference's in-place update races), and the
    run stays finite with the same iteration counts as without smoothing on
    the first step."""
    from sphere_b200.engine import Engine
    d = ns_case(65)
    d.ns_gamma = 0.2
    path = str(tmp_path / "s.bin")
    binfile.write_bin(d, path)
    eng = Engine(path, fluid=True)
    for _ in range(4):
        assert eng.step(1) in (0, 1)
    assert numpy.isfinite(eng.get("ns_epsilon")).all()
    assert numpy.isfinite(eng.get("darcy_v")).all()
    eng.close()


def test_ns_with_mixed_precision_contacts(tmp_path):
    """The fluid stage is FP64 in every precision; with mixed-precision
    contacts the coupled run stays within the mixed mode's force tolerance
    of the faithful one over a few steps, with the same iteration counts."""
    from sphere_b200.engine import Engine
    d = ns_case(66, top_wall=True)
    path = str(tmp_path / "m.bin")
    binfile.write_bin(d, path)
    a = Engine(path, fluid=True, precision="faithful")
    b = Engine(path, fluid=True, precision="mixed")
    for _ in range(5):
        assert a.step(1) == 0 and b.step(1) == 0
        assert int(a.get("darcy_iters")[0]) == int(b.get("darcy_iters")[0])
    for name in ("darcy_p", "darcy_v", "ns_f_d"):
        x, y = numpy.asarray(b.get(name), dtype=float), numpy.asarray(a.get(name), dtype=float)
        assert numpy.linalg.norm(x - y) <= 1e-5 * numpy.linalg.norm(y), name
    a.close()
    b.close()


def _cfd_box(ptop=None):
    """The reference's tests/cfd_tests.py set-up: one sphere (r = 0.05 m) in
    a 1 m box, fluid with mu = 0 and p = 0, ten time steps, a file each."""
    from sphere_b200.binfile import BinData
    d = BinData()
    configs._particles(d, 1)
    d.radius = numpy.array([0.05])
    d.x[0, :] = [0.5, 0.5, 0.5]
    configs.default_params(d)
    configs.grid_for(d, L=[1.0, 1.0, 1.0])
    configs.init_temporal(d, total=0.2, file_dt=0.01)
    d.time_file_dt = d.time_dt * 0.99
    d.time_total = d.time_dt * 10
    configs.init_fluid_ns(d, mu=0.0)
    if ptop is not None:
        d.p_f[:, :, -1] = ptop
    return d


def _run_files(tmp_path, d, sid):
    from sphere_b200.engine import Engine
    path = str(tmp_path / f"{sid}.bin")
    binfile.write_bin(d, path)
    out = tmp_path / sid
    out.mkdir()
    eng = Engine(path, fluid=True, output_dir=str(out))
    assert eng.run() == 0
    eng.close()
    last = sorted(p for p in os.listdir(out) if ".output" in p)[-1]
    conv = numpy.loadtxt(str(out / f"{sid}-conv.log"), ndmin=2)
    return binfile.read_bin(str(out / last), fluid=True), conv


def test_ns_reference_cfd_invariants(tmp_path):
    """The checks of the reference's tests/cfd_tests.py (Dirichlet
    boundaries) through run(), its files and its conv log: a fluid at rest
    stays at rest with no iterations; a raised top pressure relaxes to a
    linear profile (within 0.1 of it) with downward flow only."""
    py, conv = _run_files(tmp_path, _cfd_box(), "rest")
    assert numpy.array_equal(py.p_f, numpy.zeros(py.p_f.shape))
    assert conv[:, 1].sum() == 0.0
    assert (numpy.abs(py.v_f) < 1.0e-6).all()
    d = _cfd_box(ptop=1.1)
    py, conv = _run_files(tmp_path, d, "grad")
    ideal = numpy.linspace(d.p_f[0, 0, 0], d.p_f[0, 0, -1], int(d.num[2]))
    assert numpy.abs(ideal - py.p_f[0, 0, :]).max() < 1.0e-1
    assert (py.v_f[:, :, :, 2] < 0.0).all() and (py.v_f[:, :, :, 0:1] < 1.0e-7).all()


def _one_fluid_box(positions, ndem=1, g=None, p_bot=None, p_top=None, total=0.01, file_dt=0.001):
    """The reference's tests/fluid_particle_interaction.py set-up: a 1 m box
    on 0.1 m cells, water (initFluid's defaults), particles of the fluid's
    density (r = 0.05 m)."""
    from sphere_b200.binfile import BinData
    d = BinData()
    configs._particles(d, len(positions))
    d.radius = numpy.full(len(positions), 0.05)
    d.x[:, :] = numpy.asarray(positions, dtype=float)
    configs.default_params(d, rho=1000.0)
    if g is not None:
        d.g = numpy.asarray(g, dtype=float)
    configs.grid_for(d, L=[1.0, 1.0, 1.0], dx=0.1)
    configs.init_temporal(d, total=total, file_dt=file_dt)
    configs.init_fluid_ns(d, ndem=ndem)
    if p_bot is not None:
        d.p_f[:, :, 0] = p_bot
    if p_top is not None:
        d.p_f[:, :, -1] = p_top
    return d


def test_ns_reference_fluid_particle_interaction(tmp_path):
    """The checks of the reference's tests/fluid_particle_interaction.py: a
    pressure gradient (10 Pa at the bottom, 1 Pa at the top) lifts a
    neutrally buoyant sphere; a fluid driven along x by gravity moves along
    x everywhere and drags the spheres with it."""
    d = _one_fluid_box([[0.5, 0.5, 0.5]], ndem=100, p_bot=10.0, p_top=1.0)
    py, _ = _run_files(tmp_path, d, "lift")
    assert py.vel[0, 2] > 0.0
    d = _one_fluid_box([[0.5, 0.5, 0.75], [0.5, 0.5, 0.50], [0.5, 0.5, 0.25]], g=[10.0, 0.0, 0.0],
                       total=0.0001, file_dt=0.00001)
    py, _ = _run_files(tmp_path, d, "drag")
    assert (py.v_f[:, :, :, 0] > 0.0).all()
    assert (py.vel[:, 0] > 0.0).all()
