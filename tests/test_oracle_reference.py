"""The oracle against the reference's own kernels compiled for the host
(oracle/_ref), live, on inputs beyond the committed golden set: bonds,
the shear-stress wall mode, Young's modulus walls.  Skipped where the
reference tree (and so oracle/_ref) is not available."""
import os

import numpy
import pytest

import oracle as O
from helpers import bonded_packing, compare_states
from sphere_b200 import binfile, configs

pytestmark = pytest.mark.skipif(
    not (O.ref_available() or O.ref_path("src")),
    reason="reference sources not present")

FIELDS = ("x", "vel", "angvel", "angpos", "force", "torque", "xyzsum", "es", "ev", "p",
          "contacts", "delta_t", "index", "cellid", "walls_nx", "walls_mvfd")


@pytest.fixture(scope="module", autouse=True)
def built():
    O.build(ref=True)


def run_pair(tmp_path, d, chunks=(1, 4, 15), extra=()):
    path = str(tmp_path / "case.bin")
    binfile.write_bin(d, path)
    orc = O.Oracle(path)
    ref = O.Reference(path)
    for c in chunks:
        assert orc.step(c) == 0, orc.error()
        ref.step(c)
        bad = compare_states(orc.get, ref.get, FIELDS + tuple(extra))
        assert not bad, bad
    return orc, ref


def test_bonds(tmp_path):
    d = bonded_packing(configs, max_bonds=300)
    assert d.nb0 > 100
    orc, _ = run_pair(tmp_path, d, extra=("bonds", "bonds_delta", "bonds_omega"))
    assert (orc.get("bonds")[0::2] < d.np).sum() > 0


def test_bonds_breaking(tmp_path):
    d = bonded_packing(configs, seed=22, max_bonds=300)
    d.sigma_b = 2e3  # weak bonds break during the run
    orc, _ = run_pair(tmp_path, d, chunks=(2, 10, 30),
                      extra=("bonds", "bonds_delta", "bonds_omega"))
    assert (orc.get("bonds")[0::2] == d.nb0).sum() > 0


def test_shear_stress_wall_mode(tmp_path):
    d = configs.settling_lattice(n=400, seed=23, nx=8, ny=8, nz=7, spacing=0.0195, steps=40)
    configs.shear_setup(d, 0.0, 20e3)
    d.w_x[0] -= 0.002
    d.wmode[0] = 3
    d.w_tau_x = 5e3
    run_pair(tmp_path, d)


def test_sigma0_modulation(tmp_path):
    d = configs.settling_lattice(n=400, seed=24, nx=8, ny=8, nz=7, spacing=0.0195, steps=40)
    configs.add_top_wall(d, 10e3)
    d.w_x[0] -= 0.002
    d.w_sigma0_A = 5e3
    d.w_sigma0_f = 50.0
    run_pair(tmp_path, d)


def test_reference_fixture_init_1e4(tmp_path):
    src = O.ref_path("output", "init-1e4.output00199.bin")
    if not src:
        pytest.skip("fixture not present")
    dst = str(tmp_path / "init.bin")
    d = binfile.upgrade_to_215(src, dst)
    assert d.np == 10000
    orc = O.Oracle(dst)
    ref = O.Reference(dst)
    orc.step(3)
    ref.step(3)
    bad = compare_states(orc.get, ref.get, FIELDS)
    assert not bad, bad
    assert (orc.get("contacts") != d.np).sum() > 10000


DARCY_FIELDS = ("darcy_p", "darcy_phi", "darcy_dphi", "darcy_k", "darcy_v", "darcy_f_p",
                "darcy_nijac_last", "force", "x", "vel")


def darcy_case(seed, periodic=1, bottom_no_flow=True, top_wall=True, ndem=1):
    d = configs.settling_lattice(n=300, seed=seed, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    d.periodic = periodic
    if top_wall:
        configs.add_top_wall(d, 10e3)
        d.w_x[0] -= 0.002
    configs.init_fluid_darcy(d, mu=1.797e-6, k_c=3.5e-13, tolerance=1e-8, maxiter=2000,
                             bottom_no_flow=bottom_no_flow, ndem=ndem)
    return d


@pytest.mark.parametrize("kw", [dict(), dict(bottom_no_flow=False), dict(periodic=2),
                                dict(top_wall=False), dict(ndem=2)],
                         ids=["neumann_bottom", "dirichlet_bottom", "periodic_x", "no_wall", "ndem2"])
def test_darcy(tmp_path, kw):
    d = darcy_case(51, **kw)
    path = str(tmp_path / "darcy.bin")
    binfile.write_bin(d, path)
    orc = O.Oracle(path, fluid=True)
    ref = O.Reference(path, fluid=True)
    for _ in range(4):
        assert orc.step(1) == 0, orc.error()
        ref.step(1)
        bad = compare_states(orc.get, ref.get, DARCY_FIELDS)
        assert not bad, bad
    assert orc.get("darcy_nijac_last")[0] > 10


def test_reference_hertz_model_gives_nan_forces(tmp_path):
    """contactmodel 3 in the reference (contactHertz, src/contactmodels.cuh:
    414-591) raises the signed overlap, which is negative for every
    contact, to the powers 3/2, 1/2 and 1/4 (powf of a negative number is
    NaN), so its first contact turns the forces and then the positions into
    NaN.  This is why the engine refuses model 3 (SPH_ERR_UNSUPPORTED) rather
    than reproduce it."""
    d = configs.two_particle(z=(2.0, 3.9), vel0=1.0)
    d.contactmodel = 3
    path = str(tmp_path / "hertz.bin")
    binfile.write_bin(d, path)
    ref = O.Reference(path)
    ref.step(1)
    assert numpy.all(numpy.isnan(ref.get("force")[:, :3]))
    assert numpy.all(numpy.isnan(ref.get("x")[:, :3]))
    # without a contact the same model leaves the particles finite
    d.x[1, 2] = 6.0
    binfile.write_bin(d, path)
    ref = O.Reference(path)
    ref.step(1)
    assert numpy.all(numpy.isfinite(ref.get("x")[:, :3]))


@pytest.mark.skipif(not O.ref_available(), reason="the reference's host build (oracle/_ref) is absent")
def test_reference_ns_reproduces_golden_fixture():
    """The Navier-Stokes fixture under tests/golden is what the reference's
    own kernels give for its input (the generator is deterministic)."""
    here = os.path.join(os.path.dirname(__file__), "golden")
    gold = numpy.load(os.path.join(here, "ns_settling.npz"))
    ref = O.Reference(os.path.join(here, "ns_settling.bin"), fluid=True)
    for step in (1, 2, 3):
        assert ref.step(1) == 0
        for key in gold.files:
            name, at = key.split("@")
            if int(at) == step:
                assert numpy.array_equal(ref.get(name), gold[key]), key
    assert int(gold["ns_nijac_last@3"][0]) > 10
    ref.close()


def test_capillary_cohesion(tmp_path):
    """Model 1 with capillary cohesion (capillaryCohesion_exp,
    src/cohesion.cuh:237-277, called for pairs within db of contact,
    src/contactsearch.cuh:91-186): oracle and reference bit for bit, and the
    cohesion changes the forces."""
    d = configs.settling_lattice(n=500, seed=25, nx=8, ny=8, nz=8, spacing=0.0195, steps=40,
                                 contactmodel=1)
    d.kappa = 0.05
    d.db = 0.002
    d.V_b = 1e-9
    d.gamma_n = 50.0
    orc, _ = run_pair(tmp_path, d)
    d.kappa = 0.0
    path = str(tmp_path / "dry.bin")
    binfile.write_bin(d, path)
    dry = O.Oracle(path)
    assert dry.step(20) == 0
    assert not numpy.array_equal(dry.get("force"), orc.get("force"))
