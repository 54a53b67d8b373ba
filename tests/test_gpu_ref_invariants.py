"""The reference's own invariant tests, run through ``sim.run()`` on the engine.

Every scene is the input file the reference's ``sim`` class writes for that
test (tests/golden/ref_scenes, made by tests/golden/make_ref_scenes.py); it is
run by ``sphere_b200.sim.run`` -- the function ``install()`` puts on the
reference's class -- with the reference's ``../input`` / ``../output`` layout,
and the outputs are read back and checked with the reference test's own
conditions and tolerances:

- tests/contactmodel.py, contactmodel_young.py: momentum and energy balance of
  two-particle collisions (pytestutils.compareFloats, 1e-3 and 0.05);
- tests/contactmodel_wall.py, contactmodel_wall_young.py: rebound velocity,
  energy balance and spin of a particle hitting the bottom wall;
- tests/io_tests.py: the first output file equals the input, the second
  equals it apart from the clock;
- tests/cfd_tests_darcy.py: exact zero pressure with zero iterations, the
  linear steady state under a pressure difference, smooth profiles under a
  fast modulation, the flow direction along x;
- tests/cfd_tests_darcy_particles.py: exact zero pressure with 1000 particles
  under three boundary pairs, the wall moving down under gravity (ndem 1 and
  10), the mean particle velocity under 0.9 and 2.0 times the fluidising
  pressure gradient equal to the reference's own kernels' values (the
  reference misses its own 0.9 bound) and fluidisation at 2.0;
- tests/fluid_particle_interaction_darcy.py: the pressure-gradient and
  buoyancy forces pull the particle down.
"""
import os

import numpy
import pytest

from sphere_b200 import sim as sphsim

import ref_scenes as R

pytestmark = pytest.mark.gpu


class _Sim(R.SceneSim):
    pass


sphsim.install(_Sim)


@pytest.fixture
def root(tmp_path, monkeypatch):
    """cwd = <root>/python, like the reference tests run from tests/."""
    (tmp_path / "python").mkdir()
    monkeypatch.chdir(tmp_path / "python")
    return str(tmp_path)


def run(name, root):
    s = _Sim(name)
    assert s.run(verbose=False) == 0
    return R.manifest()[name]


def last(root, name):
    m = R.manifest()[name]
    return R.readlast(root, m["sid"], m["fluid"])


# ---------------------------------------------------------------- contact models

@pytest.mark.parametrize("p", ["cm_", "cmy_"])
def test_elastic_normal_collisions(root, p):
    """contactmodel.py:14-67: momentum passes to the struck particle; the
    kinetic energy is kept."""
    m = run(p + "elastic_1", root)
    after = last(root, p + "elastic_1")
    assert R.compare_floats(m["orig_vel0z"], after.vel[1, 2])
    assert R.compare_floats(m["orig_ekin"], R.total_kinetic(after))
    for tag in ("elastic_2", "elastic_3"):
        m = run(p + tag, root)
        assert R.compare_floats(m["orig_ekin"], R.total_kinetic(last(root, p + tag)))


@pytest.mark.parametrize("p", ["cm_", "cmy_"])
def test_viscoelastic_normal_collisions(root, p):
    """contactmodel.py:70-138: kinetic energy lost = viscous energy (5 %)."""
    m = run(p + "visc_1", root)
    after = last(root, p + "visc_1")
    assert m["orig_vel0z"] > after.vel[1, 2]
    assert R.compare_floats(m["orig_ekin"], R.total_kinetic(after) + R.total_viscous(after),
                            0.05)
    for tag in ("visc_2", "visc_3"):
        m = run(p + tag, root)
        after = last(root, p + tag)
        assert R.compare_floats(m["orig_ekin"],
                                R.total_kinetic(after) + R.total_viscous(after), 0.05)


@pytest.mark.parametrize("p", ["cm_", "cmy_"])
def test_oblique_collisions(root, p):
    """contactmodel.py:142-219: spin about -y, and the energy balance with
    rotational, frictional and viscous terms (5 %)."""
    m = run(p + "oblique_noslip", root)
    a = last(root, p + "oblique_noslip")
    assert (a.angvel[:, 1] < 0.0).all()
    assert R.compare_floats(m["orig_ekin"], R.total_kinetic(a) + R.total_rotational(a), 0.05)

    m = run(p + "oblique_slip", root)
    a = last(root, p + "oblique_slip")
    assert R.compare_floats(m["orig_ekin"], R.total_kinetic(a) + R.total_rotational(a)
                            + R.total_frictional(a), 0.05)
    assert (a.angvel[:, 1] < 0.0).all()
    assert R.total_frictional(a) > 0.0

    m = run(p + "oblique_slip_visc", root)
    a = last(root, p + "oblique_slip_visc")
    assert R.compare_floats(m["orig_ekin"], R.total_kinetic(a) + R.total_rotational(a)
                            + R.total_frictional(a) + R.total_viscous(a), 0.05)
    assert (a.angvel[:, 1] < 0.0).all()
    assert R.total_frictional(a) > 0.0


@pytest.mark.parametrize("p", ["wall_", "wally_"])
def test_wall_collisions(root, p):
    """contactmodel_wall.py: elastic rebound at 0.1 m/s with the kinetic
    energy kept; viscous loss equal to the viscous energy (5 %); after an
    oblique viscous impact the particle spins about +y only."""
    m = run(p + "elastic_normal", root)
    a = last(root, p + "elastic_normal")
    assert R.compare_floats(a.vel[0, 2], 0.1)
    assert R.compare_floats(m["orig_ekin_total"], R.total_kinetic(a))

    m = run(p + "elastic_oblique", root)
    assert R.compare_floats(m["orig_ekin_total"], R.total_kinetic(last(root, p + "elastic_oblique")))

    m = run(p + "visc_normal", root)
    a = last(root, p + "visc_normal")
    ekin_after = R.total_kinetic(a)
    assert m["orig_ekin"] > ekin_after
    assert R.compare_floats(m["orig_ekin"], ekin_after + R.total_viscous(a), 0.05)

    # the reference's check (1/2) here compares the previous case's values
    # again (its variables are not reassigned); the energy of this case is
    # checked instead
    m = run(p + "visc_oblique", root)
    a = last(root, p + "visc_oblique")
    assert m["orig_ekin"] > R.total_kinetic(a)
    assert a.angvel[0, 0] == 0.0 and a.angvel[0, 1] > 0.0 and a.angvel[0, 2] == 0.0


# ---------------------------------------------------------------- input/output

# the fields sim.__cmp__ compares (python/sphere.py:456-700)
CMP_FIELDS = ("version", "nd", "np", "time_dt", "time_current", "time_total", "time_file_dt",
              "time_step_count", "origo", "L", "num", "periodic", "adaptive", "x", "radius",
              "xyzsum", "vel", "fixvel", "force", "angpos", "angvel", "torque", "es_dot", "es",
              "ev_dot", "ev", "p", "g", "k_n", "k_t", "k_r", "E", "gamma_n", "gamma_t",
              "gamma_r", "mu_s", "mu_d", "mu_r", "rho", "contactmodel", "kappa", "db", "V_b",
              "nw", "wmode", "w_n", "w_x", "w_m", "w_vel", "w_force", "w_sigma0", "w_sigma0_A",
              "w_sigma0_f", "w_tau_x", "gamma_wn", "gamma_wt", "lambda_bar", "nb0", "sigma_b",
              "tau_b", "bonds", "bonds_delta_n", "bonds_delta_t", "bonds_omega_n",
              "bonds_omega_t", "fluid")


def _differs(a, b):
    bad = []
    for f in CMP_FIELDS:
        x, y = numpy.asarray(getattr(a, f)), numpy.asarray(getattr(b, f))
        if x.shape != y.shape or not numpy.array_equal(x, y, equal_nan=True):
            bad.append(f)
    return bad


def test_io_round_trip(root):
    """io_tests.py:20-41: output 0 equals the input, output 1 equals it once
    the clock fields are set back."""
    from sphere_b200 import binfile
    m = run("io_initgrid", root)
    orig = binfile.parse_bin(R.scene_bytes("io_initgrid"))
    cpp = R.readstep(root, m["sid"], 0, False)
    assert _differs(orig, cpp) == []
    cuda = R.readstep(root, m["sid"], 1, False)
    cuda.time_current = orig.time_current
    cuda.time_step_count = orig.time_step_count
    assert _differs(orig, cuda) == []


# ---------------------------------------------------------------- Darcy

def _conv(root, sid):
    return numpy.loadtxt(os.path.join(root, "output", sid + "-conv.log"), ndmin=2)


def test_darcy_no_forcing(root):
    """cfd_tests_darcy.py:13-46: pressure stays exactly zero, no iterations,
    no flow."""
    m = run("cfd_no_forcing", root)
    py = last(root, "cfd_no_forcing")
    assert numpy.array_equal(py.p_f, numpy.zeros(py.p_f.shape))
    assert _conv(root, m["sid"])[:, 1].sum() == 0.0
    assert (numpy.abs(py.v_f) < 1.0e-6).all()


def test_darcy_pressure_gradient(root):
    """cfd_tests_darcy.py:50-79: the linear steady state within 0.1, flow
    towards -z only.  (The reference only prints its iteration-count check.)"""
    m = run("cfd_pressure_gradient", root)
    py = last(root, "cfd_pressure_gradient")
    ideal = numpy.asarray(m["ideal_p_z"])
    assert numpy.allclose(numpy.zeros((1, len(ideal))), ideal - py.p_f[0, 0, :], atol=1.0e-1)
    assert (py.v_f[:, :, :, 2] < 0.0).all() and (py.v_f[:, :, :, 0:1] < 1.0e-7).all()
    it = _conv(root, m["sid"])
    print("convergence rate (2/3):", bool((it[0:6, 1] < 1000).all() and (it[6:, 1] < 20).all()))


def test_darcy_fast_pressure_modulation(root):
    """cfd_tests_darcy.py:139-158: every output's profile stays within 0.5 of
    linear."""
    m = run("cfd_fast_modulation", root)
    n = R.status(root, m["sid"])
    assert n >= 9
    for it in range(1, n + 1):
        py = R.readstep(root, m["sid"], it, True)
        ideal = numpy.linspace(py.p_f[0, 0, 0], py.p_f[0, 0, -1], int(py.num[2]))
        assert numpy.allclose(numpy.zeros((1, int(py.num[2]))), ideal - py.p_f[0, 0, :],
                              atol=5.0e-1), it


def test_darcy_perturbation_and_top_flux_run(root):
    """cfd_tests_darcy.py:161-216: the pressure perturbation and the top flux
    runs (the reference checks nothing of them; they must run to the end with
    finite fields)."""
    for name in ("cfd_pressure_perturbation", "cfd_flux_top"):
        run(name, root)
        py = last(root, name)
        assert numpy.isfinite(py.p_f).all() and numpy.isfinite(py.v_f).all()


def test_darcy_gradient_along_x(root):
    """cfd_tests_darcy.py:220-240: flow towards +x everywhere."""
    run("cfd_gradient_x", root)
    py = last(root, "cfd_gradient_x")
    assert (py.v_f[:, :, :, 0] > 0.0).all()


@pytest.mark.parametrize("name", ["dp_steady_dd", "dp_steady_nd", "dp_steady_nn"])
def test_darcy_particles_steady_state(root, name):
    """cfd_tests_darcy_particles.py:6-111: 1000 particles, no gravity, no
    forcing: the pressure stays exactly zero and there is no flow."""
    run(name, root)
    py = last(root, name)
    assert numpy.array_equal(py.p_f, numpy.zeros(py.p_f.shape))
    assert (numpy.abs(py.v_f) < 1.0e-6).all()


@pytest.mark.parametrize("name", ["dp_wall_ndem1", "dp_wall_ndem10"])
def test_darcy_consolidation_wall_moves(root, name):
    """cfd_tests_darcy_particles.py:115-163: on the consolidated cube-init
    packing the wall moves down."""
    m = run(name, root)
    assert m["orig_w_x0"] > last(root, name).w_x[0]


@pytest.mark.parametrize("factor", [0.9, 2.0])
def test_darcy_fluidisation(root, factor):
    """cfd_tests_darcy_particles.py:166-215: the mean vertical particle
    velocity at every output file equals the one the reference's own kernels
    (compiled for the host) give on the same input, within 1e-3 relative
    (ref_scenes/answers.json).  The reference test asks for less than
    0.002 m/s at 0.9 times the fluidising gradient and more at 2.0; its own
    kernels give 0.047 m/s at 0.9 on this set-up (the bottom pressure is
    switched on against a zero interior, and the packing lifts before the
    pressure diffuses up the 2.8 m column), so the 0.9 condition is held
    against the reference's values and the 2.0 condition is asserted as
    written."""
    name = f"dp_fluidization_{factor}"
    m = run(name, root)
    ref = R.answers()[name]
    assert R.status(root, m["sid"]) == len(ref["mean_vz"])
    for i, want in enumerate(ref["mean_vz"]):
        w = float(numpy.mean(R.readstep(root, m["sid"], i + 1, True).vel[:, 2]))
        assert abs(w - want) <= 1e-3 * abs(want), (i + 1, w, want)
    w = numpy.mean(last(root, name).vel[:, 2])
    if factor < 1.0:
        assert ref["mean_vz"][-1] > 0.002   # the reference misses its own bound
    else:
        assert w > 0.002


@pytest.mark.parametrize("name", ["fpi_pressure_gradient", "fpi_buoyancy"])
def test_fluid_particle_interaction(root, name):
    """fluid_particle_interaction_darcy.py: the particle moves towards the
    low pressure (test 1) and sinks under gravity with buoyancy (test 2)."""
    run(name, root)
    assert last(root, name).vel[0, 2] < 0.0
