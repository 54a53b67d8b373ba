"""The engine's FP64 DEM step against the CPU oracle, bit for bit.

Cell ids, sorted order, contact slot rows, forces, torques and the
integrated state must be identical after every checked step (faithful FP64
mode: FP32 vector lengths like the reference).  True-FP64 mode is compared
with the oracle's true-FP64 mode the same way.
"""
import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O

pytestmark = pytest.mark.gpu

VEC3 = ("angvel", "angpos", "force", "torque", "xyzsum", "acc", "angacc")
ALL = ("x", "vel", "angvel", "angpos", "force", "torque", "acc", "angacc", "xyzsum",
       "es_dot", "es", "ev_dot", "ev", "p", "cellid", "index", "contacts", "delta_t",
       "walls_nx", "walls_mvfd")


def _bits(a):
    return numpy.ascontiguousarray(a).view(numpy.uint8)


def compare(eng, orc, names=ALL):
    bad = {}
    for f in names:
        a, b = eng.get(f), orc.get(f)
        if f in VEC3:
            a, b = a[:, :3], b[:, :3]
        if a.shape != b.shape:
            bad[f] = f"shape {a.shape} vs {b.shape}"
        elif a.size and not numpy.array_equal(_bits(a), _bits(b)):
            d = numpy.abs(a.astype(float) - b.astype(float))
            bad[f] = f"max abs diff {numpy.nanmax(d):.3e} at {int(numpy.nanargmax(d))}"
    return bad


def dense(seed, n=600, **kw):
    return configs.settling_lattice(n=n, seed=seed, nx=10, ny=10, nz=8, spacing=0.0195,
                                    steps=100, **kw)


def cases():
    d = dense(1)
    yield "model2", d
    d = dense(1, contactmodel=1)
    yield "model1", d
    d = dense(2); d.E = 7e8; d.periodic = 0
    yield "young_nonperiodic", d
    d = dense(3); d.periodic = 2; d.gamma_n = 50.0; d.gamma_t = 20.0; d.mu_d = 0.3
    yield "periodic_x_viscous", d
    d = dense(4, n=700); configs.add_top_wall(d, 20e3); d.w_x[0] -= 0.003
    yield "top_wall", d
    d = dense(5, n=700); configs.shear_setup(d, 0.05, 20e3); d.w_x[0] -= 0.003; d.E = 7e8
    yield "shear", d


@pytest.mark.parametrize("name,data", list(cases()), ids=[c[0] for c in cases()])
@pytest.mark.parametrize("precision", ["faithful", "fp64"])
@pytest.mark.parametrize("kernel", ["stages", "persistent", "stages_staged", "stages_fused"])
def test_step_parity(tmp_path, name, data, precision, kernel):
    """Every step path -- the per-stage kernels, the fused persistent kernel,
    the per-stage kernels with the contact search reading the neighbour
    cells staged in shared memory, and the per-stage kernels with contacts
    and integration in one launch -- against the oracle, bit for bit."""
    from sphere_b200.engine import Engine
    path = tmp_path / f"{name}.bin"
    binfile.write_bin(data, path)
    orc = O.Oracle(str(path), precision="faithful" if precision == "faithful" else "fp64")
    eng = Engine(str(path), precision=precision, graph_steps=8, step_kernel=kernel)
    for k, n in enumerate((1, 1, 3, 10, 25)):
        assert eng.step(n) == 0
        assert orc.step(n) == 0, orc.error()
        bad = compare(eng, orc)
        assert not bad, f"after chunk {k}: {bad}"
    occupied = (orc.get("contacts") != data.np).sum()
    assert occupied > 0 or data.contactmodel == 1
    eng.close()


@pytest.mark.parametrize("precision", ["faithful", "fp64"])
def test_persistent_autotuned_run(tmp_path, precision):
    """A call long enough to start the block-shape autotuner (trial launches
    of every shape on real steps) still advances exactly like the oracle."""
    from sphere_b200.engine import Engine
    d = dense(6, n=700)
    configs.shear_setup(d, 0.05, 20e3)
    d.w_x[0] -= 0.003
    path = tmp_path / "tuned.bin"
    binfile.write_bin(d, path)
    orc = O.Oracle(str(path), precision=precision)
    eng = Engine(str(path), precision=precision, step_kernel="persistent")
    for n in (60, 7):
        assert eng.step(n) == 0
        assert orc.step(n) == 0, orc.error()
        bad = compare(eng, orc)
        assert not bad, bad
    assert int(eng.get("iter")[0]) == 67
    eng.close()


@pytest.mark.parametrize("precision", ["faithful", "fp64"])
def test_autotuned_run_over_every_step_path(tmp_path, precision):
    """The automatic choice with a call long enough for the autotuner: trial
    steps on every block shape of the persistent kernel, on the per-stage
    kernels and on the per-stage kernels with contacts and integration in
    one launch (whose steps alternate the x / vel / angvel buffers), then the
    winner -- the state must advance exactly like the oracle throughout."""
    from sphere_b200.engine import Engine
    d = dense(12, n=700)
    configs.shear_setup(d, 0.05, 20e3)
    d.w_x[0] -= 0.003
    path = tmp_path / "auto.bin"
    binfile.write_bin(d, path)
    orc = O.Oracle(str(path), precision=precision)
    eng = Engine(str(path), precision=precision, graph_steps=8)
    for n in (90, 7, 16):
        assert eng.step(n) == 0
        assert orc.step(n) == 0, orc.error()
        bad = compare(eng, orc)
        assert not bad, bad
    assert eng.info().tuned == 1
    assert int(eng.get("iter")[0]) == 113
    eng.close()


def test_persistent_refuses_bonds(tmp_path):
    """The fused step does not cover bonds: asking for it is an error, the
    automatic choice falls back to the per-stage kernels."""
    from sphere_b200.engine import Engine, EngineError
    from helpers import bonded_packing
    d = bonded_packing(configs, n=300, seed=3)
    path = tmp_path / "bonded.bin"
    binfile.write_bin(d, path)
    with pytest.raises(EngineError):
        Engine(str(path), step_kernel="persistent")
    with pytest.raises(EngineError):
        Engine(str(path), step_kernel="stages_fused")
    with Engine(str(path)) as eng:
        assert eng.step(2) == 0


def extra_cases():
    d = dense(7, n=700); configs.add_top_wall(d, 10e3); d.w_x[0] -= 0.003
    d.w_sigma0_A = 5e3; d.w_sigma0_f = 50.0
    yield "sigma0_sinusoid", d, 3
    d = dense(8, n=700); configs.shear_setup(d, 0.05, 20e3); d.w_x[0] -= 0.003; d.E = 7e8
    yield "shear_ty2", d, 2
    d = dense(9, n=700); configs.add_top_wall(d, 20e3); d.w_x[0] -= 0.003
    d.gamma_n = 50.0; d.gamma_t = 20.0
    yield "top_wall_viscous_ty2", d, 2


@pytest.mark.parametrize("name,data,integrator", list(extra_cases()),
                         ids=[c[0] for c in extra_cases()])
@pytest.mark.parametrize("kernel", ["stages", "persistent", "stages_fused"])
def test_step_parity_wall_modulation_and_ty2(tmp_path, name, data, integrator, kernel):
    """The sinusoidal normal stress of wall 0 (sigma0 + A sin(2 pi f t),
    src/integration.cuh:383-384) and the two-term Taylor integrator
    (src/integration.cuh:192-220, 417-427) on every step path, bit for bit."""
    from sphere_b200.engine import Engine
    path = tmp_path / f"{name}.bin"
    binfile.write_bin(data, path)
    orc = O.Oracle(str(path), integrator=integrator)
    eng = Engine(str(path), integrator=integrator, graph_steps=8, step_kernel=kernel)
    for k, n in enumerate((1, 2, 9, 30)):
        assert eng.step(n) == 0
        assert orc.step(n) == 0, orc.error()
        bad = compare(eng, orc)
        assert not bad, f"after chunk {k}: {bad}"
    eng.close()


def shear_stress_box(seed):
    d = dense(seed, n=700)
    configs.shear_setup(d, 0.0, 20e3)
    d.w_x[0] -= 0.003
    d.wmode[0] = 3
    d.w_tau_x = 5e3
    return d


@pytest.mark.parametrize("precision", ["faithful", "fp64"])
def test_step_parity_shear_stress_wall(tmp_path, precision):
    """Wall mode 3: the top particles are driven by the shear stress tau_x
    plus the effective stress of the fixed moving particles
    (findShearStressOnFixedMovingParticles + summation,
    src/integration.cuh:457-484, on the device as k_shear_stress and
    k_tau_partials), bit for bit.  The fused step refuses wmode 3, so the
    automatic choice runs the per-stage kernels."""
    from sphere_b200.engine import Engine, EngineError
    d = shear_stress_box(10)
    path = tmp_path / "wmode3.bin"
    binfile.write_bin(d, path)
    orc = O.Oracle(str(path), precision=precision)
    eng = Engine(str(path), precision=precision, graph_steps=8)
    for k, n in enumerate((1, 2, 9, 30)):
        assert eng.step(n) == 0
        assert orc.step(n) == 0, orc.error()
        bad = compare(eng, orc)
        assert not bad, f"after chunk {k}: {bad}"
    moved = eng.get("vel")[:, 0][d.fixvel > 0]
    assert numpy.abs(moved).max() > 0.0     # the stress moved the top layer
    eng.close()
    with pytest.raises(EngineError):
        Engine(str(path), precision=precision, step_kernel="persistent")
    with pytest.raises(EngineError):
        Engine(str(path), precision=precision, step_kernel="stages_fused")


def capillary_box(seed):
    """Model 1 (linear-viscous, no history) with capillary cohesion: pairs
    within db of contact attract by kappa sqrt(r_a r_b) exp(-delta/lambda)
    (capillaryCohesion_exp, src/cohesion.cuh:237-277)."""
    d = dense(seed, n=700, contactmodel=1)
    d.kappa = 0.05
    d.db = 0.002
    d.V_b = 1e-9
    d.gamma_n = 50.0
    return d


# CUDA's expf and glibc's (the oracle's) may round the capillary exponential
# differently in the last FP32 bit (CUDA's is documented within 2 ulp), so
# the capillary case compares the forces to 1e-6 of the largest force and
# the state to 1e-12 of its largest magnitude; the contact pairs must agree.
CAP_RTOL_F = 1e-6
CAP_RTOL_X = 1e-12


@pytest.mark.parametrize("precision", ["faithful", "fp64"])
@pytest.mark.parametrize("kernel", ["stages", "persistent", "stages_fused"])
def test_step_parity_capillary(tmp_path, precision, kernel):
    from sphere_b200.engine import Engine
    d = capillary_box(11)
    path = tmp_path / "capillary.bin"
    binfile.write_bin(d, path)
    orc = O.Oracle(str(path), precision=precision)
    eng = Engine(str(path), precision=precision, graph_steps=8, step_kernel=kernel)
    for k, n in enumerate((1, 2, 9, 20)):
        assert eng.step(n) == 0
        assert orc.step(n) == 0, orc.error()
        for f, tol in (("force", CAP_RTOL_F), ("torque", CAP_RTOL_F), ("x", CAP_RTOL_X),
                       ("vel", CAP_RTOL_F), ("angvel", CAP_RTOL_F)):
            a, b = eng.get(f)[:, :3], orc.get(f)[:, :3]
            scale = max(float(numpy.abs(b).max()), 1e-300)
            err = float(numpy.abs(a - b).max()) / scale
            assert err <= tol, f"after chunk {k}: {f} relative error {err:.3e}"
        assert numpy.array_equal(eng.get("index"), orc.get("index"))
    eng.close()
    # the cohesion acted: without it the first step's forces differ
    d0 = capillary_box(11)
    d0.kappa = 0.0
    path0 = tmp_path / "no_capillary.bin"
    binfile.write_bin(d0, path0)
    a, b = O.Oracle(str(path), precision=precision), O.Oracle(str(path0), precision=precision)
    assert a.step(1) == 0 and b.step(1) == 0
    assert not numpy.array_equal(a.get("force"), b.get("force"))
