"""Mixed precision against true FP64 (the engine's fp64 mode, itself
bit-identical to the oracle's fp64 mode).

Force error is the normwise relative error over all particles,
||F_mixed - F_fp64||_2 / ||F_fp64||_2, after steps taken from the same
state; the tolerance 1e-5 is the target the mixed mode is built to."""
import numpy
import pytest

from sphere_b200 import configs
from helpers import bonded_packing  # noqa: F401  (shared helpers module)

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def rel(a, b):
    return float(numpy.linalg.norm(a - b) / numpy.linalg.norm(b))


def dense_shear(seed, n=2000):
    d = configs.settling_lattice(n=n, seed=seed, nx=14, ny=14, nz=12, spacing=0.0196, steps=50)
    configs.shear_setup(d, 1e-3, 20e3)
    d.w_x[0] -= 0.001
    d.E = 7e8
    d.time_dt = configs.time_step(d)
    return d


@pytest.mark.parametrize("seed", [41, 42])
def test_single_step_force_error(seed):
    from sphere_b200.engine import Engine
    d = dense_shear(seed)
    ref = Engine(d, precision="fp64")
    mix = Engine(d, precision="mixed")
    ref.step(1)
    mix.step(1)
    f_ref, f_mix = ref.get("force")[:, :3], mix.get("force")[:, :3]
    t_ref, t_mix = ref.get("torque")[:, :3], mix.get("torque")[:, :3]
    assert numpy.linalg.norm(f_ref) > 0
    assert rel(f_mix, f_ref) <= FORCE_TOL, rel(f_mix, f_ref)
    # identical contact sets: overlaps are FP64 in both modes
    assert numpy.array_equal(ref.get("contacts"), mix.get("contacts"))
    # torques come only from tangential forces: compare against the force scale
    scale = numpy.linalg.norm(f_ref) * float(numpy.mean(d.radius))
    assert numpy.linalg.norm(t_mix - t_ref) / scale <= FORCE_TOL


@pytest.mark.parametrize("step_kernel", ["auto", "stages_fused"])
def test_force_error_stays_small_over_100_steps(step_kernel):
    """Over 100 sheared steps, on the automatic step path and on the
    per-stage path with contacts and integration in one launch (whose mixed
    integration rounds with FMA contraction, like the persistent kernel's)."""
    from sphere_b200.engine import Engine
    d = dense_shear(43)
    ref = Engine(d, precision="fp64")
    mix = Engine(d, precision="mixed", step_kernel=step_kernel)
    for _ in range(4):
        ref.step(25)
        mix.step(25)
        e = rel(mix.get("force")[:, :3], ref.get("force")[:, :3])
        assert e <= 1e-4, e
        dx = numpy.abs(mix.get("x")[:, :3] - ref.get("x")[:, :3]).max()
        assert dx < 1e-9, dx


def test_mixed_step_from_reference_state_matches_fp64():
    """Fresh engines stepped from the same state after a shared history."""
    from sphere_b200.engine import Engine
    d = dense_shear(44)
    ref = Engine(d, precision="fp64")
    ref.step(50)
    state = {f: ref.get(f) for f in ("x", "vel", "angvel")}
    hist = ref.get("delta_t")
    rows = ref.get("contacts")
    mix = Engine(d, precision="mixed")
    ref2 = Engine(d, precision="fp64")
    for e in (mix, ref2):
        for f, v in state.items():
            e.set(f, v)
        e.set("contacts", rows)
        e.set("delta_t", hist)
        e.step(1)
    assert rel(mix.get("force")[:, :3], ref2.get("force")[:, :3]) <= FORCE_TOL


def test_staged_contact_kernel_mixed():
    """The staged-cell contact kernel (step_kernel 3) in mixed precision:
    the same contact sets as the list kernel and forces within the mixed
    mode's bound of FP64 (FP32 arithmetic may contract differently in the
    two kernels, so equality is not asked)."""
    from sphere_b200.engine import Engine
    d = dense_shear(43)
    ref = Engine(d, precision="fp64")
    lst = Engine(d, precision="mixed", step_kernel="stages")
    stg = Engine(d, precision="mixed", step_kernel="stages_staged")
    for e in (ref, lst, stg):
        assert e.step(20) == 0
    f_ref = ref.get("force")[:, :3]
    assert numpy.array_equal(lst.get("contacts"), stg.get("contacts"))
    assert rel(stg.get("force")[:, :3], f_ref) <= FORCE_TOL * 10
    assert rel(lst.get("force")[:, :3], f_ref) <= FORCE_TOL * 10
    for e in (ref, lst, stg):
        e.close()
