"""Error reporting of the step on the device, where the reference goes on
silently: a contact row that runs out of slots (src/contactsearch.cuh:298-299
writes past the particle's row) and a particle that leaves the grid (the
reference's hash then indexes outside its cell arrays).  Both stop the step
with a status and a message naming the particle; the engine closes cleanly
and a new engine on the same device steps normally.  An empty particle set
steps without error."""
import numpy
import pytest

from sphere_b200 import configs

pytestmark = pytest.mark.gpu


def dense(seed=91, n=600):
    return configs.settling_lattice(n=n, seed=seed, nx=10, ny=10, nz=8, spacing=0.0195, steps=100)


def test_capacity_overflow_is_reported():
    from sphere_b200.engine import Engine, EngineError
    d = dense()
    probe = Engine(d, capacity=32)
    assert probe.step(5) == 0
    rows = probe.get("contacts").reshape(d.np, -1)
    most = int((rows != d.np).sum(axis=1).max())
    probe.close()
    assert most >= 3
    for kernel in ("stages", "persistent", "stages_fused"):
        e = Engine(d, capacity=2, step_kernel=kernel)
        with pytest.raises(EngineError) as exc:
            e.step(5)
        assert exc.value.status == -6
        assert "particle" in str(exc.value)
        e.close()
    ok = Engine(d, capacity=32)
    assert ok.step(5) == 0
    ok.close()


def test_particle_leaving_the_grid_is_reported():
    from sphere_b200.engine import Engine, EngineError
    d = configs.two_particle(z=(2.0, 6.0), vel0=0.0)
    d.vel[1, 0] = 2000.0      # across the 10 m box (non-periodic) within the steps
    d.periodic = 0
    e = Engine(d)
    with pytest.raises(EngineError) as exc:
        e.step(2000)
    assert exc.value.status == -5
    assert "particle 1" in str(exc.value)
    e.close()
    ok = Engine(dense())
    assert ok.step(3) == 0
    ok.close()


def test_empty_particle_set_steps():
    from sphere_b200.engine import Engine
    d = configs.two_particle(z=(2.0, 6.0), vel0=0.0)
    d.np = 0
    for f in ("x", "radius", "xyzsum", "vel", "fixvel", "force", "angpos", "angvel", "torque",
              "es_dot", "es", "ev_dot", "ev", "p", "color"):
        setattr(d, f, getattr(d, f)[:0])
    with Engine(d) as e:
        assert e.step(10) == 0
        info = e.info()
        assert info.np == 0 and info.iter == 10
        assert abs(info.time - 10 * float(d.time_dt)) < 1e-9 * max(1.0, info.time)
