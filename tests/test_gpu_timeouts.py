"""Bounded device waits that run out, without a GPU fault.

Every cooperative kernel of the engine waits on other blocks through bounded
polls (the cell re-sort's grid barrier, the fused step's group barrier, the
neighbour waits of the Darcy and Navier-Stokes Jacobi kernels).  With
sph_opts.inject_timeout the selected kernel's waits target a value that
nothing writes and give up after about a thousand polls: the kernel returns,
the call reports SPH_ERR_TIMEOUT (-9) and the GPU context stays usable.  Each
test then checks that an engine opened afterwards on the same device steps
exactly like one opened before the timeout (and, for the DEM, like the
oracle).
"""
import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O

pytestmark = pytest.mark.gpu

TIMEOUT = -9


def dem_box(seed=3):
    d = configs.settling_lattice(n=700, seed=seed, nx=10, ny=10, nz=8, spacing=0.0195, steps=100)
    configs.add_top_wall(d, 20e3)
    d.w_x[0] -= 0.003
    return d


def run_fields(make, steps, fields):
    eng = make()
    try:
        for n in steps:
            assert eng.step(n) >= 0
        return {f: numpy.array(eng.get(f), copy=True) for f in fields}
    finally:
        eng.close()


def same_bits(a, b):
    for f in a:
        x, y = numpy.ascontiguousarray(a[f]), numpy.ascontiguousarray(b[f])
        assert x.shape == y.shape and numpy.array_equal(x.view(numpy.uint8), y.view(numpy.uint8)), f


DEM_FIELDS = ("x", "vel", "angvel", "force", "contacts", "delta_t", "walls_nx")


def check_dem_after(tmp_path, d, before, step_kernel):
    from sphere_b200.engine import Engine
    after = run_fields(lambda: Engine(d, step_kernel=step_kernel), (3, 9), DEM_FIELDS)
    same_bits(before, after)
    path = str(tmp_path / "box.bin")
    binfile.write_bin(d, path)
    orc = O.Oracle(path)
    assert orc.step(12) == 0, orc.error()
    for f in ("x", "vel", "contacts", "delta_t"):
        a, b = after[f], orc.get(f)
        assert numpy.array_equal(numpy.ascontiguousarray(a).view(numpy.uint8),
                                 numpy.ascontiguousarray(b).view(numpy.uint8)), f


def test_resort_grid_barrier_timeout(tmp_path):
    """The initial cell sort at open runs the re-sort kernel: its first grid
    barrier gives up and the open fails with SPH_ERR_TIMEOUT."""
    from sphere_b200.engine import Engine, EngineError
    d = dem_box(3)
    before = run_fields(lambda: Engine(d, step_kernel="stages"), (3, 9), DEM_FIELDS)
    with pytest.raises(EngineError) as ei:
        Engine(d, step_kernel="stages", inject_timeout="resort")
    assert ei.value.status == TIMEOUT
    assert "timed out" in str(ei.value)
    check_dem_after(tmp_path, d, before, "stages")


def test_persistent_group_barrier_timeout(tmp_path):
    from sphere_b200.engine import Engine, EngineError
    d = dem_box(4)
    before = run_fields(lambda: Engine(d, step_kernel="persistent"), (3, 9), DEM_FIELDS)
    eng = Engine(d, step_kernel="persistent", inject_timeout="persistent")
    with pytest.raises(EngineError) as ei:
        eng.step(5)
    assert ei.value.status == TIMEOUT
    eng.close()
    check_dem_after(tmp_path, d, before, "persistent")


def darcy_box(seed=51):
    d = configs.settling_lattice(n=300, seed=seed, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    configs.add_top_wall(d, 10e3)
    d.w_x[0] -= 0.002
    configs.init_fluid_darcy(d, mu=1.797e-6, k_c=3.5e-13, tolerance=1e-8, maxiter=2000,
                             bottom_no_flow=True)
    return d


FLUID_FIELDS = ("darcy_p", "darcy_phi", "x", "vel", "force", "darcy_iters")


def test_darcy_jacobi_wait_timeout():
    from sphere_b200.engine import Engine, EngineError
    d = darcy_box()
    before = run_fields(lambda: Engine(d, fluid=True), (1, 2), FLUID_FIELDS)
    eng = Engine(d, fluid=True, inject_timeout="darcy")
    with pytest.raises(EngineError) as ei:
        eng.step(1)
    assert ei.value.status == TIMEOUT
    eng.close()
    after = run_fields(lambda: Engine(d, fluid=True), (1, 2), FLUID_FIELDS)
    same_bits(before, after)
    assert int(after["darcy_iters"][0]) > 10


def ns_box(seed=31):
    d = configs.settling_lattice(n=300, seed=seed, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    configs.init_fluid_ns(d, mu=8.9e-4, hydrostatic=True, tolerance=1e-6, maxiter=2000)
    return d


def test_ns_jacobi_barrier_timeout():
    from sphere_b200.engine import Engine, EngineError
    d = ns_box()
    before = run_fields(lambda: Engine(d, fluid=True), (1, 2), FLUID_FIELDS)
    eng = Engine(d, fluid=True, inject_timeout="ns")
    with pytest.raises(EngineError) as ei:
        eng.step(1)
    assert ei.value.status == TIMEOUT
    eng.close()
    after = run_fields(lambda: Engine(d, fluid=True), (1, 2), FLUID_FIELDS)
    same_bits(before, after)
