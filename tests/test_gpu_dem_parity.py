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
@pytest.mark.parametrize("kernel", ["stages", "persistent"])
def test_step_parity(tmp_path, name, data, precision, kernel):
    """Both step paths -- the per-stage kernels and the fused persistent
    kernel -- against the oracle, bit for bit."""
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
    with Engine(str(path)) as eng:
        assert eng.step(2) == 0
