"""The large polydisperse cohesive packing (log-normal radii, bonds between
initial neighbours): a 2e5-sphere cut of the generator stepped by the
engine's faithful FP64 path and by the oracle, bit for bit, over enough
steps for contacts to form and bonds to strain; a few steps of the full
4e6-sphere system compared the same way; the mixed mode's force error
against FP64."""
import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("x", "vel", "angvel", "force", "torque", "contacts", "delta_t", "bonds", "bonds_delta",
          "bonds_omega")


def bits(a):
    return numpy.ascontiguousarray(a).view(numpy.uint8)


def compare(e, o):
    bad = []
    for f in FIELDS:
        a, b = e.get(f), o.get(f)
        if f in ("angvel", "force", "torque"):
            a, b = a[:, :3], b[:, :3]
        if a.shape != b.shape or not numpy.array_equal(bits(a), bits(b)):
            bad.append(f)
    return bad


def test_cut_matches_oracle(tmp_path):
    from sphere_b200.engine import Engine
    # fast initial velocities so contacts form within the compared steps
    d = configs.large_cohesive_packing(n=200_000, seed=7, v_max=1.0)
    assert d.nb0 > d.np
    path = tmp_path / "cut.bin"
    binfile.write_bin(d, path)
    orc = O.Oracle(str(path), precision="faithful")
    with Engine(str(path), precision="faithful") as e:
        for n in (1, 9, 50):
            assert e.step(n) == 0
            assert orc.step(n) == 0, orc.error()
            bad = compare(e, orc)
            assert not bad, f"after {n} more steps: {bad}"
        occupied = int((e.get("contacts") != d.np).sum())
        assert occupied > 100
        strained = int((numpy.abs(e.get("bonds_delta")[:, 3]) > 0).sum())
        assert strained > d.nb0 // 2


def test_full_system_first_steps(tmp_path):
    """Two steps of the full 4e6-sphere packing against the oracle."""
    from sphere_b200.engine import Engine
    d = configs.large_cohesive_packing()
    path = tmp_path / "full.bin"
    binfile.write_bin(d, path)
    orc = O.Oracle(str(path), precision="faithful")
    with Engine(str(path), precision="faithful") as e:
        assert e.step(2) == 0
        assert orc.step(2) == 0, orc.error()
        bad = compare(e, orc)
        assert not bad, bad


def test_mixed_force_error():
    from sphere_b200.engine import Engine
    d = configs.large_cohesive_packing(n=200_000, seed=8, v_max=1.0)
    out = {}
    for prec in ("fp64", "mixed"):
        with Engine(d, precision=prec) as e:
            assert e.step(20) == 0
            out[prec] = e.get("force")[:, :3]
    a, b = out["mixed"], out["fp64"]
    err = float(numpy.linalg.norm(a - b) / numpy.linalg.norm(b))
    assert err <= 1e-5, err


def test_step_paths_agree_on_the_shear_benchmark():
    """The benchmark box itself (1e5 spheres, dense shear, faithful FP64):
    300 DEM steps on the per-stage kernels and on the per-stage kernels with
    contacts and integration in one launch (the step path the autotuner
    picks there) end in bit-identical states, resorts and list rebuilds
    included; the oracle pins the per-stage kernels on the smaller cases."""
    from sphere_b200.engine import Engine
    d = configs.shear_benchmark(n=100_000, seed=1)
    names = ("x", "vel", "angvel", "angpos", "force", "torque", "acc", "angacc", "xyzsum",
             "es", "ev", "p", "index", "contacts", "delta_t", "walls_nx", "walls_mvfd", "iter")
    states = []
    for kernel in ("stages", "stages_fused"):
        with Engine(d, precision="faithful", graph_steps=50, step_kernel=kernel) as e:
            assert e.step(300) == 0
            states.append({f: e.get(f) for f in names})
            assert e.info().resorts > 0
    bad = [f for f in names if not numpy.array_equal(bits(states[0][f]), bits(states[1][f]))]
    assert not bad, bad
