"""The batch engine (many boxes in one launch of the persistent step kernel)
against the oracle run box by box, bit for bit in the FP64 modes; mixed
precision against standalone engines (same kernel, same arithmetic); the
autotuner and the graph replay."""
import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("x", "vel", "angvel", "force", "torque", "contacts", "delta_t", "walls_nx",
          "walls_mvfd", "es", "ev", "p")
VEC3 = ("angvel", "force", "torque")


def _bits(a):
    return numpy.ascontiguousarray(a).view(numpy.uint8)


def boxes():
    """Uneven small boxes with different parameters, walls and grids."""
    out = []
    d = configs.settling_lattice(n=150, seed=31, nx=6, ny=6, nz=6, spacing=0.0195)
    out.append(d)
    d = configs.settling_lattice(n=420, seed=32, nx=8, ny=8, nz=8, spacing=0.0195)
    d.mu_s = d.mu_d = 0.35
    out.append(d)
    d = configs.settling_lattice(n=700, seed=33, nx=10, ny=10, nz=8, spacing=0.0195)
    configs.shear_setup(d, 0.05, 40e3)
    d.w_x[0] -= 0.003
    out.append(d)
    d = configs.settling_lattice(n=260, seed=34, nx=7, ny=7, nz=7, spacing=0.0195)
    d.periodic = 2
    d.gamma_n = 30.0
    out.append(d)
    d = configs.fcc_shear_box(500, 35, sigma0=80e3, shear_velocity=5e-4, mu=0.45)
    out.append(d)
    return out


def compare_box(batch, i, orc):
    bad = {}
    for f in FIELDS:
        a, b = batch.get(i, f), orc.get(f)
        if f in VEC3:
            a, b = a[:, :3], b[:, :3]
        if a.shape != b.shape:
            bad[f] = f"shape {a.shape} vs {b.shape}"
        elif a.size and not numpy.array_equal(_bits(a), _bits(b)):
            bad[f] = "differs"
    return bad


@pytest.mark.parametrize("precision", ["faithful", "fp64"])
def test_batch_matches_oracle_per_box(tmp_path, precision):
    from sphere_b200.engine import Batch
    ds = boxes()
    orcs = []
    for i, d in enumerate(ds):
        p = tmp_path / f"b{i}.bin"
        binfile.write_bin(d, p)
        orcs.append(O.Oracle(str(p), precision=precision))
    with Batch(ds, precision=precision) as batch:
        for n in (1, 4, 20):
            assert batch.step(n) == 0
            for i, orc in enumerate(orcs):
                assert orc.step(n) == 0, orc.error()
                bad = compare_box(batch, i, orc)
                assert not bad, f"box {i} after {n}: {bad}"
        assert batch.config()["tuned"] == 0


def test_batch_autotune_and_graph(tmp_path):
    """A long call tunes the launch on its first steps; all trials step the
    boxes exactly like the oracle; later calls of one length replay a graph."""
    from sphere_b200.engine import Batch
    ds = boxes()[:3]
    orcs = []
    for i, d in enumerate(ds):
        p = tmp_path / f"t{i}.bin"
        binfile.write_bin(d, p)
        orcs.append(O.Oracle(str(p), precision="faithful"))
    with Batch(ds, precision="faithful") as batch:
        assert batch.step(300) == 0
        cfg = batch.config()
        assert cfg["tuned"] == 1 and cfg["ntrials"] >= 6
        trials = batch.trials()
        assert len(trials) == cfg["ntrials"]
        assert all(t["ms_per_step"] > 0 for t in trials)
        assert batch.step(5) == 0
        assert batch.step(5) == 0
        for i, orc in enumerate(orcs):
            assert orc.step(310) == 0, orc.error()
            bad = compare_box(batch, i, orc)
            assert not bad, f"box {i}: {bad}"
        assert int(batch.get(0, "iter")[0]) == 310


def test_batch_mixed_equals_standalone_engines():
    """Mixed precision: a box stepped inside a batch equals the same box
    stepped alone on the persistent path (same kernel arithmetic)."""
    from sphere_b200.engine import Batch, Engine
    ds = boxes()
    with Batch(ds, precision="mixed") as batch:
        assert batch.step(30) == 0
        for i, d in enumerate(ds):
            with Engine(d, precision="mixed", step_kernel="persistent") as e:
                assert e.step(30) == 0
                for f in ("x", "vel", "force", "contacts"):
                    a, b = batch.get(i, f), e.get(f)
                    assert numpy.array_equal(_bits(a), _bits(b)), (i, f)
