"""Exact resume: a run written as .bin + side-car and reopened continues bit
for bit like the uninterrupted run; from the .bin alone it does not (the
reference's restart loses the contact history and the Taylor
accelerations)."""
import numpy
import pytest

from sphere_b200 import binfile, configs
from sphere_b200 import resume as R

pytestmark = pytest.mark.gpu

FIELDS = ("x", "vel", "angvel", "force", "torque", "contacts", "delta_t", "acc", "angacc",
          "walls_nx", "walls_mvfd", "walls_acc", "es", "ev", "iter")


def bits(a):
    return numpy.ascontiguousarray(a).view(numpy.uint8)


def shear_box(seed):
    d = configs.settling_lattice(n=400, seed=seed, nx=8, ny=8, nz=8, spacing=0.0195)
    configs.shear_setup(d, 0.05, 40e3)
    d.w_x[0] -= 0.003
    return d


@pytest.mark.parametrize("precision", ["faithful", "mixed"])
@pytest.mark.parametrize("step_kernel", ["stages", "persistent", "stages_fused"])
def test_resume_is_exact(tmp_path, precision, step_kernel):
    from sphere_b200.engine import Engine
    d = shear_box(71)
    src = tmp_path / "start.bin"
    binfile.write_bin(d, src)
    kw = dict(precision=precision, step_kernel=step_kernel)
    mid = tmp_path / "mid.bin"
    with Engine(str(src), **kw) as a:
        assert a.step(15) == 0
        sc = R.write_bin_with_resume(a, mid)
        assert a.step(15) == 0
        want = {f: a.get(f) for f in FIELDS}
    assert numpy.count_nonzero(want["contacts"] != 400) > 100
    with R.open_resumed(mid, **kw) as b:
        assert int(b.get("iter")[0]) == 15
        assert b.step(15) == 0
        for f in FIELDS:
            assert numpy.array_equal(bits(b.get(f)), bits(want[f])), f
    # the .bin alone restarts the history: the run differs
    with Engine(str(mid), **kw) as c:
        assert c.step(15) == 0
        assert not numpy.array_equal(bits(c.get("x")), bits(want["x"]))
    # a side-car for another engine shape is refused
    state = R.read_resume(sc)
    with Engine(str(mid), capacity=16, **kw) as e2:
        with pytest.raises(R.ResumeError):
            R.apply_resume(e2, state)
