"""sim.run() drop-in (python/sphere.py:4482-4540): install/uninstall, the
dry run (read + checkValues + report, no device), the real reference
``sim`` class patched by install(), and a full run on the GPU engine with
the reference's ``../input`` / ``../output`` layout."""
import os

import numpy
import pytest

from sphere_b200 import binfile, configs, sim as sphsim

from helpers import Count, import_reference_sphere


class FakeSim:
    """The part of sphere's ``sim`` that run() uses: ``sid``, ``fluid`` and
    ``writebin(folder='../input/', verbose=...)``."""

    def __init__(self, sid, data):
        self.sid = sid
        self.data = data
        self.fluid = bool(data.fluid)

    def writebin(self, folder="../input/", verbose=True):
        os.makedirs(folder, exist_ok=True)
        binfile.write_bin(self.data, os.path.join(folder, self.sid + ".bin"))

    def run(self, *a, **k):
        return "reference run"


@pytest.fixture
def in_python_dir(tmp_path, monkeypatch):
    """cwd = <root>/python with <root>/input present, like a user running
    sphere's scripts from its python/ folder."""
    py = tmp_path / "python"
    py.mkdir()
    (tmp_path / "input").mkdir()
    monkeypatch.chdir(py)
    return tmp_path


def test_install_uninstall():
    class S(FakeSim):
        pass
    sphsim.install(S)
    assert S.run is sphsim.run and S.run_reference(None) == "reference run"
    sphsim.install(S)                       # idempotent
    assert S.run_reference is not sphsim.run
    sphsim.uninstall(S)
    assert S.run(None) == "reference run" and not hasattr(S, "run_reference")


def test_dry_run_reports(in_python_dir, capsys):
    class S(FakeSim):
        pass
    sphsim.install(S)
    d = configs.settling_lattice(n=64, seed=1, nx=4, ny=4, nz=4)
    assert S("dry", d).run(dry=True) == 0
    out = capsys.readouterr().out
    assert "Number of particles:  np = 64" in out
    assert "Linear-elastic-visco-frictional" in out
    assert (in_python_dir / "input" / "dry.bin").exists()
    assert not (in_python_dir / "output").exists()


def test_dry_run_rejects_bad_input(in_python_dir, capsys):
    class S(FakeSim):
        pass
    sphsim.install(S)
    d = configs.settling_lattice(n=64, seed=1, nx=4, ny=4, nz=4)
    d.radius[3] = -1.0
    status = S("bad", d).run(dry=True)
    assert status < 0
    assert "Warning: the sphere run returned with status" in capsys.readouterr().out


def test_reference_sim_class_dry_run(in_python_dir, capsys):
    """The reference's own sim class, patched by install(): its writebin
    writes ../input/<sid>.bin and the dry run validates it."""
    sphere = import_reference_sphere()
    try:
        sphsim.install(sphere.sim)
        n = 50
        s = sphere.sim(np=n, sid="refdry")
        s.np = numpy.asarray(s.np).view(Count)
        rng = numpy.random.default_rng(3)
        s.radius[:] = rng.uniform(0.009, 0.011, n)
        s.x[:, :] = rng.uniform(0.05, 0.45, (n, 3))
        s.defineWorldBoundaries(L=[0.5, 0.5, 0.5])
        s.setYoungsModulus(7e8)
        s.initTemporal(total=1e-4, file_dt=1e-5)
        assert s.run(dry=True) == 0
        assert "Using Young's modulus" in capsys.readouterr().out
        assert (in_python_dir / "input" / "refdry.bin").exists()
    finally:
        sphsim.uninstall(sphere.sim)


@pytest.mark.gpu
def test_run_on_engine(in_python_dir):
    class S(FakeSim):
        pass
    sphsim.install(S)
    d = configs.settling_lattice(n=300, seed=2, nx=7, ny=7, nz=7, spacing=0.0195)
    dt = float(d.time_dt)
    d.time_total = 40 * dt
    d.time_file_dt = 10 * dt
    assert S("eng", d).run(verbose=False) == 0
    out = in_python_dir / "output"
    names = sorted(os.listdir(out))
    assert "eng.output00000.bin" in names and "eng.output00004.bin" in names
    assert "eng.status.dat" in names
    last = binfile.read_bin(str(out / "eng.output00004.bin"))
    assert last.time_step_count == 4
    assert abs(last.time_current - 40 * dt) < 1e-3 * dt
