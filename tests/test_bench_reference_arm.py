"""The benchmark's input and its CPU reference arm need no GPU.

The settled 100,000-sphere packing ships as a packaged fixture
(sphere_b200/data, written by `python -m sphere_b200.prepack --pack` from the
packing configs.settle_packing made on the GPU), so the dense-shear workload
is the same bytes on every machine and `bench.py --impl reference` times the
reference's own kernels built for the host (or the oracle where that build is
absent) without loading the engine library."""
import hashlib
import os
import subprocess
import sys

from sphere_b200 import binfile, configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SHEAR_SHA256 = "b940b05d1ed7f0bf"


def test_packaged_packing_gives_the_pinned_workload():
    d = configs.shear_benchmark(n=100000, seed=1)
    assert d.np == 100000
    digest = hashlib.sha256(binfile.serialize_bin(d)).hexdigest()
    assert digest.startswith(SHEAR_SHA256), digest


def test_reference_arm_never_loads_the_engine():
    code = (
        "import sys, types; sys.path.insert(0, %r); import bench\n"
        "a = types.SimpleNamespace(particles=100000, warmup=0, steps=1, ref_sample=1, gpus=1)\n"
        "out = bench.run_reference(a)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('engine-module', 'sphere_b200.engine' in sys.modules)\n"
        "print('engine-library', 'libsphere_b200.so' in maps)\n"
        "print('reference-library', 'libsphere_ref.so' in maps or 'liboracle.so' in maps)\n"
        "print('kind', out['cpu_baseline']['kind'])\n"
        "print('config', out['config']['dem_steps_per_step'])\n" % ROOT)
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT,
                       env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines() if " " in line)
    assert lines["engine-module"] == "False"
    assert lines["engine-library"] == "False"
    assert lines["reference-library"] == "True"
    import oracle as O
    assert lines["kind"] == ("reference" if O.ref_available() else "port")
    assert lines["config"] == "1"


def test_step_path_names():
    """The benchmark line names the step path the engine reports
    (sph_info.step_path)."""
    import types
    sys.path.insert(0, ROOT)
    import bench
    name = lambda p: bench.step_path_name(types.SimpleNamespace(step_path=p))  # noqa: E731
    assert name(0) == "per-stage"
    assert name(1) == "persistent"
    assert name(2) == "per-stage, contacts and integration in one launch"
