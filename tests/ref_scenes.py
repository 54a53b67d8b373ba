"""Access to the input files of the reference's invariant tests
(tests/golden/ref_scenes, written by the reference's own ``sim`` class, see
tests/golden/make_ref_scenes.py) and the reference tests' comparison rules.
"""
import gzip
import json
import os

import numpy

from sphere_b200 import binfile

HERE = os.path.dirname(os.path.abspath(__file__))
SCENES = os.path.join(HERE, "golden", "ref_scenes")


def manifest():
    with open(os.path.join(SCENES, "manifest.json")) as f:
        return json.load(f)


def answers():
    """The reference's own kernels' values for scenes whose reference test
    condition they do not meet themselves (tests/golden/make_ref_scene_answers.py)."""
    with open(os.path.join(SCENES, "answers.json")) as f:
        return json.load(f)


def scene_bytes(name):
    with gzip.open(os.path.join(SCENES, name + ".bin.gz"), "rb") as f:
        return f.read()


class SceneSim:
    """The part of sphere's ``sim`` that ``run()`` uses, carrying one scene:
    ``writebin`` puts the reference-written file at ``../input/<sid>.bin``."""

    def __init__(self, name):
        m = manifest()[name]
        self.name = name
        self.sid = m["sid"]
        self.fluid = m["fluid"]
        self.data = scene_bytes(name)

    def run(self, *a, **k):
        """Stands for the reference's run (its binary), which install()
        replaces."""
        raise RuntimeError("the reference binary is not part of this build")

    def writebin(self, folder="../input/", verbose=True):
        os.makedirs(folder, exist_ok=True)
        with open(os.path.join(folder, self.sid + ".bin"), "wb") as f:
            f.write(self.data)


def status(root, sid):
    """sim.status(): the last output file number in ../output/<sid>.status.dat
    (python/sphere.py:5179-5196)."""
    with open(os.path.join(root, "output", sid + ".status.dat")) as f:
        return int(f.read().split()[2])


def readstep(root, sid, step, fluid):
    return binfile.read_bin(os.path.join(root, "output", f"{sid}.output{step:05d}.bin"),
                            fluid=fluid)


def readlast(root, sid, fluid):
    return readstep(root, sid, status(root, sid), fluid)


def compare_floats(first, second, tolerance=1e-3):
    """pytestutils.compareFloats (tests/pytestutils.py:29-39): relative to
    the first value."""
    return abs((first - second) / first) < tolerance


# sim's energy bookkeeping (python/sphere.py:4219-4310): mass from the
# radius and density, moment of inertia 2/5 m r^2
def _mass(d):
    return 4.0 / 3.0 * numpy.pi * d.radius ** 3 * float(d.rho)


def total_kinetic(d):
    m = _mass(d)
    return float(sum(0.5 * m[i] * numpy.sqrt(numpy.dot(d.vel[i], d.vel[i])) ** 2
                     for i in range(d.np)))


def total_rotational(d):
    m = _mass(d)
    return float(sum(0.5 * (2.0 / 5.0 * m[i] * d.radius[i] ** 2)
                     * numpy.sqrt(numpy.dot(d.angvel[i], d.angvel[i])) ** 2
                     for i in range(d.np)))


def total_viscous(d):
    return float(numpy.sum(d.ev))


def total_frictional(d):
    return float(numpy.sum(d.es))
