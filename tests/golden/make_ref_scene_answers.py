"""Runs the fluidisation scenes of the reference's
tests/cfd_tests_darcy_particles.py (ref_scenes/dp_fluidization_*.bin.gz) on the
reference's own kernels compiled for the host (oracle/_ref) and records, at
every output file of the run, the mean vertical particle velocity -- the
quantity that test checks.  Output: ref_scenes/answers.json.

The file cadence is DEM::startTime's (src/device.cu:845-2684): the file clock
advances by dt per step, a file is written when it reaches file_dt and is then
restarted; the run ends when the time passes time_total.  Writing the file
matters to the solver: the Darcy block zeroes dphi on every step that does
not end at a file output.

Run from the repository root after oracle.build(ref=True):
``python tests/golden/make_ref_scene_answers.py [scene ...]`` (about ten
minutes per scene on one core).
"""
import json
import os
import sys
import tempfile

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
import ref_scenes as R  # noqa: E402

SCENES = ("dp_fluidization_0.9", "dp_fluidization_2.0")
OUT = os.path.join(R.SCENES, "answers.json")


def file_steps(dt, file_dt, total, t0=0.0):
    """Steps between consecutive outputs, as the run loop counts them."""
    out = []
    t, fc = t0, 0.0
    while t <= total:
        n, output = 0, False
        while t <= total:
            t += dt
            fc += dt
            n += 1
            if fc >= file_dt:
                output = True
                break
        out.append((n, output))
        if output:
            fc = 0.0
    return out


def answer(name):
    from sphere_b200 import binfile
    d = binfile.parse_bin(R.scene_bytes(name), fluid=True)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "in.bin")
        with open(path, "wb") as f:
            f.write(R.scene_bytes(name))
        ref = O.Reference(path, fluid=True)
        res = {"steps": [], "mean_vz": []}
        done = 0
        for n, output in file_steps(float(d.time_dt), float(d.time_file_dt),
                                    float(d.time_total), float(d.time_current)):
            if ref.step(n) != 0:
                raise RuntimeError(f"{name}: reference step failed")
            done += n
            if output:
                ref.write_bin(os.path.join(td, "out.bin"))
                res["steps"].append(done)
                res["mean_vz"].append(float(numpy.mean(ref.get("vel")[:, 2])))
                print(name, done, res["mean_vz"][-1], flush=True)
        ref.close()
    return res


def main(names):
    out = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            out = json.load(f)
    for n in names:
        out[n] = answer(n)
        with open(OUT, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or SCENES)
