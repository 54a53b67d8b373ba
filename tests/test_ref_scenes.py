"""The input files of the reference's invariant tests (tests/golden/ref_scenes):
intact, readable by the .bin codec, accepted by the engine library's input
checks (no device needed), and -- where the reference tree is present --
exactly what the reference's own ``sim`` class writes for those tests today."""
import hashlib
import os

import pytest

from sphere_b200 import binfile
from sphere_b200.engine import check_file

import oracle
import ref_scenes as R

NAMES = sorted(R.manifest())


def test_manifest_covers_every_reference_invariant_test():
    prefixes = {n.split("_")[0] for n in NAMES}
    assert prefixes == {"cm", "cmy", "wall", "wally", "io", "cfd", "dp", "fpi"}
    assert len(NAMES) == 42


@pytest.mark.parametrize("name", NAMES)
def test_scene_is_intact_and_valid(tmp_path, name):
    m = R.manifest()[name]
    data = R.scene_bytes(name)
    assert hashlib.sha256(data).hexdigest() == m["sha256"]
    d = binfile.parse_bin(data, fluid=m["fluid"])
    assert d.np == m["np"] and d.version == 2.15
    assert binfile.serialize_bin(d) == data
    path = str(tmp_path / (m["sid"] + ".bin"))
    with open(path, "wb") as f:
        f.write(data)
    rc, msg = check_file(path, m["fluid"])
    assert rc == 0, msg


@pytest.mark.skipif(oracle.ref_path("python") is None, reason="reference tree not present")
def test_scenes_match_the_reference_sim_class(tmp_path):
    """Re-running the generator against the reference's sphere.py gives the
    committed files byte for byte."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_ref_scenes", os.path.join(R.HERE, "golden", "make_ref_scenes.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    fresh = mod.main(out=str(tmp_path))
    committed = R.manifest()
    assert sorted(fresh) == NAMES
    for n in NAMES:
        assert fresh[n] == committed[n], n


def test_answers_follow_the_output_cadence():
    """answers.json holds one value per output file of the run, at the step
    counts the run loop's file clock gives for the scene's dt, file_dt and
    total time."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_ref_scene_answers", os.path.join(R.HERE, "golden", "make_ref_scene_answers.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    ans = R.answers()
    assert sorted(ans) == sorted(mod.SCENES)
    for name, a in ans.items():
        d = binfile.parse_bin(R.scene_bytes(name), fluid=True)
        steps, done = [], 0
        for n, output in mod.file_steps(float(d.time_dt), float(d.time_file_dt),
                                        float(d.time_total), float(d.time_current)):
            done += n
            if output:
                steps.append(done)
        assert steps == a["steps"] and len(a["mean_vz"]) == len(steps)
