"""The resume side-car's file format, without a device: a fake engine
supplies the fields; round trip, magic, version and truncation checks."""
import struct
import types

import numpy
import pytest

from sphere_b200 import resume as R


class FakeEngine:
    def __init__(self, np_=5, cap=4, nw=1, seed=0):
        rng = numpy.random.default_rng(seed)
        self._info = types.SimpleNamespace(np=np_, capacity=cap, nw=nw)
        self.fields = {
            "contacts": rng.integers(0, np_ + 1, np_ * cap).astype(numpy.uint32),
            "distmod": rng.normal(size=(np_ * cap, 4)),
            "delta_t": rng.normal(size=(np_ * cap, 4)),
            "acc": rng.normal(size=(np_, 4)),
            "angacc": rng.normal(size=(np_, 4)),
            "walls_acc": rng.normal(size=nw),
            "iter": numpy.array([123], dtype=numpy.int64),
            "velocity_state": numpy.array([1], dtype=numpy.int64),
        }
        self.set_calls = {}

    def info(self):
        return self._info

    def get(self, name):
        return self.fields[name]

    def field_bytes(self, name):
        return self.fields[name].nbytes

    def set(self, name, arr):
        self.set_calls[name] = numpy.array(arr)


def test_round_trip(tmp_path):
    a, b = FakeEngine(seed=1), FakeEngine(seed=2)
    p = tmp_path / "s.resume"
    R.write_resume(a, p)
    R.apply_resume(b, R.read_resume(p))
    assert set(b.set_calls) == set(R.FIELDS)
    for name in R.FIELDS:
        assert numpy.array_equal(b.set_calls[name].ravel(), a.fields[name].ravel()), name
        assert b.set_calls[name].dtype == a.fields[name].dtype, name


def test_rejects_bad_files(tmp_path):
    a = FakeEngine()
    p = tmp_path / "s.resume"
    R.write_resume(a, p)
    raw = p.read_bytes()
    (tmp_path / "magic").write_bytes(b"X" + raw[1:])
    with pytest.raises(R.ResumeError, match="not a resume"):
        R.read_resume(tmp_path / "magic")
    bad_ver = raw[:12] + struct.pack("<I", 99) + raw[16:]
    (tmp_path / "ver").write_bytes(bad_ver)
    with pytest.raises(R.ResumeError, match="version"):
        R.read_resume(tmp_path / "ver")
    (tmp_path / "trunc").write_bytes(raw[:-3])
    with pytest.raises(R.ResumeError, match="truncated"):
        R.read_resume(tmp_path / "trunc")
    (tmp_path / "trail").write_bytes(raw + b"\0")
    with pytest.raises(R.ResumeError, match="trailing"):
        R.read_resume(tmp_path / "trail")
    with pytest.raises(R.ResumeError, match="does not match"):
        R.apply_resume(FakeEngine(np_=6), R.read_resume(p))
