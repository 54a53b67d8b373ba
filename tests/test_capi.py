"""The C ABI library loads and exports every function include/sphere_b200.h
declares (no GPU needed)."""
import ctypes
import os
import re

from sphere_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "sphere_b200.h")).read()
    return sorted(set(re.findall(r"\b(sph_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = engine.lib()
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n


def test_version_string():
    v = engine.lib().sph_version().decode()
    assert "sm_100a" in v
