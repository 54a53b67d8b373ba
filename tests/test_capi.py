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


def documented_opts_class():
    """The _Opts class of the ctypes binding shown in INTEGRATION.md."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"class _Opts\(ctypes\.Structure\):.*?\n(    _fields_ = \[.*?\])\n", text, re.S)
    assert m, "INTEGRATION.md has no _Opts binding"
    ns = {"ctypes": ctypes}
    exec("class _Opts(ctypes.Structure):\n" + m.group(1) + "\n", ns)
    return ns["_Opts"]


def test_documented_binding_matches_the_library_struct():
    doc = documented_opts_class()
    assert [f[0] for f in doc._fields_] == [f[0] for f in engine.SphOpts._fields_]
    assert [f[1] for f in doc._fields_] == [f[1] for f in engine.SphOpts._fields_]
    assert ctypes.sizeof(doc) == ctypes.sizeof(engine.SphOpts)


class _ShortOpts(ctypes.Structure):
    """An older caller's sph_opts: the fields up to output_dir only."""
    _fields_ = engine.SphOpts._fields_[:10]


def test_default_opts_refuses_a_mismatched_struct_size():
    lib = engine.lib()
    short = _ShortOpts()
    short.struct_size = ctypes.sizeof(_ShortOpts)
    short.fluid = 7
    assert lib.sph_default_opts(ctypes.cast(ctypes.byref(short), ctypes.POINTER(engine.SphOpts))) == -8
    assert short.fluid == 7          # nothing was written
    full = engine.SphOpts()
    full.struct_size = ctypes.sizeof(engine.SphOpts)
    assert lib.sph_default_opts(ctypes.byref(full)) == 0
    assert full.contact_capacity == 32 and full.integrator == 3 and full.device == -1


def test_open_refuses_a_mismatched_struct_size(tmp_path):
    """The size check comes before the file or the device is touched."""
    lib = engine.lib()
    short = _ShortOpts()
    short.struct_size = ctypes.sizeof(_ShortOpts)
    h = ctypes.c_void_p()
    rc = lib.sph_open(str(tmp_path / "absent.bin").encode(),
                      ctypes.cast(ctypes.byref(short), ctypes.POINTER(engine.SphOpts)), ctypes.byref(h))
    assert rc == -8 and not h.value
    assert b"struct_size" in lib.sph_open_error()


def test_open_refuses_an_unknown_step_kernel(tmp_path):
    """step_kernel is checked before the device is touched: 0-4 are the
    automatic choice and the four step paths, anything else is an argument
    error."""
    from sphere_b200 import binfile, configs
    assert engine.STEP_KERNEL == {"auto": 0, "stages": 1, "persistent": 2, "stages_staged": 3,
                                  "stages_fused": 4}
    path = tmp_path / "two.bin"
    binfile.write_bin(configs.two_particle(z=(2.0, 6.0), vel0=0.0), path)
    lib = engine.lib()
    opts = engine.make_opts(step_kernel=5)
    h = ctypes.c_void_p()
    rc = lib.sph_open(str(path).encode(), ctypes.byref(opts), ctypes.byref(h))
    assert rc == -8 and not h.value
    assert b"step_kernel" in lib.sph_open_error()
