"""Input checks of the C ABI (DEM::checkValues, src/sphere.cpp:145-345, and
the reader's version check, src/file_io.cpp:47-54) return status codes
instead of exiting.  These run before any device work, so no GPU is needed."""
import ctypes
import os

import numpy
import pytest

from sphere_b200 import binfile, configs, engine


def open_status(tmp_path, d=None, raw=None, **opt):
    path = str(tmp_path / "v.bin")
    if raw is None:
        binfile.write_bin(d, path)
    else:
        open(path, "wb").write(raw)
    L = engine.lib()
    h = ctypes.c_void_p()
    o = engine.make_opts(**opt)
    rc = L.sph_open(path.encode(), ctypes.byref(o), ctypes.byref(h))
    msg = L.sph_open_error().decode()
    if h.value:
        L.sph_close(h)
    return rc, msg


def base():
    return configs.settling_lattice(n=64, seed=1, nx=4, ny=4, nz=4)


def test_missing_file():
    L = engine.lib()
    h = ctypes.c_void_p()
    assert L.sph_open(b"/nonexistent/x.bin", None, ctypes.byref(h)) == -1


def test_wrong_version(tmp_path):
    raw = binfile.serialize_bin(base())
    rc, msg = open_status(tmp_path, raw=numpy.float64(2.11).tobytes() + raw[8:])
    assert rc == -2 and "2.11" in msg


def test_truncated(tmp_path):
    raw = binfile.serialize_bin(base())
    assert open_status(tmp_path, raw=raw[: len(raw) // 2])[0] == -1


def test_trailing_bytes_means_fluid_flag_mismatch(tmp_path):
    raw = binfile.serialize_bin(base())
    assert open_status(tmp_path, raw=raw + b"\x01\x00\x00\x00")[0] == -1


@pytest.mark.parametrize("mutate,needle", [
    (lambda d: d.radius.__setitem__(3, 0.0), "radius"),
    (lambda d: d.x.__setitem__((5, 0), numpy.nan), "NaN"),
    (lambda d: d.x.__setitem__((7, 2), 10.0), "outside"),
    (lambda d: setattr(d, "k_n", 0.0), "k_n"),
    (lambda d: setattr(d, "rho", -1.0), "rho"),
    (lambda d: setattr(d, "time_current", 1e9), "time"),
])
def test_value_checks(tmp_path, mutate, needle):
    d = base()
    mutate(d)
    rc, msg = open_status(tmp_path, d)
    assert rc == -3 and needle.lower() in msg.lower(), msg


def test_wall_below_particles(tmp_path):
    d = base()
    configs.add_top_wall(d, 1e4)
    d.w_x[0] = 0.0
    rc, msg = open_status(tmp_path, d)
    assert rc == -3 and "wall" in msg


def test_hertz_model_is_reported_unsupported(tmp_path):
    d = base()
    d.contactmodel = 3
    assert open_status(tmp_path, d)[0] == -7


def test_navier_stokes_fluid_density_is_checked(tmp_path):
    """checkValues for cfd_solver 0 (src/sphere.cpp:311-317): a fluid density
    that is not positive fails the value check."""
    d = base()
    configs.init_fluid_ns(d, rho_f=0.0)
    assert open_status(tmp_path, d, fluid=True)[0] == -3
