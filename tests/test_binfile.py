"""The .bin v2.15 codec: round trips, the reference's shipped fixtures,
upgrades from 2.11, truncation/version errors, and byte equality with the
reference's own Python writer (python/sphere.py:1355-1553) where the
reference tree is present."""
import os
import sys
import types

import numpy
import pytest

from sphere_b200 import binfile, configs

from helpers import Count as _Count, import_reference_sphere as _import_reference_sphere

import oracle

REF_OUT = oracle.ref_path("output") or ""


def test_roundtrip_dry():
    d = configs.settling_lattice(n=200, seed=3, nx=6, ny=6, nz=6)
    buf = binfile.serialize_bin(d)
    e = binfile.parse_bin(buf)
    assert binfile.serialize_bin(e) == buf
    assert e.np == 200 and numpy.array_equal(e.x, d.x)


def test_roundtrip_walls_bonds():
    d = configs.settling_lattice(n=150, seed=4, nx=6, ny=6, nz=6)
    configs.shear_setup(d, 1e-3, 20e3)
    d.nb0 = 3
    d.bonds = numpy.array([[0, 1], [2, 3], [4, 5]], dtype=numpy.uint32)
    d.bonds_delta_n = numpy.arange(3.0)
    d.bonds_delta_t = numpy.ones((3, 3))
    d.bonds_omega_n = -numpy.arange(3.0)
    d.bonds_omega_t = numpy.full((3, 3), 2.0)
    buf = binfile.serialize_bin(d)
    e = binfile.parse_bin(buf)
    assert binfile.serialize_bin(e) == buf
    assert e.nw == 1 and e.wmode[0] == 1 and e.nb0 == 3


def test_roundtrip_fluid():
    d = configs.settling_lattice(n=100, seed=5, nx=5, ny=5, nz=5)
    nx, ny, nz = (int(v) for v in d.num)
    d.fluid = True
    d.cfd_solver = 1
    d.mu = 1.797e-6
    rng = numpy.random.default_rng(0)
    d.v_f = rng.normal(size=(nx, ny, nz, 3))
    d.p_f = rng.normal(size=(nx, ny, nz))
    d.phi = rng.uniform(0.3, 0.6, size=(nx, ny, nz))
    d.dphi = numpy.zeros((nx, ny, nz))
    d.p_f_constant = numpy.zeros((nx, ny, nz), dtype=numpy.int32)
    d.p_f_constant[0, 1, 2] = 1
    d.f_p = numpy.zeros((d.np, 3))
    buf = binfile.serialize_bin(d)
    e = binfile.parse_bin(buf, fluid=True)
    assert binfile.serialize_bin(e) == buf
    assert numpy.array_equal(e.p_f, d.p_f) and e.p_f_constant[0, 1, 2] == 1
    # fluid auto-detection from the trailing byte count
    assert binfile.parse_bin(buf).fluid


def test_errors():
    d = configs.settling_lattice(n=50, seed=6, nx=4, ny=4, nz=4)
    buf = binfile.serialize_bin(d)
    with pytest.raises(binfile.BinFormatError):
        binfile.parse_bin(buf[:-10])
    with pytest.raises(binfile.BinFormatError):
        binfile.parse_bin(numpy.float64(2.14).tobytes() + buf[8:])
    with pytest.raises(binfile.BinFormatError):
        binfile.parse_bin(buf + b"\0\0\0\0", fluid=False)


@pytest.mark.skipif(not os.path.isdir(REF_OUT), reason="reference fixtures not present")
@pytest.mark.parametrize("name,np_expected", [("init-1e4.output00199.bin", 10000),
                                               ("cube-init.output00029.bin", 1000)])
def test_reference_fixtures_upgrade(tmp_path, name, np_expected):
    src = os.path.join(REF_OUT, name)
    dst = str(tmp_path / "up.bin")
    d = binfile.upgrade_to_215(src, dst)
    assert d.np == np_expected
    e = binfile.read_bin(dst)
    assert e.version == 2.15 and e.adaptive == 0 and e.E == 0.0
    assert numpy.array_equal(e.x, d.x) and numpy.array_equal(e.radius, d.radius)
    with pytest.raises(binfile.BinFormatError):
        binfile.read_bin(src)  # 2.11 is rejected like the reference does


def test_writer_matches_reference_python_writer(tmp_path):
    sphere = _import_reference_sphere()
    n = 40
    sim = sphere.sim(np=n, sid="codec")
    sim.np = numpy.asarray(sim.np).view(_Count)
    rng = numpy.random.default_rng(9)
    sim.radius[:] = rng.uniform(0.01, 0.02, n)
    sim.x[:, :] = rng.uniform(0.1, 0.9, (n, 3))
    sim.vel[:, :] = rng.normal(size=(n, 3))
    sim.defineWorldBoundaries(L=[1.0, 1.0, 1.0])
    sim.setYoungsModulus(7e8)
    sim.initTemporal(total=0.01, file_dt=0.001)
    sim.writebin(folder=str(tmp_path), verbose=False)
    ref_bytes = open(tmp_path / "codec.bin", "rb").read()
    d = binfile.parse_bin(ref_bytes)
    assert binfile.serialize_bin(d) == ref_bytes
    assert d.E == 7e8 and d.np == n
    assert d.time_dt == pytest.approx(configs.time_step(d), rel=0, abs=0)


def test_navier_stokes_block_reads_in_the_c_library(tmp_path):
    """A Navier-Stokes input passes the library's reader and value checks
    (no device needed), and a grid under 3 cells per axis is rejected."""
    from sphere_b200 import binfile, configs
    from sphere_b200.engine import check_file
    d = configs.settling_lattice(n=300, seed=61, nx=7, ny=7, nz=7, spacing=0.0195, steps=0)
    configs.init_fluid_ns(d, hydrostatic=True, bc_bot=1)
    path = str(tmp_path / "ns.bin")
    binfile.write_bin(d, path)
    rc, msg = check_file(path, fluid=True)
    assert rc == 0, msg
    back = binfile.read_bin(path, fluid=True)
    assert back.cfd_solver == 0 and back.bc_bot == 1 and back.bc_top == 0
    assert numpy.array_equal(back.p_f, d.p_f)
    small = d.copy()
    small.num = numpy.array([2, 7, 7], dtype=numpy.uint32)
    small.L = numpy.array(d.L, dtype=float)
    configs.init_fluid_ns(small)
    binfile.write_bin(small, str(tmp_path / "small.bin"))
    rc, msg = check_file(str(tmp_path / "small.bin"), fluid=True)
    assert rc != 0 and "3 cells" in msg
