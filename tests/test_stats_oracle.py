"""The diagnostics oracle (oracle/stats_oracle.py) pinned against the
reference itself: sim.energy() of the reference's python/sphere.py for every
method, and DEM::porosity / DEM::findOverlaps of the reference's C++ built
for the host (oracle/_ref)."""
import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O
import stats_oracle as SO

from helpers import Count, bonded_packing, import_reference_sphere

METHODS = ("pot", "kin", "rot", "shear", "shearrate", "visc_n", "visc_n_rate", "bondpot")


def state_with_bonds(seed=5, n=120):
    d = bonded_packing(configs, n=n, seed=seed)
    rng = numpy.random.default_rng(seed)
    d.vel = rng.normal(0, 0.02, (n, 3))
    d.angvel = rng.normal(0, 0.5, (n, 3))
    d.es = rng.uniform(0, 1e-3, n)
    d.es_dot = rng.uniform(0, 1e-2, n)
    d.ev = rng.uniform(0, 1e-3, n)
    d.ev_dot = rng.uniform(0, 1e-2, n)
    d.bonds_delta_n = rng.normal(0, 1e-5, d.nb0)
    d.bonds_delta_t = rng.normal(0, 1e-5, (d.nb0, 3))
    d.bonds_omega_n = rng.normal(0, 1e-3, d.nb0)
    d.bonds_omega_t = rng.normal(0, 1e-3, (d.nb0, 3))
    return d


def oracle_energy(d, method):
    x4 = numpy.column_stack([d.x, d.radius])
    v4 = numpy.column_stack([d.vel, d.fixvel])
    w4 = numpy.column_stack([d.angvel, numpy.zeros(d.np)])
    bd = numpy.column_stack([d.bonds_delta_t, d.bonds_delta_n])
    bo = numpy.column_stack([d.bonds_omega_t, d.bonds_omega_n])
    return SO.energy(method, x4, v4, w4, d.es, d.es_dot, d.ev, d.ev_dot, d.rho, d.g,
                     d.bonds, bd, bo, d.lambda_bar, d.k_n, d.k_t)


def test_energy_matches_reference_python():
    sphere = import_reference_sphere()
    d = state_with_bonds()
    s = sphere.sim(np=d.np, sid="energy")
    s.np = numpy.asarray([d.np]).view(Count)
    s.radius = d.radius.copy()
    s.x = d.x.copy()
    s.vel = d.vel.copy()
    s.angvel = d.angvel.copy()
    for f in ("es", "es_dot", "ev", "ev_dot"):
        setattr(s, f, getattr(d, f).copy())
    s.rho = numpy.ones(1) * d.rho
    s.g = numpy.array(d.g)
    s.k_n = numpy.ones(1) * d.k_n
    s.k_t = numpy.ones(1) * d.k_t
    s.lambda_bar = numpy.ones(1) * d.lambda_bar
    s.nb0 = d.nb0
    s.bonds = d.bonds.astype(numpy.int64)
    s.bonds_delta_n = d.bonds_delta_n.copy()
    s.bonds_delta_t = d.bonds_delta_t.copy()
    s.bonds_omega_n = d.bonds_omega_n.copy()
    s.bonds_omega_t = d.bonds_omega_t.copy()
    for m in METHODS:
        want = float(numpy.asarray(s.energy(m)).ravel()[0])
        got = float(numpy.asarray(oracle_energy(d, m)).ravel()[0])
        assert got == pytest.approx(want, rel=1e-13, abs=0.0), m
    assert oracle_energy(d, "bondpot") > 0
    with pytest.raises(Exception):
        s.energy("nope")
    with pytest.raises(ValueError):
        oracle_energy(d, "nope")


def _ref_or_skip():
    if not O.ref_available():
        pytest.skip("host build of the reference (oracle/_ref) not present")


def settled_file(tmp_path, walls):
    d = configs.settling_lattice(n=300, seed=9, nx=7, ny=7, nz=7, spacing=0.0195)
    if walls:
        configs.add_top_wall(d, 10e3)
    d.fixvel[:5] = 1.0
    p = tmp_path / ("w.bin" if walls else "n.bin")
    binfile.write_bin(d, p)
    # a few reference steps so the packing has overlaps
    r = O.Reference(str(p))
    assert r.step(30) == 0
    out = tmp_path / ("w30.bin" if walls else "n30.bin")
    r.write_bin(str(out))
    r.close()
    return out


@pytest.mark.parametrize("walls", [False, True])
def test_porosity_and_overlaps_match_reference_cpp(tmp_path, walls):
    _ref_or_skip()
    path = settled_file(tmp_path, walls)
    d = binfile.read_bin(str(path))
    x4 = numpy.column_stack([d.x, d.radius])
    v4 = numpy.column_stack([d.vel, d.fixvel])
    r = O.Reference(str(path))
    top = float(d.w_x[0]) if d.nw > 0 else float(d.L[2])
    for slices in (1, 4, 7):
        z_ref, p_ref = r.porosity(slices)
        z, p = SO.porosity(x4, top, float(d.origo[2]), d.L, slices)
        # the reference prints 17 significant digits and sums serially
        assert numpy.allclose(z, z_ref, rtol=1e-15, atol=0)
        assert numpy.allclose(p, p_ref, rtol=1e-12, atol=1e-14)
    pairs_ref, d_ref = r.overlaps()
    pairs, dd = SO.overlaps(x4, v4)
    assert len(pairs_ref) > 50
    assert numpy.array_equal(pairs, pairs_ref)
    assert numpy.array_equal(dd.view(numpy.uint64), d_ref.view(numpy.uint64))
    r.close()


def test_porosity_slice_check_uses_last_radius():
    """DEM::r_max returns the last particle's radius: a large radius earlier
    in the list does not trip the slice-height check."""
    x4 = numpy.array([[0.5, 0.5, 0.5, 0.2], [0.5, 0.5, 0.2, 0.01]])
    z, p = SO.porosity(x4, 1.0, 0.0, [1.0, 1.0, 1.0], 3)   # h = 0.333 <= 0.4 = 2 r_max
    assert len(p) == 3
    with pytest.raises(SO.SliceError):
        SO.porosity(x4[::-1].copy(), 1.0, 0.0, [1.0, 1.0, 1.0], 3)


def test_porosity_single_sphere_cases():
    """One sphere, hand-computed: fully inside a slab, and crossing the
    boundary between two slabs (the reference's 'V_sphere + cap' branch)."""
    r = 0.1
    V = 4.0 / 3.0 * numpy.pi * r ** 3
    x4 = numpy.array([[0.5, 0.5, 0.25, r]])
    z, p = SO.porosity(x4, 1.0, 0.0, [1.0, 1.0, 1.0], 2)
    assert numpy.allclose(z, [0.25, 0.75])
    assert numpy.allclose(p, [(0.5 - V) / 0.5, 1.0])
    # centre 0.04 above the boundary z = 0.5
    x4 = numpy.array([[0.5, 0.5, 0.54, r]])
    z, p = SO.porosity(x4, 1.0, 0.0, [1.0, 1.0, 1.0], 2)
    cap_below = numpy.pi * 0.06 ** 2 / 3.0 * (3 * r - 0.06)
    assert p[0] == pytest.approx((0.5 - cap_below) / 0.5, rel=1e-12)
    assert p[1] == pytest.approx((0.5 - (V + cap_below)) / 0.5, rel=1e-12)
