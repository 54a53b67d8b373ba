"""Device diagnostics (energies, porosity profile, overlap list) against the
diagnostics oracle evaluated on the same state read back from the engine,
and the engine's step results unchanged by the queries."""
import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O
import stats_oracle as SO

from helpers import bonded_packing

pytestmark = pytest.mark.gpu

METHODS = ("pot", "kin", "rot", "shear", "shearrate", "visc_n", "visc_n_rate")
# sums over particles in a different order than the reference's serial loop
RTOL = 1e-12


def engine_state(e):
    return dict(x4=e.get("x"), v4=e.get("vel"), w4=e.get("angvel"), es=e.get("es"),
                es_dot=e.get("es_dot"), ev=e.get("ev"), ev_dot=e.get("ev_dot"))


def oracle_energy(d, s, method, e=None):
    kw = {}
    if method == "bondpot":
        kw = dict(bonds=e.get("bonds").reshape(-1, 2), bonds_delta=e.get("bonds_delta"),
                  bonds_omega=e.get("bonds_omega"), lambda_bar=d.lambda_bar, k_n=d.k_n, k_t=d.k_t)
    return SO.energy(method, s["x4"], s["v4"], s["w4"], s["es"], s["es_dot"], s["ev"],
                     s["ev_dot"], d.rho, d.g, **kw)


def lattice(seed, walls):
    d = configs.settling_lattice(n=300, seed=seed, nx=7, ny=7, nz=7, spacing=0.0195)
    if walls:
        configs.add_top_wall(d, 10e3)
    d.fixvel[:5] = 1.0
    return d


@pytest.mark.parametrize("precision", ["faithful", "mixed"])
@pytest.mark.parametrize("walls", [False, True])
def test_diagnostics_match_oracle(tmp_path, precision, walls):
    from sphere_b200.engine import Engine
    d = lattice(61 + walls, walls)
    path = tmp_path / "s.bin"
    binfile.write_bin(d, path)
    with Engine(str(path), precision=precision) as e:
        assert e.step(30) == 0
        s = engine_state(e)
        for m in METHODS:
            got, want = e.energy(m), float(oracle_energy(d, s, m))
            assert got == pytest.approx(want, rel=RTOL, abs=1e-300), m
        assert e.energy("bondpot") == 0.0
        top = float(e.get("walls_nx")[0, 3]) if walls else float(d.L[2])
        for slices in (1, 3, 5):
            phi, z = e.porosity(slices)
            z_o, phi_o = SO.porosity(s["x4"], top, float(d.origo[2]), d.L, slices)
            assert numpy.array_equal(z, z_o)
            assert numpy.allclose(phi, phi_o, rtol=RTOL, atol=1e-14)
        pairs, delta = e.find_overlaps()
        pairs_o, delta_o = SO.overlaps(s["x4"], s["v4"])
        assert len(delta_o) > 50
        assert numpy.array_equal(pairs.T, pairs_o.astype(numpy.int32))
        assert numpy.array_equal(delta.view(numpy.uint64), delta_o.view(numpy.uint64))
        z = e.coordination_number()
        assert z.sum() == 2 * len(delta) and numpy.all(z[:5] == 0)


def test_queries_leave_the_run_unchanged(tmp_path):
    """Stepping with diagnostics in between gives the oracle's state bit for
    bit."""
    from sphere_b200.engine import Engine
    d = lattice(63, True)
    path = tmp_path / "q.bin"
    binfile.write_bin(d, path)
    orc = O.Oracle(str(path))
    with Engine(str(path)) as e:
        for _ in range(4):
            assert e.step(7) == 0
            e.energy("kin")
            e.porosity(4)
            e.find_overlaps()
        assert orc.step(28) == 0
        for f in ("x", "vel", "angvel", "force", "torque", "contacts", "delta_t"):
            a, b = e.get(f), orc.get(f)
            assert numpy.array_equal(numpy.ascontiguousarray(a).view(numpy.uint8),
                                     numpy.ascontiguousarray(b).view(numpy.uint8)), f


def test_bond_energy(tmp_path):
    from sphere_b200.engine import Engine
    d = bonded_packing(configs, n=300, seed=23)
    with Engine(d, precision="faithful", step_kernel="stages") as e:
        assert e.step(20) == 0
        s = engine_state(e)
        got = e.energy("bondpot")
        want = float(oracle_energy(d, s, "bondpot", e))
        assert want > 0
        assert got == pytest.approx(want, rel=RTOL)


def test_larger_packing_overlaps():
    """10,000 particles: the grid search finds exactly the O(N^2) list."""
    from sphere_b200.engine import Engine
    d = configs.settling_lattice(n=10000, seed=64, nx=22, ny=22, nz=21, spacing=0.0195)
    with Engine(d, precision="mixed") as e:
        assert e.step(40) == 0
        s = engine_state(e)
        pairs, delta = e.find_overlaps()
    pairs_o, delta_o = SO.overlaps(s["x4"], s["v4"])
    assert len(delta_o) > 1000
    assert numpy.array_equal(pairs.T, pairs_o.astype(numpy.int32))
    assert numpy.array_equal(delta, delta_o)


def test_errors(tmp_path):
    from sphere_b200.engine import Engine, EngineError
    d = lattice(65, False)
    with Engine(d) as e:
        with pytest.raises(EngineError, match="Unknown energy"):
            e.energy("nope")
        with pytest.raises(EngineError, match="z-slices is too high"):
            e.porosity(1000)
        assert e.step(3) == 0
