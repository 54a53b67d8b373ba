"""Why the mixed mode keeps overlaps in FP64: positions stored as an FP64
cell origin plus an FP32 offset cannot resolve the overlaps of the dense
shear packing.

On the benchmark packing (100,000 settled spheres, E = 7e8 Pa) the median
overlap is a few times 1e-8 m, while an FP32 offset inside a 0.025 m cell
resolves about 2e-9 m.  The normal contact forces computed from such
positions (k_n = pi/2 E r_bar, the Young's-modulus law of
src/contactmodels.cuh:241-408) then differ from the FP64 ones by far more
than the 1e-5 force error the mixed mode is held to."""
import numpy
import pytest

from sphere_b200 import configs

FORCE_TOL = 1e-5


def _normal_forces(x, r, a, b, hit, kn):
    xab = x[a] - x[b]
    ln = numpy.sqrt((xab * xab).sum(1))
    delta = ln - (r[a] + r[b])
    n = xab / ln[:, None]
    fmag = numpy.where(hit, -kn * delta, 0.0)
    F = numpy.zeros_like(x)
    numpy.add.at(F, a, fmag[:, None] * n)
    numpy.add.at(F, b, -fmag[:, None] * n)
    return F, delta


def test_fp32_offsets_miss_the_force_bound():
    spatial = pytest.importorskip("scipy.spatial")
    d = configs.shear_benchmark(n=100000, seed=1)
    x = numpy.asarray(d.x, dtype=numpy.float64)
    r = numpy.asarray(d.radius, dtype=numpy.float64)
    cell = numpy.asarray(d.L) / numpy.asarray(d.num)
    pairs = spatial.cKDTree(x).query_pairs(2.0 * r.max(), output_type="ndarray")
    a, b = pairs[:, 0], pairs[:, 1]
    xab = x[a] - x[b]
    hit = numpy.sqrt((xab * xab).sum(1)) - (r[a] + r[b]) < 0.0
    assert hit.sum() > 100000
    kn = numpy.pi / 2.0 * float(d.E) * (r[a] + r[b]) / 2.0
    F, delta = _normal_forces(x, r, a, b, hit, kn)
    # FP64 origin of the particle's cell plus the FP32 offset inside it
    origin = numpy.floor(x / cell) * cell
    xq = origin + (x - origin).astype(numpy.float32).astype(numpy.float64)
    Fq, _ = _normal_forces(xq, r, a, b, hit, kn)
    err = float(numpy.linalg.norm(Fq - F) / numpy.linalg.norm(F))
    assert float(numpy.median(-delta[hit])) < 1e-7
    assert err > 100.0 * FORCE_TOL, err
