"""Long runs: past the first steps the mixed-precision and FP64 trajectories
separate (the dynamics is chaotic), so they are compared as ensemble
statistics -- kinetic energy, mean coordination number and the porosity
profile sampled over a long run of a settling packing -- rather than particle
by particle."""
import numpy
import pytest

from sphere_b200 import configs

pytestmark = pytest.mark.gpu


def sample_run(d, precision, chunks, per_chunk):
    from sphere_b200.engine import Engine
    ke, z, phi = [], [], []
    with Engine(d, precision=precision) as e:
        for _ in range(chunks):
            assert e.step(per_chunk) == 0
            ke.append(e.energy("kin"))
            z.append(float(numpy.mean(e.coordination_number())))
            phi.append(e.porosity(4)[0])
    return numpy.array(ke), numpy.array(z), numpy.array(phi)


def test_mixed_and_fp64_agree_as_ensembles():
    # a dense settling box: the lattice spacing is below the mean diameter,
    # so the packing starts compressed and keeps rearranging
    d = configs.settling_lattice(n=3000, seed=91, nx=15, ny=15, nz=14, spacing=0.0195)
    chunks, per_chunk = 20, 1000
    ke64, z64, phi64 = sample_run(d, "fp64", chunks, per_chunk)
    kem, zm, phim = sample_run(d, "mixed", chunks, per_chunk)
    h = chunks // 2
    print("kinetic energy", ke64[h:].mean(), kem[h:].mean(), "coordination", z64[h:].mean(),
          zm[h:].mean(), "porosity", phi64[h:].mean(axis=0), phim[h:].mean(axis=0))
    # contacts persist and the two runs have separated
    assert z64[h:].mean() > 0.3
    assert not numpy.array_equal(ke64, kem)
    # ensemble statistics over the second half agree
    assert abs(kem[h:].mean() - ke64[h:].mean()) <= 0.10 * ke64[h:].mean()
    assert abs(zm[h:].mean() - z64[h:].mean()) <= 0.05 * z64[h:].mean()
    assert numpy.allclose(phim[h:].mean(axis=0), phi64[h:].mean(axis=0), rtol=0.02, atol=0.005)
