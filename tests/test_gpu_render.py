"""The engine's ray tracer against the reference's own ray-tracing kernels
(compiled for the host in oracle/_ref) and against the renderer's CPU
restatement, pixel for pixel, for every colouring method, with and without
the cut-off, on a stepped packing; and the PPM writer."""
import os

import numpy
import pytest

from sphere_b200 import binfile, configs

import oracle as O
import render_oracle as R

pytestmark = pytest.mark.gpu


def state(e):
    return dict(x4=e.get("x"), vel4=e.get("vel"), angvel4=e.get("angvel"), xyzsum4=e.get("xyzsum"),
                angpos4=e.get("angpos"), p=e.get("p"))


@pytest.mark.parametrize("method,max_val,cutoff", [(0, 1e3, 0.0), (1, 50.0, 0.0), (2, 0.05, 0.0),
                                                    (3, 1.0, 0.0), (4, 1e-4, 0.0), (5, 1e-3, 0.0),
                                                    (2, 0.05, 0.01)])
def test_render_matches_oracle(method, max_val, cutoff):
    from sphere_b200.engine import Engine
    d = configs.settling_lattice(n=300, seed=101, nx=7, ny=7, nz=7, spacing=0.0195)
    d.fixvel[:10] = 1.0
    with Engine(d, precision="faithful") as e:
        assert e.step(60) == 0
        s = state(e)
        for w, h in ((64, 64), (48, 96)):
            img = e.render(method=method, max_val=max_val, lower_cutoff=cutoff, width=w, height=h)
            val = R.method_values(method, s["x4"], s["vel4"], s["angvel4"], s["xyzsum4"],
                                  s["angpos4"], s["p"])
            ref = R.render(s["x4"], s["vel4"], d.L, w, h, method=method, val=val, max_val=max_val,
                           lower_cutoff=cutoff)
            assert (ref[:, :, :3] != 255).any()          # spheres are in view
            bad = numpy.argwhere((img[:, :, :3] != ref[:, :, :3]).any(axis=2))
            assert len(bad) == 0, (w, h, bad[:5], img[tuple(bad[0])], ref[tuple(bad[0])])


@pytest.mark.skipif(not O.ref_available(), reason="host build of the reference not present")
def test_render_matches_reference_kernels(tmp_path):
    """The same packing stepped by the engine and by the reference's host
    build (bit-identical states), then rendered by each: identical images."""
    from sphere_b200.engine import Engine
    d = configs.settling_lattice(n=300, seed=101, nx=7, ny=7, nz=7, spacing=0.0195, steps=0)
    d.fixvel[:10] = 1.0
    path = os.path.join(str(tmp_path), "rt.bin")
    binfile.write_bin(d, path)
    ref = O.Reference(path)
    assert ref.step(60) == 0
    with Engine(path, precision="faithful") as e:
        assert e.step(60) == 0
        assert numpy.array_equal(e.get("x"), ref.get("x"))
        for method, max_val, cutoff in ((0, 1e3, 0.0), (1, 50.0, 0.0), (2, 0.05, 0.0),
                                        (3, 1.0, 0.0), (4, 1e-4, 0.0), (5, 1e-3, 0.0),
                                        (2, 0.05, 0.01)):
            for w, h in ((64, 64), (48, 96)):
                img = e.render(method=method, max_val=max_val, lower_cutoff=cutoff, width=w,
                               height=h)
                want = ref.render(method, max_val, cutoff, w, h)
                bad = numpy.argwhere((img[:, :, :3] != want[:, :, :3]).any(axis=2))
                assert len(bad) == 0, (method, w, h, bad[:5])
    ref.close()


def test_ppm(tmp_path):
    from sphere_b200.engine import Engine, write_ppm
    d = configs.settling_lattice(n=100, seed=102, nx=5, ny=5, nz=4, spacing=0.0195)
    with Engine(d) as e:
        img = e.render(method=0, width=40, height=40)
    p = tmp_path / "x.ppm"
    write_ppm(p, img)
    raw = p.read_bytes()
    assert raw.startswith(b"P6 40 40 255\n")
    assert raw[len(b"P6 40 40 255\n"):] == img[:, :, :3].tobytes()
