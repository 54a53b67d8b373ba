"""The renderer's CPU restatement (oracle/render_oracle.py) against the
reference's own ray-tracing kernels (src/raytracer.cuh, compiled for the
host in oracle/_ref), pixel for pixel, and on cases whose answer is known
without either: the camera basis, a single sphere seen on the optical axis,
the colour map's end points, the cut-off and fixed-particle rules."""
import math
import os

import numpy
import pytest

import oracle as O
import render_oracle as R

CASES = [(0, 1e3, 0.0), (1, 50.0, 0.0), (2, 0.05, 0.0), (3, 1.0, 0.0), (4, 1e-4, 0.0),
         (5, 1e-3, 0.0), (2, 0.05, 0.01)]


@pytest.mark.skipif(not O.ref_available(), reason="host build of the reference not present")
def test_oracle_matches_reference_kernels(tmp_path):
    """rayInitPerspective, rayIntersectSpheres and rayIntersectSpheresColormap
    of the reference, run one thread at a time on a stepped packing, give the
    restatement's image for every colouring method, square and tall images,
    with and without the cut-off."""
    from sphere_b200 import binfile, configs
    d = configs.settling_lattice(n=300, seed=101, nx=7, ny=7, nz=7, spacing=0.0195, steps=0)
    d.fixvel[:10] = 1.0
    path = os.path.join(str(tmp_path), "rt.bin")
    binfile.write_bin(d, path)
    ref = O.Reference(path)
    assert ref.step(60) == 0
    s = {k: ref.get(k) for k in ("x", "vel", "angvel", "xyzsum", "angpos", "p")}
    for method, max_val, cutoff in CASES:
        val = R.method_values(method, s["x"], s["vel"], s["angvel"], s["xyzsum"], s["angpos"],
                              s["p"])
        for w, h in ((64, 64), (48, 96)):
            img = ref.render(method, max_val, cutoff, w, h)
            want = R.render(s["x"], s["vel"], d.L, w, h, method=method, val=val,
                            max_val=max_val, lower_cutoff=cutoff)
            assert (want[:, :, :3] != 255).any()
            bad = numpy.argwhere((img[:, :, :3] != want[:, :, :3]).any(axis=2))
            assert len(bad) == 0, (method, w, h, bad[:5])
    ref.close()


def test_camera_basis():
    C = R.camera([1.0, 1.0, 1.0], [0.8, 0.8, 0.8], 64, 64)
    u, v, w = (numpy.array(C[k], dtype=float) for k in ("u", "v", "w"))
    for a in (u, v, w):
        assert abs(numpy.linalg.norm(a) - 1.0) < 1e-6
    assert abs(u @ v) < 1e-6 and abs(u @ w) < 1e-6 and abs(v @ w) < 1e-6
    eye = numpy.array(C["eye"], dtype=float)
    lookat = numpy.array([0.4, 0.4, 0.4])
    # w points from the look-at point back... the reference's w is -view / |view|
    assert numpy.allclose(w, -(eye - lookat) / numpy.linalg.norm(eye - lookat), atol=1e-6)
    assert abs(C["d"] - 0.8 * numpy.linalg.norm(eye - lookat)) < 1e-5


def test_single_sphere_on_the_axis():
    """A sphere at the look-at point is hit by the central rays; the central
    pixel's shade follows the Lambertian rule of the reference."""
    L = [1.0, 1.0, 1.0]
    # the look-at point is half the largest coordinates (from 0): a sphere
    # at the origin sits on the optical axis
    x4 = numpy.array([[0.0, 0.0, 0.0, 0.3]])
    vel4 = numpy.zeros((1, 4))
    img = R.render(x4, vel4, L, 65, 65)
    c = img[32, 32]
    assert not (c[:3] == 255).all()            # the centre hits the sphere
    assert (img[0, 0, :3] == 255).all()         # a corner does not
    # shade = 200 * max(0, n . light) + 50, times the channel weights
    C = R.camera(L, [0.0, 0.0, 0.0], 65, 65)
    eye = numpy.array(C["eye"], dtype=float)
    ctr = numpy.array([0.0, 0.0, 0.0])
    # ray through the pixel centre nearest the image centre
    w, u, v = (numpy.array(C[k], dtype=float) for k in ("w", "u", "v"))
    pl = C["plane"]
    pu = pl[0] + (pl[1] - pl[0]) * 32.5 / 65
    pv = pl[2] + (pl[3] - pl[2]) * 32.5 / 65
    d = -C["d"] * w + pu * u + pv * v
    ec = eye - ctr
    t = (-(d @ ec) - math.sqrt((d @ ec) ** 2 - (d @ d) * (ec @ ec - 0.3 ** 2))) / (d @ d)
    n = (eye + t * d - ctr)
    n /= numpy.linalg.norm(n)
    shade = 200.0 * max(0.0, n @ numpy.array(C["light"], dtype=float)) + 50.0
    assert abs(int(c[0]) - int(shade * 0.48)) <= 1
    assert abs(int(c[1]) - int(shade * 0.41)) <= 1
    assert abs(int(c[2]) - int(shade * 0.27)) <= 1


def test_colour_map_and_rules():
    r, g, b = R._cm(numpy.array([0.01, 0.99], dtype=numpy.float32))
    assert abs(r[0] - (0.209e-6 - 2.49e-4 + 0.03 + 0.0109)) < 1e-6
    assert g[1] == numpy.float32(min(1.0, -2.44 * 0.99 ** 2 + 2.15 * 0.99 + 0.369)) or abs(
        g[1] - (-2.44 * 0.99 ** 2 + 2.15 * 0.99 + 0.369)) < 1e-6
    L = [1.0, 1.0, 1.0]
    x4 = numpy.array([[0.0, 0.0, 0.0, 0.3]])
    vel4 = numpy.zeros((1, 4))
    val = numpy.array([500.0])
    on = R.render(x4, vel4, L, 33, 33, method=1, val=val, max_val=1e3)
    assert not (on[16, 16, :3] == 255).all()
    # below the cut-off: not drawn
    off = R.render(x4, vel4, L, 33, 33, method=1, val=val, max_val=1e3, lower_cutoff=600.0)
    assert (off[16, 16, :3] == 255).all()
    # fixed particles are grey (equal channels)
    vel4[0, 3] = 1.0
    grey = R.render(x4, vel4, L, 33, 33, method=1, val=val, max_val=1e3)
    assert grey[16, 16, 0] == grey[16, 16, 1] == grey[16, 16, 2]
