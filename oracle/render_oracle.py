"""CPU restatement of the reference's renderer -- TEST INFRASTRUCTURE ONLY
(imported by tests/ as the checker of the engine's ray tracer; the product
never imports it).

Follows src/raytracer.cuh: DEM::render's camera (eye, look-at, image width)
and DEM::cameraInit (image plane, u/v/w basis, focal distance, light), the
per-pixel ray of rayInitPerspective, the sphere tests of
rayIntersectSpheres and rayIntersectSpheresColormap (first of equally near
hits, in particle order) and their Lambertian shading, and the colour map
of src/colorbar.h.  All of it is IEEE single precision, as numpy float32
evaluates it; vector lengths and normalisation use sqrt and a division
(the host form of the reference's vector helpers).

Parity is pinned against the reference's own kernels (rayInitPerspective,
rayIntersectSpheres, rayIntersectSpheresColormap of src/raytracer.cuh,
compiled for the host in oracle/_ref and run one thread at a time) and by
analytic cases, in tests/test_render_oracle.py.
"""
from __future__ import annotations

import numpy

F = numpy.float32


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _length(v):
    return numpy.sqrt(_dot(v, v))


def _normalize(v):
    inv = F(1.0) / numpy.sqrt(_dot(v, v))
    return (v[0] * inv, v[1] * inv, v[2] * inv)


def camera(L, x_max, width, height):
    """DEM::render + DEM::cameraInit; x_max = the largest particle
    coordinates (from 0)."""
    imgw = F(L[0] * numpy.float64(F(1.35)))
    lookat = (F(x_max[0]) / F(2.0), F(x_max[1]) / F(2.0), F(x_max[2]) / F(2.0))
    eye = (F(L[0] * numpy.float64(F(2.3))), F(L[1] * numpy.float64(F(-5.0))),
           F(L[2] * numpy.float64(F(1.3))))
    hw = F(height // width)
    plane = (F(-0.5) * imgw, F(0.5) * imgw, F(-0.5) * imgw * hw, F(0.5) * imgw * hw)
    view = (eye[0] - lookat[0], eye[1] - lookat[1], eye[2] - lookat[2])
    up = (F(0.0), F(0.0), F(1.0))
    lv = _length(view)
    w = (-view[0] / lv, -view[1] / lv, -view[2] / lv)
    cu = _cross(up, w)
    lc = _length(cu)
    u = (cu[0] / lc, cu[1] / lc, cu[2] / lc)
    v = _cross(w, u)
    d = lv * F(0.8)
    m1 = (F(-1.0) * eye[0], F(-1.0) * eye[1], F(-1.0) * eye[2])
    light = _normalize((m1[0] * F(1.0), m1[1] * F(0.2), m1[2] * F(0.6)))
    return dict(eye=eye, u=u, v=v, w=w, d=d, plane=plane, light=light)


def _cm(r):
    red = numpy.minimum(F(1.0), F(0.209) * r * r * r - F(2.49) * r * r + F(3.0) * r + F(0.0109))
    green = numpy.minimum(F(1.0), F(-2.44) * r * r + F(2.15) * r + F(0.369))
    blue = numpy.minimum(F(1.0), F(-2.21) * r * r + F(1.61) * r + F(0.573))
    return red, green, blue


def render(x4, vel4, L, width, height, method=0, val=None, max_val=1.0e3, lower_cutoff=0.0):
    """Image (height, width, 4) uint8 of spheres x4 (original order, rows
    x, y, z, r); val: the per-particle colour-map values (FP64) for methods
    1-5; vel4[:, 3] is fixvel."""
    x4 = numpy.asarray(x4, dtype=numpy.float64)
    np_ = len(x4)
    x_max = [max(0.0, float(x4[:, k].max())) if np_ else 0.0 for k in range(3)]
    C = camera(L, x_max, width, height)
    pixels = width * height
    mempos = numpy.arange(pixels, dtype=numpy.int64)
    i = (mempos % width).astype(F)
    j = (numpy.floor(mempos.astype(F) / F(width)).astype(numpy.int64) % width).astype(F)
    pl = C["plane"]
    p_u = pl[0] + (pl[1] - pl[0]) * (i + F(0.5)) / F(width)
    p_v = pl[2] + (pl[3] - pl[2]) * (j + F(0.5)) / F(height)
    nd = -C["d"]
    d = tuple(nd * C["w"][k] + p_u * C["u"][k] + p_v * C["v"][k] for k in range(3))
    e = C["eye"]
    tdist = numpy.full(pixels, F(1e10), dtype=F)
    n = [numpy.zeros(pixels, dtype=F) for _ in range(3)]
    hit = numpy.zeros(pixels, dtype=numpy.int64)
    cut = lower_cutoff > 0.0
    maxv = F(max_val)
    lowc = F(lower_cutoff)
    with numpy.errstate(invalid="ignore", divide="ignore"):
        for q in range(np_):
            c = (F(x4[q, 0]), F(x4[q, 1]), F(x4[q, 2]))
            R = F(x4[q, 3])
            ec = (e[0] - c[0], e[1] - c[1], e[2] - c[2])
            dec = _dot(d, ec)
            dd = _dot(d, d)
            ecec = _dot(ec, ec)
            Delta = (F(2.0) * dec) * (F(2.0) * dec) - F(4.0) * dd * (ecec - R * R)
            take = Delta > F(0.0)
            if method != 0 and cut:
                take &= (F(val[q]) > lowc) & (F(vel4[q, 3]) == F(0.0))
            if not take.any():
                continue
            mdec = _dot((-d[0], -d[1], -d[2]), ec)
            t = (mdec - numpy.sqrt(dec * dec - dd * (ecec - R * R))) / dd
            upd = take & (numpy.abs(t) < tdist)
            if not upd.any():
                continue
            p = tuple(e[k] + t * d[k] for k in range(3))
            nn = _normalize(tuple(F(2.0) * (p[k] - c[k]) for k in range(3)))
            tdist = numpy.where(upd, numpy.abs(t), tdist)
            for k in range(3):
                n[k] = numpy.where(upd, nn[k], n[k])
            hit = numpy.where(upd, q, hit)
    img = numpy.full((pixels, 4), 255, dtype=numpy.uint8)
    hitm = tdist < F(1e10)
    dotprod = numpy.maximum(F(0.0), _dot(n, C["light"]))
    shade = F(5.0) * F(40.0) * dotprod + F(10.0) * F(5.0)
    if method == 0:
        rgb = (shade * F(0.48), shade * F(0.41), shade * F(0.27))
    else:
        vv = numpy.asarray(val, dtype=numpy.float64)
        ratio = (vv[hit] / numpy.float64(maxv)).astype(F)
        ratio = numpy.where(ratio < F(0.01), F(0.01), ratio)
        ratio = numpy.where(ratio > F(0.99), F(0.99), ratio)
        r, g, b = _cm(ratio)
        grey = F(numpy.asarray(vel4)[hit, 3]) > F(0.0) if np_ else numpy.zeros(pixels, bool)
        r = numpy.where(grey, F(0.5), r)
        g = numpy.where(grey, F(0.5), g)
        b = numpy.where(grey, F(0.5), b)
        rgb = (shade * r, shade * g, shade * b)
    for k in range(3):
        img[hitm, k] = numpy.trunc(rgb[k][hitm]).astype(numpy.uint8)
    return img.reshape(height, width, 4)


def method_values(method, x4, vel4, angvel4, xyzsum4, angpos4, p):
    """The per-particle value each colour-map method draws (DEM::render)."""
    if method == 1:
        return numpy.asarray(p, dtype=numpy.float64)
    if method == 2:
        v = vel4
    elif method == 3:
        v = angvel4
    elif method == 4:
        return numpy.asarray(xyzsum4[:, 0], dtype=numpy.float64)
    elif method == 5:
        v = angpos4
    else:
        return numpy.zeros(len(x4))
    return numpy.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])
