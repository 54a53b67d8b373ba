"""CPU restatement of the reference's state diagnostics -- TEST
INFRASTRUCTURE ONLY (imported by tests/ as the checker of the engine's
device diagnostics; the product never imports it).

- energy(): sim.energy(method), python/sphere.py:4311-4380, the same numpy
  expressions on arrays in the reference's layout;
- porosity(): DEM::porosity, src/sphere.cpp:487-605 (slices from z = 0,
  the slice-height check against the LAST particle's radius because
  DEM::r_max returns it, sphere.cpp:474-484, and the "V_sphere + cap"
  branches as written);
- overlaps(): DEM::findOverlaps, src/sphere.cpp:677-725, the O(N^2) pair
  scan, vectorised per particle.

Pinned in tests/test_stats_oracle.py against the reference's own Python
sim.energy and against DEM::porosity / DEM::findOverlaps compiled for the
host (oracle/_ref).
"""
from __future__ import annotations

import math

import numpy

M_PI = math.pi


def energy(method, x4, vel4, angvel4, es, es_dot, ev, ev_dot, rho, g,
           bonds=None, bonds_delta=None, bonds_omega=None, lambda_bar=1.0, k_n=0.0, k_t=0.0):
    """sim.energy(method); vectors in Float4 rows (x, y, z, radius / fixvel)."""
    radius = x4[:, 3]
    np_ = len(radius)
    if method in ("pot", "kin", "rot"):
        m = numpy.ones(np_) * 4.0 / 3.0 * math.pi * radius ** 3 * rho
    if method == "pot":
        return numpy.sum(m * math.sqrt(numpy.dot(g, g)) * x4[:, 2])
    if method == "kin":
        v = vel4[:, :3]
        return float(numpy.sum(0.5 * m * numpy.sqrt(numpy.einsum("ij,ij->i", v, v)) ** 2))
    if method == "rot":
        w = angvel4[:, :3]
        return float(numpy.sum(0.5 * 2.0 / 5.0 * m * radius ** 2
                               * numpy.sqrt(numpy.einsum("ij,ij->i", w, w)) ** 2))
    if method == "shear":
        return numpy.sum(es)
    if method == "shearrate":
        return numpy.sum(es_dot)
    if method == "visc_n":
        return numpy.sum(ev)
    if method == "visc_n_rate":
        return numpy.sum(ev_dot)
    if method == "bondpot":
        if bonds is None or len(bonds) == 0:
            return 0.0
        bonds = numpy.asarray(bonds).reshape(-1, 2)
        R_bar = lambda_bar * numpy.minimum(radius[bonds[:, 0]], radius[bonds[:, 1]])
        A = numpy.pi * R_bar ** 2
        I = 0.25 * numpy.pi * R_bar ** 4
        J = I * 2.0
        delta_t, delta_n = bonds_delta[:, :3], bonds_delta[:, 3]
        omega_t, omega_n = bonds_omega[:, :3], bonds_omega[:, 3]
        fn = numpy.sum(0.5 * A * k_n * numpy.abs(delta_n) ** 2)
        ft = numpy.sum(0.5 * A * k_t * numpy.linalg.norm(delta_t) ** 2)
        tn = numpy.sum(0.5 * J * k_t * numpy.abs(omega_n) ** 2)
        tt = numpy.sum(0.5 * I * k_n * numpy.linalg.norm(omega_t) ** 2)
        return fn + ft + tn + tt
    raise ValueError(f'Unknownw energy() method "{method}"')


def spherical_cap(h, r):
    return M_PI * h * h / 3.0 * (3.0 * r - h)


class SliceError(ValueError):
    pass


def porosity(x4, top, origo_z, L, z_slices):
    """DEM::porosity: returns (z_pos, porosity) arrays of z_slices values."""
    h_slice = (top - origo_z) / float(z_slices)
    if h_slice <= x4[-1, 3] * 2.0:
        raise SliceError("Error! The number of z-slices is too high.")
    V_slice = h_slice * L[0] * L[1]
    c = x4[:, 2]
    radius = x4[:, 3]
    lo, hi = c - radius, c + radius
    V_sphere = 4.0 / 3.0 * M_PI * radius * radius * radius
    z_pos = numpy.zeros(z_slices)
    por = numpy.zeros(z_slices)
    for iz in range(z_slices):
        z_low = iz * h_slice
        z_high = z_low + h_slice
        inside = (z_low <= lo) & (hi <= z_high)
        sub = numpy.where(inside, V_sphere, 0.0)
        low_a = ~inside & (z_low >= c) & (z_low <= hi)
        low_b = ~inside & ~low_a & (z_low < c) & (z_low > lo)
        sub = sub + numpy.where(low_a, spherical_cap(hi - z_low, radius), 0.0)
        sub = sub + numpy.where(low_b, V_sphere + spherical_cap(z_low - lo, radius), 0.0)
        up_a = ~inside & (z_high <= c) & (z_high >= lo)
        up_b = ~inside & ~up_a & (z_high > c) & (z_high < hi)
        sub = sub + numpy.where(up_a, spherical_cap(z_high - lo, radius), 0.0)
        sub = sub + numpy.where(up_b, V_sphere + spherical_cap(hi - z_high, radius), 0.0)
        z_pos[iz] = z_low + 0.5 * h_slice
        por[iz] = (V_slice - numpy.sum(sub)) / V_slice
    return z_pos, por


def overlaps(x4, vel4):
    """DEM::findOverlaps: pairs (M x 2 uint32, i < j, i then j ascending)
    and separations |x_j - x_i| - (r_i + r_j) < 0 of pairs whose fixvel
    flags are both zero."""
    n = len(x4)
    pairs, deltas = [], []
    free = vel4[:, 3] == 0
    for i in range(n - 1):
        if not free[i]:
            continue
        xj = x4[i + 1:]
        dx = xj[:, 0] - x4[i, 0]
        dy = xj[:, 1] - x4[i, 1]
        dz = xj[:, 2] - x4[i, 2]
        length = numpy.sqrt(dx * dx + dy * dy + dz * dz)
        d = length - (x4[i, 3] + xj[:, 3])
        hit = numpy.nonzero((d < 0.0) & free[i + 1:])[0]
        for h in hit:
            pairs.append((i, i + 1 + h))
            deltas.append(d[h])
    return (numpy.array(pairs, dtype=numpy.uint32).reshape(-1, 2),
            numpy.array(deltas, dtype=numpy.float64))
