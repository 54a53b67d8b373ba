"""Shared helpers for the tests."""
import os
import sys
import types

import numpy
import pytest

import oracle

# the reference's python tree, read-only; present only where it is mounted
REF_PY = oracle.ref_path("python")

VEC3 = ("angvel", "angpos", "force", "torque", "xyzsum", "acc", "angacc")


def bits_equal(a, b):
    a = numpy.ascontiguousarray(a)
    b = numpy.ascontiguousarray(b)
    return a.shape == b.shape and numpy.array_equal(a.view(numpy.uint8), b.view(numpy.uint8))


def diff_report(name, a, b):
    a = numpy.asarray(a, dtype=float)
    b = numpy.asarray(b, dtype=float)
    if a.shape != b.shape:
        return f"{name}: shape {a.shape} vs {b.shape}"
    d = numpy.abs(a - b)
    i = int(numpy.nanargmax(d)) if d.size else 0
    return f"{name}: max abs diff {numpy.nanmax(d) if d.size else 0:.3e} at flat index {i}"


def compare_states(get_a, get_b, fields):
    """Bit-for-bit comparison of named fields; returns the mismatches."""
    bad = []
    for f in fields:
        a, b = get_a(f), get_b(f)
        if f in VEC3:
            a, b = a[:, :3], b[:, :3]
        if not bits_equal(a, b):
            bad.append(diff_report(f, a, b))
    return bad


def bonded_packing(configs, n=300, seed=21, spacing=0.0195, factor=1.05, max_bonds=None):
    """Small dense packing with parallel bonds between initial pairs closer
    than factor * (r_i + r_j).  max_bonds keeps the first bonds only: the
    reference's reader sizes the bond displacement arrays by np, not nb0
    (src/file_io.cpp:234-253), so inputs for the reference need nb0 <= np."""
    d = configs.settling_lattice(n=n, seed=seed, nx=7, ny=7, nz=7, spacing=spacing, steps=40)
    x, r = d.x, d.radius
    pairs = []
    for i in range(n):
        dist = numpy.sqrt(((x[i + 1:] - x[i]) ** 2).sum(axis=1))
        js = numpy.nonzero(dist < factor * (r[i + 1:] + r[i]))[0] + i + 1
        pairs.extend((i, int(j)) for j in js)
    if max_bonds is not None:
        pairs = pairs[:max_bonds]
    d.nb0 = len(pairs)
    d.bonds = numpy.array(pairs, dtype=numpy.uint32).reshape(-1, 2)
    d.bonds_delta_n = numpy.zeros(d.nb0)
    d.bonds_delta_t = numpy.zeros((d.nb0, 3))
    d.bonds_omega_n = numpy.zeros(d.nb0)
    d.bonds_omega_t = numpy.zeros((d.nb0, 3))
    d.lambda_bar = 1.0
    d.sigma_b = 1e5
    d.tau_b = numpy.inf
    d.k_n = 1e7
    return d


def import_reference_sphere():
    """Imports python/sphere.py read-only with stand-ins for what it needs
    but does not use here: matplotlib, and numpy.infty (NumPy 2)."""
    if not REF_PY or not os.path.isdir(REF_PY):
        pytest.skip("reference python tree not present")
    for m in ("matplotlib", "matplotlib.pyplot", "matplotlib.collections",
              "matplotlib.colors", "matplotlib.cm", "matplotlib.patches",
              "matplotlib.ticker", "matplotlib.font_manager"):
        sys.modules.setdefault(m, types.ModuleType(m))
    mpl = sys.modules["matplotlib"]
    mpl.use = lambda *a, **k: None
    mpl.rc = lambda *a, **k: None
    mpl.rcParams = {}
    sys.modules["matplotlib.font_manager"].FontProperties = object
    if not hasattr(numpy, "infty"):
        numpy.infty = numpy.inf
    sys.path.insert(0, REF_PY)
    try:
        import sphere
    finally:
        sys.path.remove(REF_PY)
    return sphere


class Count(numpy.ndarray):
    """1-element count arrays that work in range() (sphere.py predates NumPy 2)."""

    def __index__(self):
        return int(self[0])
