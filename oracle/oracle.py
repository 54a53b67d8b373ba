"""ctypes access to the CPU oracle and to the host build of the reference.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker.  The product never
imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsphere_ref.so")
# The reference tree (read-only), where it is mounted: the host build of its
# kernels and the tests that read its files use it; machines without it skip
# them.  $SPHERE_REF_ROOT overrides the location.
REF_ROOT = os.environ.get("SPHERE_REF_ROOT", "/root/reference")


def ref_path(*parts):
    """Path of a file or directory of the reference tree, or None where the
    tree (or that entry) is absent."""
    p = os.path.join(REF_ROOT, *parts)
    return p if os.path.exists(p) else None

_FIELD4 = {"x", "vel", "angvel", "angpos", "force", "torque", "acc", "angacc",
           "xyzsum", "walls_nx", "walls_mvfd", "bonds_delta", "bonds_omega"}
_SLOT4 = {"delta_t", "distmod"}
_U32 = {"cellid", "index", "cellstart", "cellend", "contacts", "bonds"}


def build(ref: bool = True) -> None:
    """Compile liboracle.so and, when the reference sources exist, _ref."""
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so", "liboracle_powprod.so"])
    ref_dir = os.environ.get("REF_DIR") or ref_path("src")
    if ref and ref_dir and os.path.isdir(ref_dir):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF_DIR={ref_dir}"])


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run oracle.build())")
    return ctypes.CDLL(path)


_libs = {}
# the sensitivity probe (pow replaced by products in the Darcy block)
POWPROD_SO = os.path.join(HERE, "liboracle_powprod.so")


def lib(path=None):
    path = path or ORACLE_SO
    _lib = _libs.get(path)
    if _lib is None:
        _lib = _load(path)
        _libs[path] = _lib
        _lib.orc_load.restype = ctypes.c_void_p
        _lib.orc_load.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_int)]
        _lib.orc_free.argtypes = [ctypes.c_void_p]
        _lib.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        _lib.orc_step.restype = ctypes.c_int
        _lib.orc_error.argtypes = [ctypes.c_void_p]
        _lib.orc_error.restype = ctypes.c_char_p
        _lib.orc_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                 ctypes.c_void_p, ctypes.c_size_t]
        _lib.orc_get.restype = ctypes.c_int64
        _lib.orc_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                 ctypes.c_void_p, ctypes.c_size_t]
        _lib.orc_write_bin.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        for f in ("orc_np", "orc_nc", "orc_nw"):
            getattr(_lib, f).argtypes = [ctypes.c_void_p]
        for f in ("orc_stage_hash_sort_reorder", "orc_stage_topology",
                  "orc_stage_interact"):
            getattr(_lib, f).argtypes = [ctypes.c_void_p]
            getattr(_lib, f).restype = ctypes.c_int
    return _lib


def _shape(name, nbytes):
    if name in ("ns_f_d", "ns_f_p", "ns_f_v", "ns_f_sum"):
        return numpy.float64, (nbytes // 32, 4)
    if name in ("ns_nijac_last", "ns_nijac_total", "ns_converged"):
        return numpy.int64, (nbytes // 8,)
    if name in ("ns_v", "ns_F_pf", "ns_v_face"):
        return numpy.float64, (nbytes // 24, 3)
    if name in _FIELD4:
        return numpy.float64, (nbytes // 32, 4)
    if name in _SLOT4:
        return numpy.float64, (nbytes // 32, 4)
    if name in _U32:
        return numpy.uint32, (nbytes // 4,)
    if name in ("iter", "darcy_nijac_last", "darcy_nijac_total"):
        return numpy.int64, (nbytes // 8,)
    if name == "darcy_p_constant":
        return numpy.int32, (nbytes // 4,)
    return numpy.float64, (nbytes // 8,)


class OracleError(RuntimeError):
    pass


class Oracle:
    """The CPU oracle's state for one ``.bin`` input."""

    def __init__(self, path, fluid=False, precision="faithful", integrator=3, nc=32,
                 lib_path=None):
        status = ctypes.c_int(0)
        prec = {"faithful": 0, "fp64": 1, "true": 1}[precision]
        self._L = lib(lib_path)
        self._h = self._L.orc_load(os.fsencode(path), int(bool(fluid)), prec,
                                 int(integrator), int(nc), ctypes.byref(status))
        if not self._h:
            raise OracleError(f"orc_load failed with status {status.value}")

    def close(self):
        if self._h:
            self._L.orc_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        rc = self._L.orc_step(self._h, int(n))
        return rc

    def error(self):
        return self._L.orc_error(self._h).decode()

    def get(self, name):
        need = self._L.orc_get(self._h, name.encode(), None, 0)
        if need < 0:
            raise KeyError(name)
        dtype, shape = _shape(name, need)
        out = numpy.empty(shape, dtype=dtype)
        rc = self._L.orc_get(self._h, name.encode(), out.ctypes.data, out.nbytes)
        if rc != 0:
            raise OracleError(f"orc_get({name}) returned {rc}")
        return out

    def set(self, name, arr):
        arr = numpy.ascontiguousarray(arr)
        rc = self._L.orc_set(self._h, name.encode(), arr.ctypes.data, arr.nbytes)
        if rc != 0:
            raise OracleError(f"orc_set({name}) returned {rc}")

    def stage(self, which):
        fn = {"sort": self._L.orc_stage_hash_sort_reorder,
              "topology": self._L.orc_stage_topology,
              "interact": self._L.orc_stage_interact}[which]
        return fn(self._h)

    def write_bin(self, path):
        return self._L.orc_write_bin(self._h, os.fsencode(path))

    @property
    def np(self):
        return self._L.orc_np(self._h)

    @property
    def nc(self):
        return self._L.orc_nc(self._h)


_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = _load(REF_SO)
        _ref.ref_open.restype = ctypes.c_void_p
        _ref.ref_open.argtypes = [ctypes.c_char_p, ctypes.c_int]
        _ref.ref_step.argtypes = [ctypes.c_void_p, ctypes.c_long]
        _ref.ref_write.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        _ref.ref_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                 ctypes.c_void_p, ctypes.c_size_t]
        _ref.ref_get.restype = ctypes.c_long
        _ref.ref_close.argtypes = [ctypes.c_void_p]
        _ref.ref_porosity.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p]
        _ref.ref_porosity.restype = ctypes.c_long
        _ref.ref_overlaps.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_long]
        _ref.ref_overlaps.restype = ctypes.c_long
        _ref.ref_render.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p]
        _ref.ref_render.restype = ctypes.c_int
    return _ref


class Reference:
    """The reference's own kernels compiled for the host (oracle/_ref)."""

    def __init__(self, path, fluid=False):
        self._h = ref_lib().ref_open(os.fsencode(path), int(bool(fluid)))

    def step(self, n=1):
        return ref_lib().ref_step(self._h, int(n))

    def get(self, name):
        need = ref_lib().ref_get(self._h, name.encode(), None, 0)
        if need < 0:
            raise KeyError(name)
        dtype, shape = _shape(name, need)
        out = numpy.empty(shape, dtype=dtype)
        ref_lib().ref_get(self._h, name.encode(), out.ctypes.data, out.nbytes)
        return out

    def write_bin(self, path):
        return ref_lib().ref_write(self._h, os.fsencode(path))

    def porosity(self, slices):
        """DEM::porosity (the `porosity` program): (z_pos, porosity)."""
        z = numpy.zeros(slices)
        p = numpy.zeros(slices)
        n = ref_lib().ref_porosity(self._h, int(slices), z.ctypes.data, p.ctypes.data)
        if n != slices:
            raise OracleError(f"porosity printed {n} of {slices} lines")
        return z, p

    def render(self, method=1, max_val=1.0e3, lower_cutoff=0.0, width=800, height=800):
        """DEM::render's image of the current state (`sphere --render`):
        height x width x 4 bytes (RGBA; alpha untouched, 0)."""
        img = numpy.zeros((height, width, 4), dtype=numpy.uint8)
        rc = ref_lib().ref_render(self._h, int(method), float(max_val), float(lower_cutoff),
                                  int(width), int(height), img.ctypes.data)
        if rc != 0:
            raise OracleError(f"render method {method} not understood")
        return img

    def overlaps(self):
        """DEM::findOverlaps: (pairs M x 2, separations M)."""
        m = ref_lib().ref_overlaps(self._h, None, None, 0)
        pairs = numpy.zeros((m, 2), dtype=numpy.uint32)
        d = numpy.zeros(m)
        ref_lib().ref_overlaps(self._h, pairs.ctypes.data, d.ctypes.data, m)
        return pairs, d

    def close(self):
        if self._h:
            ref_lib().ref_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
