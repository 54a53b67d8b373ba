"""ctypes binding of the engine's C ABI (``include/sphere_b200.h``).

The library is ``sphere_b200/libsphere_b200.so``, built in-tree by
``sphere_b200/build.py``.  There is no fallback: if the library is missing
or a CUDA device is unavailable, opening an engine raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Union

import numpy

from . import binfile

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsphere_b200.so")

PREC = {"faithful": 0, "fp64": 1, "mixed": 2}

FIELDS = [
    "x", "vel", "angvel", "angpos", "force", "torque", "acc", "angacc", "xyzsum",
    "es_dot", "es", "ev_dot", "ev", "p", "cellid", "index", "cellstart", "cellend",
    "contacts", "delta_t", "distmod", "walls_nx", "walls_mvfd", "walls_acc", "iter",
    "time", "darcy_p", "darcy_phi", "darcy_dphi", "darcy_k", "darcy_v", "darcy_f_p",
    "darcy_iters", "darcy_iters_total", "darcy_iters_exact", "darcy_warm", "bonds", "bonds_delta", "bonds_omega",
    "velocity_state", "ns_epsilon", "ns_norm", "ns_v_face", "ns_f_d", "ns_f_v", "ns_f_sum",
]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
_VEC4 = {"x", "vel", "angvel", "angpos", "force", "torque", "acc", "angacc", "xyzsum",
         "delta_t", "distmod", "walls_nx", "walls_mvfd", "darcy_f_p", "bonds_delta",
         "bonds_omega", "ns_f_d", "ns_f_v", "ns_f_sum"}
_U32 = {"cellid", "index", "cellstart", "cellend", "contacts", "bonds"}
_I64 = {"iter", "velocity_state", "darcy_iters", "darcy_iters_total", "darcy_iters_exact", "darcy_warm"}

STATUS = {
    0: "ok", 1: "Darcy solve did not converge", -1: "file error", -2: "version",
    -3: "input check failed", -4: "CUDA error", -5: "particle outside the grid or a non-finite value",
    -6: "contact capacity exceeded", -7: "unsupported input", -8: "bad argument",
    -9: "device wait timed out",
}


class SphOpts(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_size_t), ("fluid", ctypes.c_int),
                ("device", ctypes.c_int), ("verbose", ctypes.c_int),
                ("precision", ctypes.c_int), ("integrator", ctypes.c_int),
                ("contact_capacity", ctypes.c_int), ("warm_start", ctypes.c_int),
                ("graph_steps", ctypes.c_int), ("output_dir", ctypes.c_char_p),
                ("step_kernel", ctypes.c_int), ("darcy_exact_stop", ctypes.c_int),
                ("inject_timeout", ctypes.c_int)]


# sph_opts.inject_timeout bits (SPH_INJECT_*)
INJECT = {"resort": 1, "persistent": 2, "darcy": 4, "ns": 8}


class SphInfo(ctypes.Structure):
    _fields_ = [("np", ctypes.c_uint32), ("nw", ctypes.c_uint32), ("nb0", ctypes.c_uint32),
                ("capacity", ctypes.c_uint32), ("num", ctypes.c_uint32 * 3),
                ("periodic", ctypes.c_int32), ("contactmodel", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("fluid", ctypes.c_int32),
                ("iter", ctypes.c_int64), ("time", ctypes.c_double),
                ("time_total", ctypes.c_double), ("dt", ctypes.c_double),
                ("file_dt", ctypes.c_double), ("step_count", ctypes.c_uint32),
                ("resorts", ctypes.c_int64), ("step_path", ctypes.c_int32),
                ("step_threads", ctypes.c_int32), ("step_grid", ctypes.c_int32),
                ("tuned", ctypes.c_int32)]


class SphProfile(ctypes.Structure):
    _fields_ = [("resort_ms", ctypes.c_double), ("contacts_ms", ctypes.c_double),
                ("bonds_ms", ctypes.c_double), ("fluid_ms", ctypes.c_double),
                ("integrate_ms", ctypes.c_double), ("step_ms", ctypes.c_double),
                ("steps", ctypes.c_uint64)]


class SphBatchConfig(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("group_size", ctypes.c_int), ("grid", ctypes.c_int),
                ("tuned", ctypes.c_int), ("ntrials", ctypes.c_int), ("graph", ctypes.c_int)]


class SphBatchTrial(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("group_size", ctypes.c_int), ("grid", ctypes.c_int),
                ("ms_per_step", ctypes.c_double)]


class EngineError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)} ({status}): {message}")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """Loads the engine library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m sphere_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    L.sph_default_opts.argtypes = [ctypes.POINTER(SphOpts)]
    L.sph_default_opts.restype = ctypes.c_int
    L.sph_open.argtypes = [ctypes.c_char_p, ctypes.POINTER(SphOpts), ctypes.POINTER(P)]
    L.sph_open_buffer.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(SphOpts),
                                  ctypes.c_char_p, ctypes.POINTER(P)]
    L.sph_run.argtypes = [P]
    L.sph_step.argtypes = [P, ctypes.c_uint64]
    L.sph_step_timed.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]
    L.sph_profile_steps.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(SphProfile)]
    L.sph_field_bytes.argtypes = [P, ctypes.c_int]
    L.sph_field_bytes.restype = ctypes.c_int64
    L.sph_get.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
    L.sph_set.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
    L.sph_write_bin.argtypes = [P, ctypes.c_char_p]
    L.sph_get_info.argtypes = [P, ctypes.POINTER(SphInfo)]
    L.sph_last_error.argtypes = [P]
    L.sph_last_error.restype = ctypes.c_char_p
    L.sph_open_error.restype = ctypes.c_char_p
    L.sph_check_file.argtypes = [ctypes.c_char_p, ctypes.c_int]
    L.sph_check_file.restype = ctypes.c_int
    L.sph_energy.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
    L.sph_time_sort.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.sph_render.argtypes = [P, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_uint32,
                             ctypes.c_uint32, ctypes.c_void_p]
    L.sph_porosity.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.sph_overlaps.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                               ctypes.POINTER(ctypes.c_uint64)]
    L.sph_close.argtypes = [P]
    L.sph_version.restype = ctypes.c_char_p
    # batches
    L.sph_open_batch_buffers.argtypes = [ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
                                         ctypes.POINTER(SphOpts), ctypes.POINTER(P)]
    L.sph_open_batch.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                 ctypes.POINTER(SphOpts), ctypes.POINTER(P)]
    L.sph_batch_open_error.restype = ctypes.c_char_p
    L.sph_batch_step.argtypes = [P, ctypes.c_uint64]
    L.sph_batch_step_timed.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]
    L.sph_batch_autotune.argtypes = [P, ctypes.c_uint64]
    L.sph_batch_size.argtypes = [P]
    L.sph_batch_field_bytes.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.sph_batch_field_bytes.restype = ctypes.c_int64
    L.sph_batch_get.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
    L.sph_batch_write_bin.argtypes = [P, ctypes.c_int, ctypes.c_char_p]
    L.sph_batch_get_config.argtypes = [P, ctypes.POINTER(SphBatchConfig)]
    L.sph_batch_get_trials.argtypes = [P, ctypes.POINTER(SphBatchTrial), ctypes.c_int]
    L.sph_batch_last_error.argtypes = [P]
    L.sph_batch_last_error.restype = ctypes.c_char_p
    L.sph_batch_close.argtypes = [P]
    # warm-start network
    L.sph_wsnet_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                   ctypes.POINTER(P)]
    L.sph_wsnet_set_params.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.sph_wsnet_get_params.argtypes = [P, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.sph_wsnet_forward.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
    L.sph_wsnet_gradients.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p]
    L.sph_wsnet_destroy.argtypes = [P]
    _lib = L
    return L


STEP_KERNEL = {"auto": 0, "stages": 1, "persistent": 2, "stages_staged": 3, "stages_fused": 4}


def make_opts(fluid=False, precision="faithful", integrator=3, capacity=32, device=-1,
              graph_steps=0, warm_start=False, verbose=False, output_dir=None,
              step_kernel="auto", darcy_exact_stop=False, inject_timeout=0) -> SphOpts:
    o = SphOpts()
    o.struct_size = ctypes.sizeof(SphOpts)
    rc = lib().sph_default_opts(ctypes.byref(o))
    if rc != 0:
        raise EngineError(rc, "sph_default_opts refused this build's sph_opts layout")
    o.fluid = int(bool(fluid))
    o.precision = PREC[precision] if isinstance(precision, str) else int(precision)
    o.integrator = int(integrator)
    o.contact_capacity = int(capacity)
    o.device = int(device)
    o.graph_steps = int(graph_steps)
    o.warm_start = int(warm_start) if not isinstance(warm_start, bool) else int(warm_start)
    o.verbose = int(bool(verbose))
    o.output_dir = os.fsencode(output_dir) if output_dir else None
    o.step_kernel = STEP_KERNEL[step_kernel] if isinstance(step_kernel, str) else int(step_kernel)
    o.darcy_exact_stop = int(bool(darcy_exact_stop))
    if isinstance(inject_timeout, str):
        inject_timeout = INJECT[inject_timeout]
    o.inject_timeout = int(inject_timeout)
    return o


class Engine:
    """One simulation on the GPU.

    ``source`` is a ``.bin`` path or a :class:`~sphere_b200.binfile.BinData`
    (serialised in memory).  Vector fields come back in the reference's
    Float4 layout, one row per particle in original order.
    """

    def __init__(self, source: Union[str, os.PathLike, binfile.BinData], fluid: Optional[bool] = None,
                 precision="faithful", integrator=3, capacity=32, device=-1, graph_steps=0,
                 warm_start=False, verbose=False, output_dir=None, sid=None, step_kernel="auto",
                 darcy_exact_stop=False, inject_timeout=0):
        L = lib()
        h = ctypes.c_void_p()
        extra = dict(darcy_exact_stop=darcy_exact_stop, inject_timeout=inject_timeout)
        if isinstance(source, binfile.BinData):
            fl = source.fluid if fluid is None else fluid
            self._opts = make_opts(fl, precision, integrator, capacity, device, graph_steps,
                                   warm_start, verbose, output_dir, step_kernel, **extra)
            buf = binfile.serialize_bin(source)
            rc = L.sph_open_buffer(buf, len(buf), ctypes.byref(self._opts),
                                   (sid or "unnamed").encode(), ctypes.byref(h))
        else:
            self._opts = make_opts(bool(fluid), precision, integrator, capacity, device,
                                   graph_steps, warm_start, verbose, output_dir, step_kernel,
                                   **extra)
            rc = L.sph_open(os.fsencode(source), ctypes.byref(self._opts), ctypes.byref(h))
        if rc < 0 or not h.value:
            raise EngineError(rc, L.sph_open_error().decode())
        self._h = h
        self.np = self.info().np

    def _check(self, rc):
        if rc < 0:
            raise EngineError(rc, lib().sph_last_error(self._h).decode())
        return rc

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().sph_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, n=1) -> int:
        return self._check(lib().sph_step(self._h, int(n)))

    def step_timed(self, n) -> float:
        """Advances n steps; returns their device time in ms (CUDA events on
        the engine's stream)."""
        ms = ctypes.c_double(0.0)
        self._check(lib().sph_step_timed(self._h, int(n), ctypes.byref(ms)))
        return ms.value

    def profile(self, n) -> SphProfile:
        """Per-stage device time per DEM step over n eager steps."""
        p = SphProfile()
        self._check(lib().sph_profile_steps(self._h, int(n), ctypes.byref(p)))
        return p

    def run(self) -> int:
        return self._check(lib().sph_run(self._h))

    def info(self) -> SphInfo:
        inf = SphInfo()
        self._check(lib().sph_get_info(self._h, ctypes.byref(inf)))
        return inf

    def field_bytes(self, name) -> int:
        return int(lib().sph_field_bytes(self._h, FIELD_ID[name]))

    def get(self, name, out: Optional[numpy.ndarray] = None) -> numpy.ndarray:
        nbytes = self.field_bytes(name)
        if name in _VEC4:
            dtype, shape = numpy.float64, (nbytes // 32, 4)
        elif name in _U32:
            dtype, shape = numpy.uint32, (nbytes // 4,)
        elif name in _I64:
            dtype, shape = numpy.int64, (nbytes // 8,)
        elif name in ("darcy_v", "ns_v_face"):
            dtype, shape = numpy.float64, (nbytes // 24, 3)
        else:
            dtype, shape = numpy.float64, (nbytes // 8,)
        if out is None:
            out = numpy.empty(shape, dtype=dtype)
        self._check(lib().sph_get(self._h, FIELD_ID[name], out.ctypes.data, out.nbytes))
        return out

    def set(self, name, arr: numpy.ndarray) -> None:
        arr = numpy.ascontiguousarray(arr)
        self._check(lib().sph_set(self._h, FIELD_ID[name], arr.ctypes.data, arr.nbytes))

    def write_bin(self, path) -> None:
        self._check(lib().sph_write_bin(self._h, os.fsencode(path)))

    def time_sort(self, reps=5) -> float:
        """Device time in ms of one forced cell hash + sort + reorder."""
        ms = ctypes.c_double(0.0)
        self._check(lib().sph_time_sort(self._h, int(reps), ctypes.byref(ms)))
        return ms.value

    # diagnostics of sphere's sim class, computed on the device

    def energy(self, method) -> float:
        """sim.energy(method) (python/sphere.py:4311-4380): 'pot', 'kin',
        'rot', 'shear', 'shearrate', 'visc_n', 'visc_n_rate' or 'bondpot'."""
        out = ctypes.c_double(0.0)
        self._check(lib().sph_energy(self._h, str(method).encode(), ctypes.byref(out)))
        return out.value

    def porosity(self, slices=10):
        """sim.porosity(slices) (python/sphere.py:4437-4480): returns
        (porosity, depth), one value per horizontal slab."""
        z = numpy.empty(int(slices), dtype=numpy.float64)
        phi = numpy.empty(int(slices), dtype=numpy.float64)
        self._check(lib().sph_porosity(self._h, int(slices), z.ctypes.data, phi.ctypes.data))
        return phi, z

    def render(self, method=1, max_val=1.0e3, lower_cutoff=0.0, width=800, height=800):
        """Ray-traced image of the current state (``sphere --render``,
        src/raytracer.cuh): a (height, width, 4) uint8 RGBA array, row j
        holding pixels i + j * width."""
        img = numpy.empty((int(height), int(width), 4), dtype=numpy.uint8)
        self._check(lib().sph_render(self._h, int(method), float(max_val), float(lower_cutoff),
                                     int(width), int(height), img.ctypes.data))
        return img

    def find_overlaps(self):
        """sim.findOverlaps() (python/sphere.py:4868-4883): returns (pairs,
        overlaps), pairs a 2 x M int32 array of particle indices (i < j) and
        overlaps the M negative separations, in the order `sphere
        --contacts` prints them."""
        L = lib()
        count = ctypes.c_uint64(0)
        self._check(L.sph_overlaps(self._h, None, None, 0, ctypes.byref(count)))
        m = int(count.value)
        pairs = numpy.empty((m, 2), dtype=numpy.uint32)
        delta = numpy.empty(m, dtype=numpy.float64)
        if m:
            self._check(L.sph_overlaps(self._h, pairs.ctypes.data, delta.ctypes.data, m,
                                       ctypes.byref(count)))
        return numpy.ascontiguousarray(pairs.T.astype(numpy.int32)), delta

    def coordination_number(self):
        """Contacts per particle (sim.findCoordinationNumber,
        python/sphere.py:4885-4894) from the overlap list."""
        pairs, _ = self.find_overlaps()
        return (numpy.bincount(pairs[0], minlength=self.np)
                + numpy.bincount(pairs[1], minlength=self.np))


def write_ppm(path, img):
    """Writes an RGBA image as a binary PPM (P6, the RGB channels), pixels in
    the order DEM::writePPM writes them (src/file_io.cpp:734-757)."""
    img = numpy.ascontiguousarray(img)
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(f"P6 {w} {h} 255\n".encode())
        f.write(img[:, :, :3].tobytes())


def check_file(path, fluid=False):
    """Reads and validates a .bin file without the device (``sphere --dry``).
    Returns (status, message)."""
    L = lib()
    rc = L.sph_check_file(os.fsencode(path), int(bool(fluid)))
    return rc, (L.sph_open_error().decode() if rc else "")


def _shape_of(name, nbytes):
    if name in _VEC4:
        return numpy.float64, (nbytes // 32, 4)
    if name in _U32:
        return numpy.uint32, (nbytes // 4,)
    if name in _I64:
        return numpy.int64, (nbytes // 8,)
    if name in ("darcy_v", "ns_v_face"):
        return numpy.float64, (nbytes // 24, 3)
    return numpy.float64, (nbytes // 8,)


class Batch:
    """Many independent dry boxes stepped by one launch of the fused
    persistent step kernel (``sph_open_batch``).  ``boxes`` are
    :class:`~sphere_b200.binfile.BinData` objects or .bin paths."""

    def __init__(self, boxes, precision="mixed", integrator=3, capacity=32, device=-1):
        L = lib()
        self._opts = make_opts(False, precision, integrator, capacity, device)
        bufs = [binfile.serialize_bin(b) if isinstance(b, binfile.BinData)
                else open(b, "rb").read() for b in boxes]
        n = len(bufs)
        self._keep = [ctypes.create_string_buffer(b, len(b)) for b in bufs]
        ptrs = (ctypes.c_void_p * n)(*[ctypes.cast(k, ctypes.c_void_p) for k in self._keep])
        sizes = (ctypes.c_size_t * n)(*[len(b) for b in bufs])
        h = ctypes.c_void_p()
        rc = L.sph_open_batch_buffers(ptrs, sizes, n, ctypes.byref(self._opts), ctypes.byref(h))
        self._keep = None
        if rc < 0 or not h.value:
            raise EngineError(rc, L.sph_batch_open_error().decode())
        self._h = h
        self.nbox = n

    def _check(self, rc):
        if rc < 0:
            raise EngineError(rc, lib().sph_batch_last_error(self._h).decode())
        return rc

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().sph_batch_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, n=1) -> int:
        return self._check(lib().sph_batch_step(self._h, int(n)))

    def step_timed(self, n) -> float:
        ms = ctypes.c_double(0.0)
        self._check(lib().sph_batch_step_timed(self._h, int(n), ctypes.byref(ms)))
        return ms.value

    def autotune(self, trial_steps=4) -> int:
        return self._check(lib().sph_batch_autotune(self._h, int(trial_steps)))

    def config(self) -> dict:
        c = SphBatchConfig()
        self._check(lib().sph_batch_get_config(self._h, ctypes.byref(c)))
        return {f: getattr(c, f) for f, _ in c._fields_}

    def trials(self) -> list:
        n = self._check(lib().sph_batch_get_trials(self._h, None, 0))
        arr = (SphBatchTrial * max(n, 1))()
        self._check(lib().sph_batch_get_trials(self._h, arr, n))
        return [{f: getattr(arr[i], f) for f, _ in SphBatchTrial._fields_} for i in range(n)]

    def get(self, box, name) -> numpy.ndarray:
        nbytes = int(lib().sph_batch_field_bytes(self._h, int(box), FIELD_ID[name]))
        dtype, shape = _shape_of(name, nbytes)
        out = numpy.empty(shape, dtype=dtype)
        self._check(lib().sph_batch_get(self._h, int(box), FIELD_ID[name], out.ctypes.data,
                                        out.nbytes))
        return out

    def write_bin(self, box, path) -> None:
        self._check(lib().sph_batch_write_bin(self._h, int(box), os.fsencode(path)))


class WSNet:
    """The Darcy warm-start network on its own (``sph_wsnet_*``): BF16
    tensor-core forward and backward on host arrays, for gradient checks."""

    def __init__(self, nx, ny, nz, seed=1):
        h = ctypes.c_void_p()
        rc = lib().sph_wsnet_create(int(nx), int(ny), int(nz), int(seed), ctypes.byref(h))
        if rc != 0:
            raise EngineError(rc, "could not create the warm-start network")
        self._h = h
        self.ncells = nx * ny * nz

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().sph_wsnet_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, layer, w, b):
        w = numpy.ascontiguousarray(w, dtype=numpy.float32)
        b = numpy.ascontiguousarray(b, dtype=numpy.float32)
        assert w.size == 27 * 256 and b.size == 16
        if lib().sph_wsnet_set_params(self._h, int(layer), w.ctypes.data, b.ctypes.data):
            raise EngineError(-4, "set_params failed")

    def get_params(self, layer):
        w = numpy.empty((27, 16, 16), dtype=numpy.float32)
        b = numpy.empty(16, dtype=numpy.float32)
        if lib().sph_wsnet_get_params(self._h, int(layer), w.ctypes.data, b.ctypes.data):
            raise EngineError(-4, "get_params failed")
        return w, b

    def forward(self, x4):
        x3 = numpy.ascontiguousarray(x4, dtype=numpy.float32)
        assert x3.size == 4 * self.ncells
        out = numpy.empty(self.ncells, dtype=numpy.float32)
        rc = lib().sph_wsnet_forward(self._h, x3.ctypes.data, out.ctypes.data)
        if rc:
            raise EngineError(rc, "forward failed")
        return out

    def gradients(self, x4, target, free):
        x3 = numpy.ascontiguousarray(x4, dtype=numpy.float32)
        assert x3.size == 4 * self.ncells
        target = numpy.ascontiguousarray(target, dtype=numpy.float32)
        free = numpy.ascontiguousarray(free, dtype=numpy.uint8)
        dw = numpy.empty((3, 27, 16, 16), dtype=numpy.float32)
        db = numpy.empty((3, 16), dtype=numpy.float32)
        rc = lib().sph_wsnet_gradients(self._h, x3.ctypes.data, target.ctypes.data,
                                       free.ctypes.data, dw.ctypes.data, db.ctypes.data)
        if rc:
            raise EngineError(rc, "gradients failed")
        return dw, db
