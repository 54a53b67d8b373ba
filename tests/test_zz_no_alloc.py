"""sph_sort_cells_noalloc: the cell sort for callers that cannot allocate
device memory (a host application whose memory pool owns the GPU, or a
loop that must not call cudaMalloc/cudaFree because they synchronise the
device).  Its output must equal the engine's own sort (sph_open, then
sph_get of cellid/index/cellstart/cellend) exactly, on two calls in a row
that share the built-in scratch array."""
import ctypes

import numpy
import pytest

from sphere_b200 import configs, engine

pytestmark = pytest.mark.gpu


def engine_sort(d):
    with engine.Engine(d) as e:
        return (e.get("cellid"), e.get("index"), e.get("cellstart"), e.get("cellend"))


def _lib():
    L = engine.lib()
    L.sph_sort_cells_noalloc.argtypes = [
        ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double),
        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint32),
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.sph_noalloc_error.restype = ctypes.c_char_p
    return L


def noalloc_sort(d):
    import torch
    L = _lib()
    n = d.np
    ncells = int(d.num[0]) * int(d.num[1]) * int(d.num[2])
    x4 = numpy.column_stack([d.x, d.radius])
    dev = torch.device("cuda", 0)
    x4_d = torch.from_numpy(numpy.ascontiguousarray(x4)).to(dev)
    # the caller owns inputs and outputs; the entry point allocates nothing
    outs = [torch.full((m,), -7, dtype=torch.int32, device=dev) for m in (n, n, ncells, ncells)]
    origo = (ctypes.c_double * 3)(*d.origo)
    Lv = (ctypes.c_double * 3)(*d.L)
    num = (ctypes.c_uint32 * 3)(*(int(v) for v in d.num))
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.sph_sort_cells_noalloc(x4_d.data_ptr(), n, origo, Lv, num,
                                  *(o.data_ptr() for o in outs), stream)
    assert rc == 0, L.sph_noalloc_error().decode()
    return tuple(o.cpu().numpy().view(numpy.uint32) for o in outs)


def check(d):
    ref = engine_sort(d)
    got = noalloc_sort(d)
    for name, a, b in zip(("cellid", "index", "cellstart", "cellend"), got, ref):
        assert numpy.array_equal(a, b), name


def test_matches_engine_sort_on_two_calls_in_a_row():
    big = configs.settling_lattice(n=5000, seed=31, nx=20, ny=20, nz=15, spacing=0.0195,
                                   steps=10)
    small = configs.settling_lattice(n=700, seed=32, nx=9, ny=9, nz=9, spacing=0.0195, steps=10)
    check(big)     # first call on this device also resolves the scratch address
    check(small)   # second call: a smaller grid over the same scratch


def test_rejects_grids_beyond_the_scratch():
    L = _lib()
    origo = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    Lv = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    num = (ctypes.c_uint32 * 3)(128, 128, 128)  # 2^21 cells > SPH_NOALLOC_MAX_CELLS
    dummy = 16  # never dereferenced: the size check comes first
    rc = L.sph_sort_cells_noalloc(None, 0, origo, Lv, num, dummy, dummy, dummy, dummy, None)
    assert rc == -8
    assert b"scratch" in L.sph_noalloc_error()


def test_rejects_a_crowded_cell():
    """600 positions in one cell of a 3 x 3 x 3 grid: more than the 512 a
    warp orders in registers, so the call refuses instead of running a
    quadratic loop on the GPU."""
    import torch
    L = _lib()
    rng = numpy.random.default_rng(5)
    n = 600
    x4 = numpy.zeros((n, 4))
    x4[:, :3] = rng.uniform(1.05, 1.95, size=(n, 3))
    x4[:, 3] = 0.01
    dev = torch.device("cuda", 0)
    x4_d = torch.from_numpy(x4).to(dev)
    outs = [torch.zeros((m,), dtype=torch.int32, device=dev) for m in (n, n, 27, 27)]
    origo = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    Lv = (ctypes.c_double * 3)(3.0, 3.0, 3.0)
    num = (ctypes.c_uint32 * 3)(3, 3, 3)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.sph_sort_cells_noalloc(x4_d.data_ptr(), n, origo, Lv, num,
                                  *(o.data_ptr() for o in outs), stream)
    assert rc == -8
    assert b"too coarse" in L.sph_noalloc_error()
