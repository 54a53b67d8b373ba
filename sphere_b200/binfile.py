"""Reader and writer for sphere's versioned ``.bin`` simulation files.

The byte layout follows the reference's C++ codec (``src/file_io.cpp:30-417``
for reading, ``:420-731`` for writing) and its Python twin
(``python/sphere.py:965-1553``).  All values are little-endian; floating point
values are IEEE binary64, counters are 32-bit.  Layout, in file order:

* header: version f64, nd i32, np u32, dt, current, total, file_dt (f64),
  step_count u32
* grid: origo[3], L[3] (f64), num[3] u32, periodic i32, adaptive i32
  (adaptive is absent before format 2.14)
* per particle: x+radius (4 f64, interleaved), xyzsum (3 f64), vel+fixvel
  (4 f64, interleaved), force, angpos, angvel, torque (3 f64 each), then the
  per-particle scalars es_dot, es, ev_dot, ev, p (one block each)
* parameters: g[3], k_n, k_t, k_r, E (E absent before 2.13), gamma_n,
  gamma_t, gamma_r, mu_s, mu_d, mu_r, gamma_wn, gamma_wt, mu_ws, mu_wd, rho,
  contactmodel u32, kappa, db, V_b
* walls: nw u32, wmode[nw] i32, (normal[3], position) per wall,
  (mass, vel, force, sigma0) per wall, sigma0_A, sigma0_f, tau_x
* bonds: lambda_bar, nb0 u32, sigma_b, tau_b, pairs (2 u32 each),
  delta_n[nb0], delta_t[nb0][3], omega_n[nb0], omega_t[nb0][3]
* fluid section (only when the run is told the file holds fluid data):
  cfd_solver i32, then the Navier-Stokes or Darcy block
  (``src/file_io.cpp:261-409``)
* color[np] i32

The reference accepts exactly version 2.15 (``src/file_io.cpp:47-54``).
:func:`upgrade_to_215` lifts older files (the shipped fixtures are 2.11) by
inserting the fields added since (``adaptive`` in 2.14, ``E`` in 2.13).
"""

from __future__ import annotations

import copy
import io
from dataclasses import dataclass, field
from typing import Optional

import numpy

VERSION = 2.15

_F8 = numpy.dtype("<f8")
_U4 = numpy.dtype("<u4")
_I4 = numpy.dtype("<i4")


class BinFormatError(ValueError):
    """The file is truncated, has trailing bytes, or an unsupported version."""


@dataclass
class BinData:
    """Contents of one ``.bin`` file.

    Attribute names follow the reference Python ``sim`` class
    (``python/sphere.py:57-454``).  Fluid fields hold the raw file values:
    ``dphi`` is stored exactly as written in the file.
    """

    version: float = VERSION
    nd: int = 3
    np: int = 0
    time_dt: float = 0.0
    time_current: float = 0.0
    time_total: float = 0.0
    time_file_dt: float = 0.0
    time_step_count: int = 0
    origo: numpy.ndarray = field(default_factory=lambda: numpy.zeros(3))
    L: numpy.ndarray = field(default_factory=lambda: numpy.zeros(3))
    num: numpy.ndarray = field(default_factory=lambda: numpy.zeros(3, dtype=numpy.uint32))
    periodic: int = 0
    adaptive: int = 0
    x: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    radius: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    xyzsum: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    vel: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    fixvel: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    force: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    angpos: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    angvel: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    torque: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    es_dot: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    es: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    ev_dot: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    ev: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    p: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    g: numpy.ndarray = field(default_factory=lambda: numpy.zeros(3))
    k_n: float = 1.16e9
    k_t: float = 1.16e9
    k_r: float = 0.0
    E: float = 0.0
    gamma_n: float = 0.0
    gamma_t: float = 0.0
    gamma_r: float = 0.0
    mu_s: float = 0.5
    mu_d: float = 0.5
    mu_r: float = 0.0
    gamma_wn: float = 1.0e3
    gamma_wt: float = 0.0
    mu_ws: float = 0.5
    mu_wd: float = 0.5
    rho: float = 2600.0
    contactmodel: int = 2
    kappa: float = 0.0
    db: float = 0.0
    V_b: float = 0.0
    nw: int = 0
    wmode: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0, dtype=numpy.int32))
    w_n: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    w_x: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    w_m: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    w_vel: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    w_force: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    w_sigma0: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    w_sigma0_A: float = 0.0
    w_sigma0_f: float = 0.0
    w_tau_x: float = 0.0
    lambda_bar: float = 1.0
    nb0: int = 0
    sigma_b: float = numpy.inf
    tau_b: float = numpy.inf
    bonds: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 2), dtype=numpy.uint32))
    bonds_delta_n: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    bonds_delta_t: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    bonds_omega_n: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0))
    bonds_omega_t: numpy.ndarray = field(default_factory=lambda: numpy.zeros((0, 3)))
    # fluid section
    fluid: bool = False
    cfd_solver: int = 0
    mu: float = 0.0
    v_f: Optional[numpy.ndarray] = None        # (nx, ny, nz, 3)
    p_f: Optional[numpy.ndarray] = None        # (nx, ny, nz)
    phi: Optional[numpy.ndarray] = None
    dphi: Optional[numpy.ndarray] = None       # raw file value
    rho_f: float = 1000.0
    p_mod_A: float = 0.0
    p_mod_f: float = 0.0
    p_mod_phi: float = 0.0
    bc_xn: int = 2
    bc_xp: int = 2
    bc_yn: int = 2
    bc_yp: int = 2
    bc_bot: int = 0
    bc_top: int = 0
    free_slip_bot: int = 1
    free_slip_top: int = 1
    bc_bot_flux: float = 0.0
    bc_top_flux: float = 0.0
    p_f_constant: Optional[numpy.ndarray] = None  # (nx, ny, nz) int32
    tolerance: float = 1e-3
    maxiter: int = 10000
    ndem: int = 1
    c_phi: float = 1.0
    f_p: Optional[numpy.ndarray] = None        # (np, 3)
    beta_f: float = 4.5e-10
    k_c: float = 4.6e-10
    # Navier-Stokes only (cfd_solver 0); kept so such files round-trip
    ns_gamma: float = 0.0
    ns_theta: float = 1.0
    ns_beta: float = 0.0
    c_v: float = 1.0
    dt_dem_fac: float = 1.0
    f_d: Optional[numpy.ndarray] = None
    f_v: Optional[numpy.ndarray] = None
    f_sum: Optional[numpy.ndarray] = None
    color: numpy.ndarray = field(default_factory=lambda: numpy.zeros(0, dtype=numpy.int32))

    def copy(self) -> "BinData":
        return copy.deepcopy(self)

    @property
    def ncells(self) -> int:
        return int(self.num[0]) * int(self.num[1]) * int(self.num[2])


class _Reader:
    def __init__(self, buf: bytes):
        self.buf = buf
        self.pos = 0

    def take(self, dtype, count=1):
        dtype = numpy.dtype(dtype)
        nbytes = dtype.itemsize * count
        if self.pos + nbytes > len(self.buf):
            raise BinFormatError(
                f"file truncated at byte {self.pos} (needed {nbytes} more)")
        arr = numpy.frombuffer(self.buf, dtype=dtype, count=count, offset=self.pos)
        self.pos += nbytes
        return arr.copy()

    def f8(self):
        return float(self.take(_F8)[0])

    def u4(self):
        return int(self.take(_U4)[0])

    def i4(self):
        return int(self.take(_I4)[0])

    @property
    def remaining(self):
        return len(self.buf) - self.pos


def _read_grid_field(r: _Reader, num, per_cell):
    """Fluid grid blocks are written z-major, x fastest."""
    nx, ny, nz = (int(v) for v in num)
    raw = r.take(_F8, nx * ny * nz * per_cell).reshape(nz, ny, nx, per_cell)
    return raw.transpose(2, 1, 0, 3)  # -> (nx, ny, nz, per_cell)


def parse_bin(buf: bytes, fluid: Optional[bool] = None,
              allow_old: bool = False) -> BinData:
    """Parse the bytes of a ``.bin`` file.

    ``fluid`` plays the role of the reference's ``--fluid`` flag
    (``src/file_io.cpp:261``); ``None`` decides from the number of bytes that
    follow the bond block.  Files older than 2.15 are rejected, as the
    reference does, unless ``allow_old`` is set.
    """
    r = _Reader(buf)
    d = BinData()
    d.version = r.f8()
    if d.version != VERSION and not allow_old:
        raise BinFormatError(
            f"file written by sphere version {d.version}, expected {VERSION}")
    d.nd = r.i4()
    if d.nd != 3:
        raise BinFormatError(f"dimensionality {d.nd} is not 3")
    n = d.np = r.u4()
    d.time_dt = r.f8()
    d.time_current = r.f8()
    d.time_total = r.f8()
    d.time_file_dt = r.f8()
    d.time_step_count = r.u4()
    d.origo = r.take(_F8, 3)
    d.L = r.take(_F8, 3)
    d.num = r.take(_U4, 3)
    d.periodic = r.i4()
    d.adaptive = r.i4() if d.version >= 2.14 else 0
    xr = r.take(_F8, 4 * n).reshape(n, 4)
    d.x = xr[:, :3].copy()
    d.radius = xr[:, 3].copy()
    d.xyzsum = r.take(_F8, 3 * n).reshape(n, 3)
    vf = r.take(_F8, 4 * n).reshape(n, 4)
    d.vel = vf[:, :3].copy()
    d.fixvel = vf[:, 3].copy()
    d.force = r.take(_F8, 3 * n).reshape(n, 3)
    d.angpos = r.take(_F8, 3 * n).reshape(n, 3)
    d.angvel = r.take(_F8, 3 * n).reshape(n, 3)
    d.torque = r.take(_F8, 3 * n).reshape(n, 3)
    d.es_dot = r.take(_F8, n)
    d.es = r.take(_F8, n)
    d.ev_dot = r.take(_F8, n)
    d.ev = r.take(_F8, n)
    d.p = r.take(_F8, n)
    d.g = r.take(_F8, 3)
    d.k_n = r.f8()
    d.k_t = r.f8()
    d.k_r = r.f8()
    d.E = r.f8() if d.version >= 2.13 else 0.0
    d.gamma_n = r.f8()
    d.gamma_t = r.f8()
    d.gamma_r = r.f8()
    d.mu_s = r.f8()
    d.mu_d = r.f8()
    d.mu_r = r.f8()
    d.gamma_wn = r.f8()
    d.gamma_wt = r.f8()
    d.mu_ws = r.f8()
    d.mu_wd = r.f8()
    d.rho = r.f8()
    d.contactmodel = r.u4()
    d.kappa = r.f8()
    d.db = r.f8()
    d.V_b = r.f8()
    nw = d.nw = r.u4()
    if nw > 6:
        raise BinFormatError(f"nw={nw} exceeds the 6 walls the format allows")
    d.wmode = r.take(_I4, nw)
    wn = r.take(_F8, 4 * nw).reshape(nw, 4)
    d.w_n = wn[:, :3].copy()
    d.w_x = wn[:, 3].copy()
    wm = r.take(_F8, 4 * nw).reshape(nw, 4)
    d.w_m = wm[:, 0].copy()
    d.w_vel = wm[:, 1].copy()
    d.w_force = wm[:, 2].copy()
    d.w_sigma0 = wm[:, 3].copy()
    d.w_sigma0_A = r.f8()
    d.w_sigma0_f = r.f8()
    d.w_tau_x = r.f8()
    d.lambda_bar = r.f8()
    nb = d.nb0 = r.u4()
    d.sigma_b = r.f8()
    d.tau_b = r.f8()
    d.bonds = r.take(_U4, 2 * nb).reshape(nb, 2)
    d.bonds_delta_n = r.take(_F8, nb)
    d.bonds_delta_t = r.take(_F8, 3 * nb).reshape(nb, 3)
    d.bonds_omega_n = r.take(_F8, nb)
    d.bonds_omega_t = r.take(_F8, 3 * nb).reshape(nb, 3)

    if fluid is None:
        fluid = r.remaining != 4 * n
    d.fluid = bool(fluid)
    if d.fluid:
        d.cfd_solver = r.i4()
        if d.cfd_solver not in (0, 1):
            raise BinFormatError(f"cfd_solver {d.cfd_solver} not understood")
        d.mu = r.f8()
        cells = _read_grid_field(r, d.num, 6)
        d.v_f = cells[..., 0:3].copy()
        d.p_f = cells[..., 3].copy()
        d.phi = cells[..., 4].copy()
        d.dphi = cells[..., 5].copy()
        d.rho_f = r.f8()
        d.p_mod_A = r.f8()
        d.p_mod_f = r.f8()
        d.p_mod_phi = r.f8()
        if d.cfd_solver == 1:
            d.bc_xn = r.i4()
            d.bc_xp = r.i4()
            d.bc_yn = r.i4()
            d.bc_yp = r.i4()
            d.bc_bot = r.i4()
            d.bc_top = r.i4()
        else:
            # The reference's NS reader takes bc_top first
            # (src/file_io.cpp:306-307).
            d.bc_top = r.i4()
            d.bc_bot = r.i4()
        d.free_slip_bot = r.i4()
        d.free_slip_top = r.i4()
        d.bc_bot_flux = r.f8()
        d.bc_top_flux = r.f8()
        nx, ny, nz = (int(v) for v in d.num)
        d.p_f_constant = r.take(_I4, d.ncells).reshape(nz, ny, nx).transpose(2, 1, 0).copy()
        if d.cfd_solver == 0:
            d.ns_gamma = r.f8()
            d.ns_theta = r.f8()
            d.ns_beta = r.f8()
            d.tolerance = r.f8()
            d.maxiter = r.u4()
            d.ndem = r.u4()
            d.c_phi = r.f8()
            d.c_v = r.f8()
            d.dt_dem_fac = r.f8()
            d.f_d = r.take(_F8, 3 * n).reshape(n, 3)
            d.f_p = r.take(_F8, 3 * n).reshape(n, 3)
            d.f_v = r.take(_F8, 3 * n).reshape(n, 3)
            d.f_sum = r.take(_F8, 3 * n).reshape(n, 3)
        else:
            d.tolerance = r.f8()
            d.maxiter = r.u4()
            d.ndem = r.u4()
            d.c_phi = r.f8()
            d.f_p = r.take(_F8, 3 * n).reshape(n, 3)
            d.beta_f = r.f8()
            d.k_c = r.f8()
    d.color = r.take(_I4, n)
    if r.remaining != 0:
        raise BinFormatError(f"{r.remaining} trailing bytes after the color block")
    return d


def read_bin(path, fluid: Optional[bool] = None, allow_old: bool = False) -> BinData:
    with open(path, "rb") as fh:
        return parse_bin(fh.read(), fluid=fluid, allow_old=allow_old)


def _f8(v):
    return numpy.asarray(v, dtype=_F8).tobytes()


def _u4(v):
    return numpy.asarray(v, dtype=_U4).tobytes()


def _i4(v):
    return numpy.asarray(v, dtype=_I4).tobytes()


def _grid_bytes(arr_xyz_c: numpy.ndarray, dtype) -> bytes:
    # (nx, ny, nz, c) -> z-major, x fastest
    return numpy.ascontiguousarray(numpy.asarray(arr_xyz_c).transpose(2, 1, 0, 3),
                                dtype=dtype).tobytes()


def serialize_bin(d: BinData) -> bytes:
    """Inverse of :func:`parse_bin`; always writes format 2.15."""
    n = int(d.np)
    nw = int(d.nw)
    nb = int(d.nb0)
    out = io.BytesIO()
    w = out.write
    w(_f8(VERSION))
    w(_i4(d.nd))
    w(_u4(n))
    for v in (d.time_dt, d.time_current, d.time_total, d.time_file_dt):
        w(_f8(v))
    w(_u4(d.time_step_count))
    w(_f8(numpy.asarray(d.origo).reshape(3)))
    w(_f8(numpy.asarray(d.L).reshape(3)))
    w(_u4(numpy.asarray(d.num).reshape(3)))
    w(_i4(d.periodic))
    w(_i4(d.adaptive))
    w(_f8(numpy.column_stack([numpy.asarray(d.x).reshape(n, 3),
                           numpy.asarray(d.radius).reshape(n)])))
    w(_f8(numpy.asarray(d.xyzsum).reshape(n, 3)))
    w(_f8(numpy.column_stack([numpy.asarray(d.vel).reshape(n, 3),
                           numpy.asarray(d.fixvel).reshape(n)])))
    for a in (d.force, d.angpos, d.angvel, d.torque):
        w(_f8(numpy.asarray(a).reshape(n, 3)))
    for a in (d.es_dot, d.es, d.ev_dot, d.ev, d.p):
        w(_f8(numpy.asarray(a).reshape(n)))
    w(_f8(numpy.asarray(d.g).reshape(3)))
    for v in (d.k_n, d.k_t, d.k_r, d.E, d.gamma_n, d.gamma_t, d.gamma_r,
              d.mu_s, d.mu_d, d.mu_r, d.gamma_wn, d.gamma_wt, d.mu_ws,
              d.mu_wd, d.rho):
        w(_f8(v))
    w(_u4(d.contactmodel))
    for v in (d.kappa, d.db, d.V_b):
        w(_f8(v))
    w(_u4(nw))
    w(_i4(numpy.asarray(d.wmode).reshape(nw)))
    w(_f8(numpy.column_stack([numpy.asarray(d.w_n).reshape(nw, 3),
                           numpy.asarray(d.w_x).reshape(nw)])))
    w(_f8(numpy.column_stack([numpy.asarray(d.w_m).reshape(nw),
                           numpy.asarray(d.w_vel).reshape(nw),
                           numpy.asarray(d.w_force).reshape(nw),
                           numpy.asarray(d.w_sigma0).reshape(nw)])))
    for v in (d.w_sigma0_A, d.w_sigma0_f, d.w_tau_x, d.lambda_bar):
        w(_f8(v))
    w(_u4(nb))
    w(_f8(d.sigma_b))
    w(_f8(d.tau_b))
    w(_u4(numpy.asarray(d.bonds).reshape(nb, 2)))
    w(_f8(numpy.asarray(d.bonds_delta_n).reshape(nb)))
    w(_f8(numpy.asarray(d.bonds_delta_t).reshape(nb, 3)))
    w(_f8(numpy.asarray(d.bonds_omega_n).reshape(nb)))
    w(_f8(numpy.asarray(d.bonds_omega_t).reshape(nb, 3)))
    if d.fluid:
        w(_i4(d.cfd_solver))
        w(_f8(d.mu))
        cells = numpy.concatenate([
            numpy.asarray(d.v_f).reshape(*d.num, 3),
            numpy.asarray(d.p_f).reshape(*d.num, 1),
            numpy.asarray(d.phi).reshape(*d.num, 1),
            numpy.asarray(d.dphi).reshape(*d.num, 1)], axis=3)
        w(_grid_bytes(cells, _F8))
        for v in (d.rho_f, d.p_mod_A, d.p_mod_f, d.p_mod_phi):
            w(_f8(v))
        if d.cfd_solver == 1:
            for v in (d.bc_xn, d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top):
                w(_i4(v))
        else:
            w(_i4(d.bc_top))
            w(_i4(d.bc_bot))
        w(_i4(d.free_slip_bot))
        w(_i4(d.free_slip_top))
        w(_f8(d.bc_bot_flux))
        w(_f8(d.bc_top_flux))
        pc = d.p_f_constant
        if pc is None:
            pc = numpy.zeros(tuple(int(v) for v in d.num), dtype=numpy.int32)
        w(_grid_bytes(numpy.asarray(pc).reshape(*d.num, 1), _I4))
        if d.cfd_solver == 0:
            for v in (d.ns_gamma, d.ns_theta, d.ns_beta, d.tolerance):
                w(_f8(v))
            w(_u4(d.maxiter))
            w(_u4(d.ndem))
            for v in (d.c_phi, d.c_v, d.dt_dem_fac):
                w(_f8(v))
            for a in (d.f_d, d.f_p, d.f_v, d.f_sum):
                w(_f8(numpy.zeros((n, 3)) if a is None else numpy.asarray(a).reshape(n, 3)))
        else:
            w(_f8(d.tolerance))
            w(_u4(d.maxiter))
            w(_u4(d.ndem))
            w(_f8(d.c_phi))
            w(_f8(numpy.zeros((n, 3)) if d.f_p is None else numpy.asarray(d.f_p).reshape(n, 3)))
            w(_f8(d.beta_f))
            w(_f8(d.k_c))
    w(_i4(numpy.asarray(d.color).reshape(n)))
    return out.getvalue()


def write_bin(d: BinData, path) -> None:
    with open(path, "wb") as fh:
        fh.write(serialize_bin(d))


def upgrade_to_215(src_path, dst_path, fluid: Optional[bool] = False) -> BinData:
    """Rewrite an older sphere file (2.11 onwards) as format 2.15.

    The fields added since 2.11 take the values older programs implied:
    ``adaptive = 0`` (added in 2.14) and ``E = 0`` (added in 2.13)
    (``python/sphere.py:1033-1036,1083-1086``).
    """
    d = read_bin(src_path, fluid=fluid, allow_old=True)
    d.version = VERSION
    write_bin(d, dst_path)
    return d


__all__ = ["BinData", "BinFormatError", "VERSION", "parse_bin", "read_bin",
           "serialize_bin", "write_bin", "upgrade_to_215"]
