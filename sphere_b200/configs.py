"""Seeded synthetic workloads for the DEM step.

Each generator returns a :class:`~sphere_b200.binfile.BinData` built the way
the reference's Python setup helpers would build it, so the same file can be
run by this engine, the oracle and the reference.  Seeds are explicit; the
same seed gives the same bytes.

Workloads (the sizes of the published benchmark configurations):

* :func:`settling_lattice` -- dry settling of N spheres on a cubic lattice
  (N = 10,000, radii U(0.009, 0.011) m, spacing 0.025 m, jitter +/-0.002 m,
  periodic x/y, linear contact k_n = k_t = 1.16e7 N/m, mu = 0.5).
* :func:`shear_benchmark` -- a settled packing under a top wall at normal
  stress sigma0 with the top layer sheared along x (N = 100,000, radii
  U(0.008, 0.012) m, Young's modulus contact E = 7e8 Pa, mu = 0.5).
* :func:`large_cohesive_packing` -- N spheres with log-normal radii bonded
  to their initial neighbours (N = 4,000,000, median radius 0.01 m, sigma_ln
  0.3, clipped to [0.004, 0.03] m, bonds within 1.05 x the radius sum,
  bond stiffness 1e7, tensile strength 1e5 Pa, E = 7e8 Pa, mu = 0.5).
* :func:`two_particle` / :func:`wall_particle` -- the reference's collision
  test set-ups (``tests/contactmodel.py``, ``tests/contactmodel_wall.py``).
"""
from __future__ import annotations

import math
import os

import numpy

from .binfile import BinData


def time_step(d: BinData, epsilon: float = 0.01) -> float:
    """The reference's automatic time step (``python/sphere.py:3307-3376``):
    dt = epsilon / sqrt(k_max / m_min)."""
    r_min = numpy.min(d.radius)
    m_min = d.rho * 4.0 / 3.0 * numpy.pi * r_min ** 3
    if d.E > 0.001:
        k_max = numpy.max(numpy.pi / 2.0 * d.E * d.radius)
    else:
        k_max = numpy.max([d.k_n, d.k_t])
    return float(epsilon / (numpy.sqrt(k_max / m_min)))


def init_temporal(d: BinData, total: float, file_dt: float = 0.05,
                  current: float = 0.0, epsilon: float = 0.01) -> None:
    d.time_dt = time_step(d, epsilon)
    d.time_current = current
    d.time_total = total
    d.time_file_dt = file_dt
    d.time_step_count = 0


def _particles(d: BinData, n: int) -> None:
    d.np = n
    d.x = numpy.zeros((n, 3))
    d.radius = numpy.ones(n)
    d.xyzsum = numpy.zeros((n, 3))
    d.vel = numpy.zeros((n, 3))
    d.fixvel = numpy.zeros(n)
    d.force = numpy.zeros((n, 3))
    d.angpos = numpy.zeros((n, 3))
    d.angvel = numpy.zeros((n, 3))
    d.torque = numpy.zeros((n, 3))
    d.es_dot = numpy.zeros(n)
    d.es = numpy.zeros(n)
    d.ev_dot = numpy.zeros(n)
    d.ev = numpy.zeros(n)
    d.p = numpy.zeros(n)
    d.color = numpy.zeros(n, dtype=numpy.int32)


def default_params(d: BinData, mu_s=0.5, mu_d=0.5, rho=2600.0, k_n=1.16e9,
                   k_t=1.16e9, gamma_n=0.0, gamma_t=0.0, gamma_wn=1.0e4,
                   gamma_wt=1.0e4) -> None:
    """``sim.defaultParams`` (``python/sphere.py:3762-3858``) without
    capillary cohesion."""
    d.rho = rho
    d.k_n = k_n
    d.k_t = k_t
    d.k_r = 0.0
    d.gamma_n = gamma_n
    d.gamma_t = gamma_t
    d.gamma_r = 0.0
    d.mu_s = mu_s
    d.mu_d = mu_d
    d.mu_r = 0.0
    d.gamma_wn = gamma_wn
    d.gamma_wt = gamma_wt
    d.mu_ws = mu_s
    d.mu_wd = mu_d
    d.kappa = 0.0
    d.V_b = 0.0
    d.db = 0.0


def grid_for(d: BinData, L, origo=(0.0, 0.0, 0.0), dx: float = -1.0) -> None:
    """``sim.defineWorldBoundaries`` (``python/sphere.py:2607-2653``)."""
    cell = dx if dx > 0.0 else 2.1 * numpy.amax(d.radius)
    d.origo = numpy.asarray(origo, dtype=numpy.float64).copy()
    d.L = numpy.asarray(L, dtype=numpy.float64).copy()
    d.num = numpy.ceil((d.L - d.origo) / cell).astype(numpy.uint32)
    if numpy.any(d.num < 3):
        raise ValueError(f"grid must be at least 3 cells per axis, got {d.num}")


def settling_lattice(n: int = 10000, seed: int = 0, nx: int = 22, ny: int = 22,
                     nz: int = 21, spacing: float = 0.025, jitter: float = 0.002,
                     r_min: float = 0.009, r_max: float = 0.011,
                     steps: int = 20000, contactmodel: int = 2) -> BinData:
    """Dry settling: N spheres on the first N sites of an nx*ny*nz cubic
    lattice, seeded jitter, radii and velocities; periodic x/y, no dynamic
    walls (the implicit bottom wall at origo.z and the fixed top at L.z
    apply)."""
    if n > nx * ny * nz:
        raise ValueError("lattice too small for n particles")
    rng = numpy.random.default_rng(seed)
    d = BinData()
    _particles(d, n)
    idx = numpy.arange(n)
    ix, iy, iz = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    centres = numpy.column_stack([ix, iy, iz]).astype(numpy.float64)
    d.x = (centres + 0.5) * spacing + rng.uniform(-jitter, jitter, size=(n, 3))
    d.radius = rng.uniform(r_min, r_max, size=n)
    d.vel = rng.uniform(-0.01, 0.01, size=(n, 3))
    default_params(d, mu_s=0.5, mu_d=0.5, k_n=1.16e7, k_t=1.16e7)
    d.contactmodel = contactmodel
    d.g = numpy.array([0.0, 0.0, -9.81])
    side = max(nx, ny) * spacing
    grid_for(d, L=[nx * spacing, ny * spacing, side])
    d.periodic = 1
    d.nw = 0
    dt = time_step(d)
    init_temporal(d, total=steps * dt, file_dt=steps * dt * 2.0)
    return d


def two_particle(radii=(1.0, 1.0), z=(2.0, 4.05), vel0=1.0, gamma_n=0.0,
                 E=0.0, angle_x=0.0, mu=0.5, total=0.1, file_dt=0.01) -> BinData:
    """The reference's two-particle collision set-up (``tests/contactmodel.py``):
    particle 0 moves towards particle 1 along z, world 10 m cubed, no
    gravity, sphere's default stiffness 1.16e9 N/m."""
    d = BinData()
    _particles(d, 2)
    d.radius = numpy.asarray(radii, dtype=numpy.float64).copy()
    d.x[0, :] = [5.0, 5.0, z[0]]
    d.x[1, :] = [5.0 + angle_x, 5.0, z[1]]
    d.vel[0, 2] = vel0
    default_params(d, mu_s=mu, mu_d=mu, gamma_wn=1.0e3, gamma_wt=0.0)
    d.gamma_n = gamma_n
    d.E = E
    grid_for(d, L=[10.0, 10.0, 10.0])
    init_temporal(d, total=total, file_dt=file_dt)
    return d


def wall_particle(radius=1.0, z=1.05, vel0=-1.0, gamma_wn=0.0, E=0.0,
                  total=0.1, file_dt=0.01) -> BinData:
    """One particle moving into the implicit bottom wall
    (``tests/contactmodel_wall.py``)."""
    d = BinData()
    _particles(d, 1)
    d.radius[:] = radius
    d.x[0, :] = [5.0, 5.0, z]
    d.vel[0, 2] = vel0
    default_params(d, gamma_wn=gamma_wn, gamma_wt=0.0)
    d.E = E
    grid_for(d, L=[10.0, 10.0, 10.0])
    init_temporal(d, total=total, file_dt=file_dt)
    return d


def add_top_wall(d: BinData, sigma0: float, wmode: int = 1, mass=None) -> None:
    """One dynamic top wall at the highest particle surface
    (``sim.adjustUpperWall`` + ``consolidate``, ``python/sphere.py:2949-3048``)."""
    zmax = float(numpy.max(d.x[:, 2] + d.radius))
    d.nw = 1
    d.wmode = numpy.array([wmode], dtype=numpy.int32)
    d.w_n = numpy.array([[0.0, 0.0, -1.0]])
    d.w_x = numpy.array([zmax])
    m = float(numpy.sum(d.rho * 4.0 / 3.0 * numpy.pi * d.radius ** 3)) if mass is None else mass
    d.w_m = numpy.array([m])
    d.w_vel = numpy.zeros(1)
    d.w_force = numpy.zeros(1)
    d.w_sigma0 = numpy.array([sigma0])


def shear_setup(d: BinData, shear_velocity: float, sigma0: float) -> None:
    """``sim.shear`` (``python/sphere.py:3097-3165``) at a given top-layer
    velocity: bottom and top layers get fixvel = 1, the top layer moves at
    shear_velocity along x, one stress-controlled top wall, no wall friction."""
    z_min = numpy.min(d.x[:, 2] - d.radius)
    z_max = numpy.max(d.x[:, 2] + d.radius)
    cell = d.L[0] / d.num[0]
    d.num = d.num.copy()
    d.num[2] += 1
    d.L = d.L.copy()
    d.L[2] = d.num[2] * cell
    d.vel[:] = 0.0
    d.angvel[:] = 0.0
    d.force[:] = 0.0
    d.torque[:] = 0.0
    d.angpos[:] = 0.0
    d.es[:] = 0.0
    d.ev[:] = 0.0
    d.xyzsum[:] = 0.0
    low = d.x[:, 2] < (z_max - z_min) * 0.3
    d_max_below = numpy.max(d.radius[low]) * 2.0
    bottom = d.x[:, 2] < (z_min + d_max_below)
    d.fixvel[bottom] = 1
    high = d.x[:, 2] > (z_max - z_min) * 0.7
    d_max_top = numpy.max(d.radius[high]) * 2.0
    top = d.x[:, 2] > (z_max - d_max_top)
    d.fixvel[top] = 1
    d.vel[top, 0] = shear_velocity
    add_top_wall(d, sigma0, wmode=1)
    d.gamma_wt = 0.0
    d.mu_ws = 0.0
    d.mu_wd = 0.0


def _lattice(n: int, seed: int, r_min: float, r_max: float, gap: float = 0.02):
    """Jittered cubic lattice with spacing 2*r_max*(1+gap), roughly twice
    as wide as tall; returns (x, radius, side, nz, spacing)."""
    rng = numpy.random.default_rng(seed)
    spacing = 2.0 * r_max * (1.0 + gap)
    side = int(math.ceil((2.0 * n) ** (1.0 / 3.0)))
    nz = int(math.ceil(n / (side * side)))
    idx = numpy.arange(n)
    ix, iy, iz = idx % side, (idx // side) % side, idx // (side * side)
    centres = numpy.column_stack([ix, iy, iz]).astype(numpy.float64)
    jit = 0.5 * gap * r_max
    x = (centres + 0.5) * spacing + rng.uniform(-jit, jit, size=(n, 3))
    radius = rng.uniform(r_min, r_max, size=n)
    return x, radius, side, nz, spacing


def settle_packing(n: int = 100000, seed: int = 1, r_min: float = 0.008,
                   r_max: float = 0.012, g_factor: float = 100.0,
                   collapse_chunk: int = 5000, collapse_max: int = 200000,
                   v_settled: float = 0.02, quench_steps: int = 6000,
                   quench_every: int = 1000, precision: str = "mixed", log=None) -> BinData:
    """A settled packing made by damped DEM settling on the GPU engine.

    Spheres start on a jittered lattice and collapse under g_factor * 9.81
    m/s^2 with strong normal and tangential damping and a 5x time step, in
    chunks of collapse_chunk steps until 99 % of the spheres are slower
    than v_settled (at most collapse_max steps); the lattice must fall by about
    half its height, which takes a few tens of milliseconds of model time.
    Then the kinetic energy is drained by setting all velocities to zero
    every quench_every steps, first at g_factor g and then at 1 g
    (quench_steps each).  Used to make the dense starting state of the
    shear workload (the 'prepacked by settling' step); it is not a timed
    path.
    """
    from .engine import Engine  # the GPU engine

    x, radius, side, nz, spacing = _lattice(n, seed, r_min, r_max)
    d = BinData()
    _particles(d, n)
    d.x = x
    d.radius = radius
    default_params(d, mu_s=0.5, mu_d=0.5, k_n=1.16e7, k_t=1.16e7)
    m_min = d.rho * 4.0 / 3.0 * numpy.pi * r_min ** 3
    d.gamma_n = 0.8 * 2.0 * math.sqrt(m_min * d.k_n)
    d.gamma_t = 0.2 * d.gamma_n
    d.gamma_wn = 4.0 * d.gamma_n
    d.gamma_wt = 0.0
    d.g = numpy.array([0.0, 0.0, -9.81 * g_factor])
    L = side * spacing
    grid_for(d, L=[L, L, (nz + 1) * spacing], dx=2.1 * r_max)
    d.periodic = 1
    d.time_dt = 5.0 * time_step(d)
    d.time_total = 1e9
    d.time_file_dt = 1e9

    def v99_of(eng):
        # 99th percentile speed: a few caged spheres rattle at 100 g long
        # after the bulk has come to rest
        v = eng.get("vel")
        return float(numpy.percentile(numpy.sqrt((v[:, :3] ** 2).sum(axis=1)), 99.0))

    def quench(eng, steps):
        zero = numpy.zeros((n, 4))
        for done in range(0, steps, quench_every):
            eng.step(quench_every)
            v = eng.get("vel")
            vmax = float(numpy.sqrt((v[:, :3] ** 2).sum(axis=1)).max())
            zero[:, 3] = v[:, 3]
            eng.set("vel", zero)
            eng.set("angvel", numpy.zeros((n, 4)))
            if log:
                log(f"settle: quench after {done + quench_every} steps, max |v| {vmax:.3e} m/s")

    eng = Engine(d, precision=precision, graph_steps=quench_every)
    done = 0
    while done < collapse_max:
        eng.step(collapse_chunk)
        done += collapse_chunk
        v99 = v99_of(eng)
        if log:
            log(f"settle: collapse {done} steps, 99th percentile |v| {v99:.3e} m/s")
        if v99 < v_settled:
            break
    quench(eng, quench_steps)
    d.x = eng.get("x")[:, :3].copy()
    eng.close()
    d.g = numpy.array([0.0, 0.0, -9.81])
    eng = Engine(d, precision=precision, graph_steps=quench_every)
    quench(eng, quench_steps)
    state = d.copy()
    state.x = eng.get("x")[:, :3].copy()
    c = eng.get("contacts")
    if log:
        log(f"settle: {float((c != n).sum()) / n:.2f} contacts per particle")
    eng.close()
    state.vel[:] = 0.0
    state.angvel[:] = 0.0
    top = float(numpy.max(state.x[:, 2] + state.radius))
    state.L = state.L.copy()
    state.num = state.num.copy()
    cell = state.L[0] / state.num[0]
    state.num[2] = int(math.ceil(top * 1.1 / cell))
    state.L[2] = state.num[2] * cell
    return state


DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def _fixture_path(n: int, seed: int) -> str:
    return os.path.join(DATA_DIR, f"settled_packing_n{n}_seed{seed}.npz")


def _byte_planes(a: numpy.ndarray) -> numpy.ndarray:
    """float64 array -> its 8 byte planes (the sign/exponent planes of
    positions in a box compress far better apart)."""
    b = numpy.ascontiguousarray(a, dtype="<f8").view(numpy.uint8).reshape(-1, 8)
    return numpy.ascontiguousarray(b.T)


def _from_planes(p: numpy.ndarray, shape) -> numpy.ndarray:
    return numpy.ascontiguousarray(p.T).view("<f8").reshape(shape)


def pack_fixture(state: BinData, seed: int) -> str:
    """Stores a settled packing (positions, radii and grid of the state
    settle_packing returns; every other field of that state is zero or a
    default) as the packaged fixture of (np, seed)."""
    os.makedirs(DATA_DIR, exist_ok=True)
    path = _fixture_path(state.np, seed)
    numpy.savez_compressed(path, x_planes=_byte_planes(state.x),
                           radius_planes=_byte_planes(state.radius),
                           L=state.L, num=state.num, origo=state.origo,
                           recipe=numpy.array(f"configs.settle_packing(n={state.np}, seed={seed})"))
    return path


def _load_fixture(n: int, seed: int):
    path = _fixture_path(n, seed)
    if not os.path.exists(path):
        return None
    z = numpy.load(path)
    d = BinData()
    _particles(d, n)
    d.x = _from_planes(z["x_planes"], (n, 3))
    d.radius = _from_planes(z["radius_planes"], (n,))
    default_params(d, mu_s=0.5, mu_d=0.5, k_n=1.16e7, k_t=1.16e7)
    d.g = numpy.array([0.0, 0.0, -9.81])
    d.origo = numpy.array(z["origo"], dtype=numpy.float64)
    d.L = numpy.array(z["L"], dtype=numpy.float64)
    d.num = numpy.array(z["num"], dtype=numpy.uint32)
    d.periodic = 1
    d.time_dt = time_step(d)
    d.time_total = 1e9
    d.time_file_dt = 1e9
    return d


def settled_packing(n: int = 100000, seed: int = 1, cache_dir=None, log=None,
                    packaged: bool = True) -> BinData:
    """The settled packing of the benchmark workloads: the packaged fixture
    where one exists for (n, seed) (no device is touched), else a .bin cached
    under cache_dir (default $SPHB_CACHE, or a folder in the system's
    temporary directory), else settled on the GPU engine and cached."""
    import tempfile
    from .binfile import read_bin, write_bin

    if packaged:
        d = _load_fixture(n, seed)
        if d is not None:
            return d
    cache_dir = cache_dir or os.environ.get("SPHB_CACHE") or os.path.join(
        tempfile.gettempdir(), "sphere_b200_cache")
    os.makedirs(cache_dir, exist_ok=True)
    path = os.path.join(cache_dir, f"packing4_n{n}_seed{seed}.bin")
    if os.path.exists(path):
        return read_bin(path)
    base = settle_packing(n=n, seed=seed, log=log)
    write_bin(base, path + ".tmp")
    os.replace(path + ".tmp", path)
    return base


def darcy_benchmark(n: int = 100000, seed: int = 1, grid=(40, 40, 80), sigma0: float = 10e3,
                    cache_dir=None, log=None) -> BinData:
    """The Darcy-coupled consolidation workload: the settled packing on a
    40 x 40 x 80 fluid (and sorting) grid, a stress-controlled top wall at
    sigma0 (the benchmark steps it 10 -> 20 -> 40 -> 80 kPa), Young's modulus
    E = 7e8 Pa, mu = 0.5, Darcy flow with mu_f = 1.797e-6 Pa s, rho_f = 1000
    kg/m^3, k_c = 3.5e-13 m^2, beta_f = 4.5e-10 1/Pa, residual tolerance
    1e-8, bottom no-flow, top Dirichlet, periodic sides."""
    d = settled_packing(n, seed, cache_dir, log).copy()
    default_params(d, mu_s=0.5, mu_d=0.5, k_n=1.16e7, k_t=1.16e7)
    d.E = 7e8
    d.gamma_wn = 1.0e4
    d.gamma_wt = 0.0
    nx, ny, nz = grid
    dx = float(d.L[0]) / nx
    d.origo = numpy.zeros(3)
    d.L = numpy.array([nx * dx, ny * dx, nz * dx])
    d.num = numpy.array([nx, ny, nz], dtype=numpy.uint32)
    d.vel[:] = 0.0
    d.angvel[:] = 0.0
    add_top_wall(d, sigma0, wmode=1)
    d.time_dt = time_step(d)
    d.time_current = 0.0
    d.time_total = 1e9 * d.time_dt
    d.time_file_dt = d.time_total
    init_fluid_darcy(d, mu=1.797e-6, rho_f=1000.0, k_c=3.5e-13, beta_f=4.5e-10,
                     tolerance=1e-8, maxiter=200000, bottom_no_flow=True)
    return d


def shear_benchmark(n: int = 100000, seed: int = 1, sigma0: float = 20e3,
                    shear_velocity: float = 1e-4, cache_dir=None, log=None) -> BinData:
    """The dense-shear workload: a settled packing of n spheres (radii
    U(0.008, 0.012) m), fixed bottom layer, top layer sheared at
    shear_velocity along x, one top wall at normal stress sigma0, Young's
    modulus contact E = 7e8 Pa, mu = 0.5, periodic x/y.  The settled packing
    is cached as a .bin file under cache_dir."""
    d = settled_packing(n, seed, cache_dir, log).copy()
    default_params(d, mu_s=0.5, mu_d=0.5, k_n=1.16e7, k_t=1.16e7)
    d.E = 7e8
    d.gamma_n = 0.0
    d.gamma_t = 0.0
    d.gamma_wn = 1.0e4
    d.gamma_wt = 1.0e4
    shear_setup(d, shear_velocity, sigma0)
    d.time_dt = time_step(d)
    d.time_current = 0.0
    d.time_total = 50000 * d.time_dt
    d.time_file_dt = d.time_total
    return d


def init_fluid_darcy(d: BinData, mu: float = 8.9e-4, rho_f: float = 1.0e3, p: float = 0.0,
                     k_c: float = 4.6e-10, beta_f: float = 4.5e-10, tolerance: float = 1.0e-3,
                     maxiter: int = 10000, ndem: int = 1, bottom_no_flow: bool = False) -> None:
    """``sim.initFluid(cfd_solver=1)`` (``python/sphere.py:3395-3508``):
    Darcy arrays on the sorting grid, periodic sides, Dirichlet top and
    bottom unless ``bottom_no_flow`` (``setFluidBottomNoFlow``, Neumann)."""
    nx, ny, nz = (int(v) for v in d.num)
    d.fluid = True
    d.cfd_solver = 1
    d.mu = mu
    d.rho_f = rho_f
    d.p_f = numpy.full((nx, ny, nz), p)
    d.v_f = numpy.zeros((nx, ny, nz, 3))
    d.phi = numpy.ones((nx, ny, nz))
    d.dphi = numpy.zeros((nx, ny, nz))
    d.p_mod_A = d.p_mod_f = d.p_mod_phi = 0.0
    d.bc_xn = d.bc_xp = d.bc_yn = d.bc_yp = 2
    d.bc_bot = 1 if bottom_no_flow else 0
    d.bc_top = 0
    d.free_slip_bot = d.free_slip_top = 1
    d.bc_bot_flux = d.bc_top_flux = 0.0
    d.p_f_constant = numpy.zeros((nx, ny, nz), dtype=numpy.int32)
    d.tolerance = tolerance
    d.maxiter = maxiter
    d.ndem = ndem
    d.c_phi = 1.0
    d.f_p = numpy.zeros((d.np, 3))
    d.beta_f = beta_f
    d.k_c = k_c


def init_fluid_ns(d: BinData, mu: float = 8.9e-4, rho_f: float = 1.0e3, p: float = 0.0,
                  hydrostatic: bool = False, tolerance: float = 1.0e-3, maxiter: int = 10000,
                  ndem: int = 1, beta: float = 0.0, theta: float = 1.0, gamma: float = 0.0,
                  c_v: float = 1.0, bc_bot: int = 0, bc_top: int = 0) -> None:
    """``sim.initFluid(cfd_solver=0)`` (``python/sphere.py:3395-3470``): the
    Navier-Stokes arrays on the sorting grid, with the solver settings of
    ``python/sphere.py:380-411``; ``hydrostatic`` sets the pressures below
    the top cells to ``p`` plus the weight of the fluid above them."""
    nx, ny, nz = (int(v) for v in d.num)
    d.fluid = True
    d.cfd_solver = 0
    d.mu = mu
    d.rho_f = rho_f
    d.p_f = numpy.full((nx, ny, nz), float(p))
    if hydrostatic:
        dz = d.L[2] / nz
        for iz in range(nz - 1):
            z = dz * iz + 0.5 * dz
            depth = d.L[2] - z
            d.p_f[:, :, iz] = p + (depth - dz) * rho_f * -d.g[2]
    d.v_f = numpy.zeros((nx, ny, nz, 3))
    d.phi = numpy.ones((nx, ny, nz))
    d.dphi = numpy.zeros((nx, ny, nz))
    d.p_mod_A = d.p_mod_f = d.p_mod_phi = 0.0
    d.bc_bot = bc_bot
    d.bc_top = bc_top
    d.free_slip_bot = d.free_slip_top = 1
    d.bc_bot_flux = d.bc_top_flux = 0.0
    d.p_f_constant = numpy.zeros((nx, ny, nz), dtype=numpy.int32)
    d.ns_gamma = gamma
    d.ns_theta = theta
    d.ns_beta = beta
    d.tolerance = tolerance
    d.maxiter = maxiter
    d.ndem = ndem
    d.c_phi = 1.0
    d.c_v = c_v
    d.dt_dem_fac = 1.0
    d.f_d = numpy.zeros((d.np, 3))
    d.f_p = numpy.zeros((d.np, 3))
    d.f_v = numpy.zeros((d.np, 3))
    d.f_sum = numpy.zeros((d.np, 3))


def _fcc_positions(n: int, d_nn: float, z0: float):
    """First n sites of a face-centred cubic lattice with nearest-neighbour
    distance d_nn, filled layer by layer from z0 upward in a square periodic
    cross-section; returns (x, nx_cells, a)."""
    a = d_nn * math.sqrt(2.0)
    nxc = max(2, int(math.ceil((n / 4.0) ** (1.0 / 3.0))))
    basis = numpy.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    nzc = int(math.ceil(n / (4.0 * nxc * nxc))) + 1
    iz, iy, ix = numpy.meshgrid(numpy.arange(nzc), numpy.arange(nxc), numpy.arange(nxc),
                                indexing="ij")
    cells = numpy.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(numpy.float64)
    sites = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    # fill by height (stable: equal heights keep lattice order)
    order = numpy.argsort(sites[:, 2], kind="stable")
    x = sites[order[:n]].copy()
    x[:, 2] += z0
    return x, nxc, a


def fcc_shear_box(n: int, seed: int, r_min: float = 0.009, r_max: float = 0.011,
                  sigma0: float = 20e3, shear_velocity: float = 1e-4, mu: float = 0.5,
                  k_n: float = 1.16e7, contactmodel: int = 2) -> BinData:
    """One shear box of the batched ensemble: n spheres (radii U(r_min,
    r_max)) on a face-centred cubic lattice whose nearest neighbours are
    2.002 r_max apart (a dense start without settling), periodic x/y, the
    sphere defaults with k_n = k_t, friction mu, gravity, then ``sim.shear``:
    fixed bottom layer, top layer at shear_velocity, a top wall at normal
    stress sigma0."""
    rng = numpy.random.default_rng(seed)
    d = BinData()
    _particles(d, n)
    d.radius = rng.uniform(r_min, r_max, size=n)
    x, nxc, a = _fcc_positions(n, 2.0 * r_max * 1.001, r_max * 1.001)
    d.x = x
    default_params(d, mu_s=mu, mu_d=mu, k_n=k_n, k_t=k_n)
    d.contactmodel = contactmodel
    d.g = numpy.array([0.0, 0.0, -9.81])
    side = nxc * a
    ncell = max(3, int(math.floor(side / (2.1 * r_max))))
    cell = side / ncell
    top = float(numpy.max(d.x[:, 2] + d.radius))
    nz = max(3, int(math.ceil(top * 1.05 / cell)))
    grid_for(d, L=[side, side, nz * cell], dx=cell)
    d.periodic = 1
    d.nw = 0
    init_temporal(d, total=1.0, file_dt=1.0)
    shear_setup(d, shear_velocity, sigma0)
    return d


def batch_shear_boxes(nbox: int = 256, seed: int = 7, n_min: int = 2000, n_max: int = 20000,
                      scale: float = 1.0):
    """The batched ensemble: nbox independent shear boxes with particle
    counts log-uniform in [n_min, n_max] (times scale), radii U(0.009,
    0.011) m, sigma0 from {10, 20, 40, 80, 160} kPa, shear velocity
    U(1e-5, 1e-3) m/s, k_n = k_t = 1.16e7 N/m, mu U(0.3, 0.6).  Returns
    (boxes, meta) with the drawn parameters per box."""
    rng = numpy.random.default_rng(seed)
    boxes, meta = [], []
    for b in range(nbox):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max))) * scale))
        n = max(n, 32)
        sigma0 = float(rng.choice([10e3, 20e3, 40e3, 80e3, 160e3]))
        vs = float(rng.uniform(1e-5, 1e-3))
        mu = float(rng.uniform(0.3, 0.6))
        boxes.append(fcc_shear_box(n, seed * 100003 + b, sigma0=sigma0, shear_velocity=vs, mu=mu))
        meta.append({"n": n, "sigma0": sigma0, "shear_velocity": vs, "mu": mu})
    return boxes, meta


def large_cohesive_packing(n: int = 4_000_000, seed: int = 4, layers=None,
                           r_median: float = 0.01, sigma_ln: float = 0.3,
                           r_lo: float = 0.004, r_hi: float = 0.03,
                           bond_factor: float = 1.05, v_max: float = 0.01) -> BinData:
    """The large polydisperse cohesive packing: n spheres with radii
    exp(N(ln r_median, sigma_ln)) clipped to [r_lo, r_hi], periodic x/y,
    the bottom wall at z = 0, gravity, Young's-modulus contact E = 7e8 Pa,
    mu = 0.5, and parallel bonds (stiffness k_n = k_t = 1e7, tensile
    strength 1e5 Pa, no shear limit, lambda_bar = 1) between every pair of
    initial neighbours closer than bond_factor x the radius sum.

    The start is dense without a settling run: radii are sorted (largest at
    the bottom) and placed in horizontal square lattices, one per layer,
    whose spacing W / cols is the smallest at or above the layer's largest
    diameter, so in-layer neighbours touch or nearly touch; each layer rests
    on the one below at the sum of the two layers' largest radii.  Nothing
    overlaps initially.  Bonds join in-layer lattice neighbours and the
    nearest sites of adjacent layers when they satisfy the distance
    criterion; pairs across the periodic faces are left unbonded (the bond
    law measures the direct distance).  Initial velocities are uniform in
    [-v_max, v_max] per axis (as in the settling lattice), so contacts form
    and bonds strain from the first steps."""
    rng = numpy.random.default_rng(seed)
    r = numpy.exp(rng.normal(math.log(r_median), sigma_ln, n)).clip(r_lo, r_hi)
    r = numpy.sort(r)[::-1].copy()
    if layers is None:
        # 150 layers at 4e6 spheres; smaller cuts keep the aspect ratio
        layers = max(3, int(round(150 * (n / 4.0e6) ** (1.0 / 3.0))))
    W = 2.0 * r_median * math.ceil(math.sqrt(n / layers))
    x = numpy.empty((n, 3))
    lay = []                                  # (start, count, cols, spacing, z)
    idx, z_prev, r_prev = 0, 0.0, 0.0
    while idx < n:
        rmax = float(r[idx])
        cols = max(3, int(W // (2.0 * rmax)))
        sp = W / cols
        cnt = min(cols * cols, n - idx)
        zc = rmax if not lay else z_prev + r_prev + rmax + 1e-7
        i = numpy.arange(cnt)
        x[idx:idx + cnt, 0] = (i % cols + 0.5) * sp
        x[idx:idx + cnt, 1] = (i // cols + 0.5) * sp
        x[idx:idx + cnt, 2] = zc
        lay.append((idx, cnt, cols, sp, zc))
        idx += cnt
        z_prev, r_prev = zc, rmax
    pairs = []
    for li, (st, cnt, cols, sp, zc) in enumerate(lay):
        i = numpy.arange(cnt)
        ix, iy = i % cols, i // cols
        for di, ok in ((1, ix + 1 < cols), (cols, iy + 1 < cols)):
            a = i[ok & (i + di < cnt)]
            b = a + di
            keep = sp < bond_factor * (r[st + a] + r[st + b])
            pairs.append(numpy.column_stack([st + a[keep], st + b[keep]]))
        if li == 0:
            continue
        # nearest sites of the layer below
        st0, cnt0, cols0, sp0, z0 = lay[li - 1]
        px, py = x[st:st + cnt, 0], x[st:st + cnt, 1]
        fx = numpy.floor(px / sp0 - 0.5).astype(numpy.int64)
        fy = numpy.floor(py / sp0 - 0.5).astype(numpy.int64)
        for ox in (0, 1):
            for oy in (0, 1):
                jx, jy = fx + ox, fy + oy
                j = jy * cols0 + jx
                ok = (jx >= 0) & (jx < cols0) & (jy >= 0) & (jy < cols0) & (j < cnt0)
                a = numpy.nonzero(ok)[0]
                jj = st0 + j[a]
                ii = st + a
                dist = numpy.sqrt(((x[ii] - x[jj]) ** 2).sum(axis=1))
                keep = dist < bond_factor * (r[ii] + r[jj])
                pairs.append(numpy.column_stack([jj[keep], ii[keep]]))
    bonds = numpy.concatenate(pairs).astype(numpy.uint32) if pairs else numpy.zeros((0, 2), numpy.uint32)

    d = BinData()
    _particles(d, n)
    d.x = x
    d.radius = r
    d.vel = rng.uniform(-v_max, v_max, size=(n, 3))
    default_params(d, mu_s=0.5, mu_d=0.5, k_n=1e7, k_t=1e7)
    d.E = 7e8
    d.g = numpy.array([0.0, 0.0, -9.81])
    cell = 2.1 * r_hi if r.max() <= r_hi else 2.1 * float(r.max())
    ncell = max(3, int(math.floor(W / cell)))
    top = float(numpy.max(x[:, 2] + r))
    nz = max(3, int(math.ceil(top * 1.1 / (W / ncell))))
    grid_for(d, L=[W, W, nz * (W / ncell)], dx=W / ncell)
    d.periodic = 1
    d.nw = 0
    d.nb0 = len(bonds)
    d.bonds = bonds
    d.bonds_delta_n = numpy.zeros(d.nb0)
    d.bonds_delta_t = numpy.zeros((d.nb0, 3))
    d.bonds_omega_n = numpy.zeros(d.nb0)
    d.bonds_omega_t = numpy.zeros((d.nb0, 3))
    d.lambda_bar = 1.0
    d.sigma_b = 1e5
    d.tau_b = numpy.inf
    init_temporal(d, total=1.0, file_dt=1.0)
    d.time_total = 5000 * d.time_dt
    d.time_file_dt = d.time_total
    return d
