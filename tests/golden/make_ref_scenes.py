"""Writes the input files of the reference's own invariant tests, built by the
reference's own ``sphere.sim`` class, into ``ref_scenes/``.

Each scene is set up exactly as the reference test sets it up before its
``run()`` call -- the same ``sim`` methods in the same order -- and written by
the reference's ``sim.writebin``:

- ``tests/contactmodel.py``, ``tests/contactmodel_young.py``: two-particle
  normal, viscous and oblique collisions (``cm_*``, ``cmy_*``);
- ``tests/contactmodel_wall.py``, ``tests/contactmodel_wall_young.py``: one
  particle against the bottom wall (``wall_*``, ``wally_*``);
- ``tests/io_tests.py``: the random grid of 100 particles (``io_initgrid``);
- ``tests/cfd_tests_darcy.py``: no forcing, pressure gradient, fast pressure
  modulation, pressure perturbation, top flux, gradient along x (``cfd_*``);
- ``tests/cfd_tests_darcy_particles.py``: steady states with 1000 particles
  under three boundary pairs, wall movement with ndem 1 and 10 and
  fluidisation at 0.9 and 2.0 times the fluidising gradient on the shipped
  ``cube-init`` packing (``dp_*``);
- ``tests/fluid_particle_interaction_darcy.py``: pressure-gradient and
  buoyancy forces on one particle (``fpi_*``).

The quantities each test takes from the ``sim`` object before its run (the
kinetic energy, the initial velocity, the wall position, the fluidising
pressure) are computed by the reference's own methods and stored in
``ref_scenes/manifest.json`` with the file's sid, its fluid flag and its step
count.  The files are stored gzip-compressed.

Run from the repository root where the reference tree is present:
``python tests/golden/make_ref_scenes.py``.  The reference's python code never
travels to the GPU machine; these files are what carries its set-up there.
"""
import gzip
import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "ref_scenes")
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from helpers import Count, import_reference_sphere  # noqa: E402
import oracle  # noqa: E402


def _fix(s):
    """sphere.py predates NumPy 2: its loops use range(self.np)."""
    s.np = numpy.asarray(s.np).reshape(-1)[:1].view(Count)
    return s


class Scenes:
    def __init__(self, sphere, workdir, out):
        self.sphere = sphere
        self.workdir = workdir
        self.out = out
        self.manifest = {}

    def new(self, *a, **k):
        return _fix(self.sphere.sim(*a, **k))

    def emit(self, name, s, **info):
        """Writes sim s as scene `name` with the reference's writebin."""
        s.writebin(folder="../input/", verbose=False)
        src = os.path.join(self.workdir, "input", str(s.sid) + ".bin")
        data = open(src, "rb").read()
        with gzip.GzipFile(os.path.join(self.out, name + ".bin.gz"), "wb", mtime=0) as f:
            f.write(data)
        dt = float(numpy.asarray(s.time_dt).reshape(-1)[0])
        total = float(numpy.asarray(s.time_total).reshape(-1)[0])
        entry = {"sid": str(s.sid), "fluid": bool(s.fluid), "np": int(s.np[0]),
                 "dt": dt, "total": total, "steps": int(round(total / dt)),
                 "sha256": hashlib.sha256(data).hexdigest()}
        entry.update({k: (float(v) if isinstance(v, (float, numpy.floating)) else v)
                      for k, v in info.items()})
        self.manifest[name] = entry


def _two_particles(S, name, r, z1, vel, young=False, gamma_n=None, mu=None, gamma_t=None):
    """tests/contactmodel.py (and _young.py): the set-up before each run."""
    orig = S.new(np=2, sid="contactmodeltest")
    orig.radius[:] = r
    orig.x[0, :] = [5.0, 5.0, 2.0]
    orig.x[1, :] = [5.0, 5.0, z1]
    for i, v in vel.items():
        orig.vel[0, i] = v
    if mu is not None:
        orig.mu_s[0] = mu
        orig.mu_d[0] = mu
    if gamma_t is not None:
        orig.gamma_t[0] = gamma_t
    orig.defineWorldBoundaries(L=[10, 10, 10])
    if young:
        orig.setYoungsModulus(7.0e9)
    orig.initTemporal(total=0.1, file_dt=0.01)
    if gamma_n is not None:
        orig.gamma_n[0] = gamma_n
    S.emit(name, orig, orig_vel0z=float(orig.vel[0, 2]),
           orig_ekin=float(orig.totalKineticEnergy()))


def contact_models(S, young):
    p = "cmy_" if young else "cm_"
    _two_particles(S, p + "elastic_1", [1.0, 1.0], 4.05, {2: 1}, young)
    _two_particles(S, p + "elastic_2", [2.0, 1.0], 5.05, {2: 1.0}, young)
    _two_particles(S, p + "elastic_3", [1.0, 2.0], 5.05, {2: 1.0}, young)
    _two_particles(S, p + "visc_1", [1.0, 1.0], 4.05, {2: 1}, young, gamma_n=1.0e6)
    _two_particles(S, p + "visc_2", [2.0, 1.0], 5.05, {2: 1.0}, young, gamma_n=1.0e6)
    _two_particles(S, p + "visc_3", [1.0, 2.0], 5.05, {2: 1.0}, young, gamma_n=1.0e6)
    _two_particles(S, p + "oblique_noslip", [1.0, 1.0], 4.05, {2: 1, 0: 1}, young, mu=1e9)
    _two_particles(S, p + "oblique_slip", [1.0, 1.0], 4.05, {2: 1, 0: 1}, young, mu=0.3)
    _two_particles(S, p + "oblique_slip_visc", [1.0, 1.0], 4.05, {2: 1, 0: 1}, young, mu=0.3,
                   gamma_t=1.0e3)


def wall_models(S, young):
    """tests/contactmodel_wall.py (and _young.py)."""
    p = "wally_" if young else "wall_"
    cases = [("elastic_normal", {2: -0.1}, 0.0, 0.0, 1.0),
             ("elastic_oblique", {2: -0.1, 0: 0.1}, 0.0, 0.0, 0.3),
             ("visc_normal", {2: -0.1}, 1.0e6, 0.0, 1.0),
             ("visc_oblique", {2: -0.1, 0: 0.1}, 1.0e6, 1.0e6, 1.0)]
    for tag, vel, gwn, gwt, total in cases:
        orig = S.new(np=1, nw=0, sid="contactmodeltest")
        orig.radius[:] = 1.0
        orig.x[0, :] = [5.0, 5.0, 1.05]
        for i, v in vel.items():
            orig.vel[0, i] = v
        orig.defineWorldBoundaries(L=[10, 10, 10])
        if young:
            orig.setYoungsModulus(7.0e9)
        orig.gamma_wn[0] = gwn
        orig.gamma_wt[0] = gwt
        orig.initTemporal(total=total, file_dt=0.01)
        S.emit(p + tag, orig, orig_ekin=float(orig.energy("kin")),
               orig_ekin_total=float(orig.totalKineticEnergy()))


def io_tests(S):
    """tests/io_tests.py:9-18."""
    numpy.random.seed(20)  # the reference test draws unseeded; any draw is an instance
    orig = S.new(np=100, nw=1, sid="test-initgrid")
    orig.generateRadii(histogram=False)
    orig.defaultParams()
    orig.g[2] = 0.0
    orig.initRandomGridPos()
    orig.initTemporal(current=0.0, total=0.0)
    orig.time_total = 2.0 * orig.time_dt
    orig.time_file_dt = orig.time_dt
    S.emit("io_initgrid", orig)


def cfd_darcy(S):
    """tests/cfd_tests_darcy.py."""
    orig = S.new(np=0, nd=3, nw=0, sid="cfdtest", fluid=True)
    orig.defaultParams()
    orig.defineWorldBoundaries([0.4, 0.3, 0.4], dx=0.1)
    orig.initFluid(cfd_solver=1)
    orig.initTemporal(total=0.2, file_dt=0.01, dt=1.0e-7)
    orig.time_file_dt = orig.time_dt * 0.99
    orig.time_total = orig.time_dt * 10
    S.emit("cfd_no_forcing", orig)
    orig.p_f[:, :, -1] = 1.0
    orig.initTemporal(total=0.5, file_dt=0.01, dt=1.0e-6)
    ideal = numpy.linspace(orig.p_f[0, 0, 0], orig.p_f[0, 0, -1], int(orig.num[2]))
    S.emit("cfd_pressure_gradient", orig, ideal_p_z=[float(v) for v in ideal])
    orig.time_total[0] = 1.0e-2
    orig.time_file_dt[0] = 0.101 * orig.time_total[0]
    orig.setFluidPressureModulation(A=1.0, f=1.0 / orig.time_total[0])
    S.emit("cfd_fast_modulation", orig)

    orig = S.new(np=0, nd=3, nw=0, sid="cfdtest", fluid=True)
    orig.defaultParams()
    orig.defineWorldBoundaries([1.0, 1.0, 1.0], dx=0.1)
    orig.initFluid(cfd_solver=1)
    orig.initTemporal(total=0.2, file_dt=0.01, dt=1.0e-7)
    orig.time_file_dt = orig.time_dt * 0.99
    orig.time_total = orig.time_dt * 10
    orig.p_f[4, 2, 5] = 2.0
    S.emit("cfd_pressure_perturbation", orig)

    orig = S.new(np=0, nd=3, nw=0, sid="cfdtest", fluid=True)
    orig.defaultParams()
    orig.defineWorldBoundaries([1.0, 1.0, 1.0], dx=0.1)
    orig.initFluid(cfd_solver=1)
    orig.initTemporal(total=0.2, file_dt=0.01, dt=1.0e-7)
    orig.time_file_dt = orig.time_dt * 0.99
    orig.time_total = orig.time_dt * 10
    orig.setFluidTopFixedFlux(1.0)
    S.emit("cfd_flux_top", orig)
    orig.p_f[:, :, :] = 0.0
    orig.p_f[0, :, :] = 2.0
    orig.setFluidXFixedPressure()
    orig.setFluidYNoFlow()
    orig.setFluidTopNoFlow()
    orig.setFluidBottomNoFlow()
    orig.initTemporal(total=0.5, file_dt=0.01, dt=1.0e-6)
    S.emit("cfd_gradient_x", orig)


def _cube_init(S):
    """sphere.sim('cube-init').readlast() on the shipped packing.  The
    reader passes 1-element arrays as counts, which NumPy 2 refuses; they are
    turned into integers for the duration of the call."""
    orig = S.new("cube-init", fluid=False)
    fromfile = numpy.fromfile

    def _fromfile(*a, count=-1, **k):
        return fromfile(*a, count=int(numpy.asarray(count).reshape(-1)[0]), **k)

    numpy.fromfile = _fromfile
    try:
        orig.readlast(verbose=False)
    finally:
        numpy.fromfile = fromfile
    return _fix(orig)


def darcy_particles(S):
    """tests/cfd_tests_darcy_particles.py."""
    numpy.random.seed(21)  # the reference test draws unseeded; any draw is an instance
    for tag, bot_noflow, top_noflow in (("dp_steady_dd", False, False),
                                        ("dp_steady_nd", True, False),
                                        ("dp_steady_nn", True, True)):
        orig = S.new("darcy_particles", np=1000)
        orig.defaultParams()
        orig.generateRadii(psd="uni", mean=5.0e-2, variance=5.0e-5)
        orig.initRandomGridPos([20, 20, 200])
        orig.initTemporal(total=0.005, file_dt=0.001)
        orig.initFluid(cfd_solver=1)
        orig.k_c[0] = 4.6e-10
        if bot_noflow:
            orig.setFluidBottomNoFlow()
        if top_noflow:
            orig.setFluidTopNoFlow()
        orig.setStiffnessNormal(36.4e9)
        orig.setStiffnessTangential(36.4e9 / 3.0)
        S.emit(tag, orig)

    for tag, ndem in (("dp_wall_ndem1", None), ("dp_wall_ndem10", 10)):
        orig = _cube_init(S)
        orig.num[2] /= 2
        orig.L[2] /= 2.0
        orig.id("darcy_fluidization")
        orig.setStiffnessNormal(36.4e9)
        orig.setStiffnessTangential(36.4e9 / 3.0)
        orig.initTemporal(total=0.0005, file_dt=0.0001)
        orig.initFluid(cfd_solver=1)
        if ndem:
            orig.setDEMstepsPerCFDstep(ndem)
        orig.setFluidBottomNoFlow()
        orig.g[2] = -10.0
        orig.consolidate()
        S.emit(tag, orig, orig_w_x0=float(orig.w_x[0]))

    orig = _cube_init(S)
    orig.num[2] /= 2
    orig.L[2] /= 2.0
    orig.id("darcy_fluidization")
    orig.setDEMstepsPerCFDstep(1)
    orig.setStiffnessNormal(36.4e9)
    orig.setStiffnessTangential(36.4e9 / 3.0)
    orig.initTemporal(total=0.0005, file_dt=0.0001)
    orig.initFluid(cfd_solver=1)
    orig.g[2] = -10.0
    mean_porosity = orig.bulkPorosity()
    fluidize_pressure = numpy.abs((orig.rho - orig.rho_f) * (1.0 - mean_porosity)
                                  * numpy.abs(orig.g[2]))
    for factor in (0.9, 2.0):
        orig.id("fluidization-" + str(factor))
        dpdz = factor * fluidize_pressure
        dp = dpdz * orig.L[2]
        orig.p_f[:, :, 0] = 0.0 + dp
        orig.p_f[:, :, -1] = 0.0
        S.emit(f"dp_fluidization_{factor}", orig, factor=factor,
               fluidize_pressure=float(numpy.asarray(fluidize_pressure).reshape(-1)[0]))


def fluid_particle_interaction(S):
    """tests/fluid_particle_interaction_darcy.py."""
    sim = S.new("fluid_particle_interaction", fluid=True)
    sim.defineWorldBoundaries([1.0, 1.0, 1.0], dx=0.1)
    sim.initFluid(cfd_solver=1)
    sim.p_f[:, :, -1] = 1.0
    sim.addParticle([0.55, 0.55, 0.55], 0.05)
    _fix(sim)
    sim.initTemporal(total=0.001, file_dt=0.0001)
    S.emit("fpi_pressure_gradient", sim)

    sim = S.new("fluid_particle_interaction", fluid=True)
    sim.defineWorldBoundaries([1.0, 1.0, 1.0], dx=0.1)
    sim.initFluid(cfd_solver=1)
    sim.p_f[:, :, -1] = 0.0
    sim.addParticle([0.5, 0.5, 0.5], 0.01)
    _fix(sim)
    sim.initTemporal(total=0.001, file_dt=0.0001)
    sim.g[2] = -10.0
    S.emit("fpi_buoyancy", sim)


def main(out=OUT):
    sphere = import_reference_sphere()
    ref_out = oracle.ref_path("output")
    if ref_out is None:
        raise SystemExit("the reference tree is not present")
    os.makedirs(out, exist_ok=True)
    work = tempfile.mkdtemp()
    for sub in ("python", "input", "output"):
        os.makedirs(os.path.join(work, sub))
    for f in ("cube-init.output00029.bin", "cube-init.status.dat"):
        shutil.copy(os.path.join(ref_out, f), os.path.join(work, "output", f))
    cwd = os.getcwd()
    os.chdir(os.path.join(work, "python"))
    try:
        S = Scenes(sphere, work, out)
        contact_models(S, young=False)
        contact_models(S, young=True)
        wall_models(S, young=False)
        wall_models(S, young=True)
        io_tests(S)
        cfd_darcy(S)
        darcy_particles(S)
        fluid_particle_interaction(S)
    finally:
        os.chdir(cwd)
        shutil.rmtree(work)
    with open(os.path.join(out, "manifest.json"), "w") as f:
        json.dump(S.manifest, f, indent=1, sort_keys=True)
    return S.manifest


if __name__ == "__main__":
    for k, v in main().items():
        print(f"{k:28s} np={v['np']:5d} steps={v['steps']:7d} fluid={v['fluid']}")
