"""Drop-in for sphere's ``sim.run()`` (python/sphere.py:4482-4540).

The reference's ``run`` writes ``../input/<sid>.bin`` with ``sim.writebin``
and then runs ``cd ..; ./sphere [-q] [--dry] [--fluid] [-d N]
input/<sid>.bin`` in a shell.  :func:`run` keeps that signature and those
paths but calls the GPU engine in-process through the C ABI: the same input
file is read, and the same outputs appear under ``../output/``
(``<sid>.output%05d.bin``, ``<sid>.status.dat``, ``<sid>-conv.log`` with
fluid).  As in the reference, a failing run prints a warning with the status
instead of raising.

:func:`install` patches an unmodified ``sphere.sim`` class::

    import sphere, sphere_b200.sim
    sphere_b200.sim.install(sphere.sim)
    sb = sphere.sim("shear", np=100000)
    ...
    sb.run()            # now runs on the B200 engine
"""
import os
import sys
import warnings

from . import binfile

# engine options a caller may set on the sim object before run()
_OPTION_ATTRS = {
    "b200_precision": "precision",      # "faithful" | "fp64" | "mixed"
    "b200_integrator": "integrator",    # 3 (TY3) | 2 (TY2)
    "b200_capacity": "capacity",        # contact slots per particle
    "b200_warm_start": "warm_start",    # learned Darcy warm start
}


def report_values(d: binfile.BinData, verbose: bool = True, out=None) -> str:
    """The summary the reference's ``--dry`` run prints
    (``DEM::reportValues``, src/sphere.cpp:349-470), as text."""
    lines = [f"  - Number of dimensions: nd = {d.nd}",
             f"  - Number of particles:  np = {d.np}",
             "  - Compiled for double precision" if verbose else "  - Compiled for  precision",
             f"  - Timestep length:      time.dt         = {float(d.time_dt):g} s",
             f"  - Start at time:        time.current    = {float(d.time_current):g} s",
             f"  - Total sim. time:      time.total      = {float(d.time_total):g} s",
             f"  - File output interval: time.file_dt    = {float(d.time_file_dt):g} s",
             f"  - Start at step count:  time.step_count = {int(d.time_step_count)}"]
    cm = int(d.contactmodel)
    lines.append({1: "  - Contact model: Linear-elastic-viscous (n), visco-frictional (t)",
                  2: "  - Contact model: Linear-elastic-visco-frictional",
                  3: "  - Contact model: Nonlinear-elastic-visco-frictional"}.get(
                      cm, f"Error: Contact model value ({cm}) not understood."))
    if float(d.E) > 0.01:
        lines.append("  - Using Young's modulus for contact stiffness")
    else:
        lines.append("  - Using global value for contact stiffness")
    if float(d.kappa) > 0.0 and float(d.V_b) > 0.0:
        lines.append("  - Capillary cohesion enabled")
    lines.append(f"  - Number of dynamic walls: {int(d.nw)}")
    per = int(d.periodic)
    if per == 1:
        lines.append("  - 1st and 2nd dim. boundaries: Periodic")
    elif per == 2:
        lines.append("  - 1st dim. boundaries: Visco-frictional walls")
    else:
        lines.append("  - 1st and 2nd dim. boundaries: Visco-frictional walls")
    if d.fluid:
        lines.append("  - Fluid: Darcy (cfd_solver 1)" if int(d.cfd_solver) == 1
                     else "  - Fluid: Navier-Stokes (cfd_solver 0)")
    lines.append(f"  - Grid: {int(d.num[0])} x {int(d.num[1])} x {int(d.num[2])} cells")
    text = "\n".join(lines) + "\n"
    (out or sys.stdout).write(text)
    return text


def run(self, verbose=True, hideinputfile=False, dry=False, valgrind=False,
        cudamemcheck=False, device=-1):
    """``sim.run`` on the GPU engine; same arguments as the reference.

    ``valgrind`` and ``cudamemcheck`` wrapped the reference binary in a
    checker; they are accepted and ignored with a warning.  ``hideinputfile``
    silenced the binary's stdout; here it silences the dry-run report.
    """
    from .engine import Engine, EngineError, check_file

    self.writebin(verbose=False)
    if valgrind or cudamemcheck:
        warnings.warn("valgrind/cudamemcheck wrap the reference binary; ignored by the "
                      "B200 engine", RuntimeWarning, stacklevel=2)
    path = os.path.join("..", "input", self.sid + ".bin")
    fluid = bool(getattr(self, "fluid", False))
    opts = {v: getattr(self, k) for k, v in _OPTION_ATTRS.items() if hasattr(self, k)}
    status = 0
    if dry:
        # read, checkValues, report, exit (src/sphere.cpp:46-51); no device
        status, msg = check_file(path, fluid)
        if status:
            print(f"Error: {msg}")
        elif not hideinputfile:
            report_values(binfile.read_bin(path, fluid=fluid), verbose=bool(verbose))
    else:
        try:
            os.makedirs(os.path.join("..", "output"), exist_ok=True)
            with Engine(path, fluid=fluid, device=int(device), verbose=bool(verbose),
                        output_dir=os.path.join("..", "output"), **opts) as eng:
                status = eng.run()
        except EngineError as exc:
            print(f"Error: {exc}")
            status = exc.status
    if status != 0:
        print("Warning: the sphere run returned with status " + str(status))
    return status


def install(sim_class):
    """Replaces ``sim_class.run`` by :func:`run`; the reference's method stays
    reachable as ``sim_class.run_reference``.  Returns the class."""
    if getattr(sim_class, "run", None) is not run:
        sim_class.run_reference = sim_class.run
        sim_class.run = run
    return sim_class


def uninstall(sim_class):
    """Restores the reference's ``run``."""
    if getattr(sim_class, "run", None) is run and hasattr(sim_class, "run_reference"):
        sim_class.run = sim_class.run_reference
        del sim_class.run_reference
    return sim_class
