"""Generates the golden fixtures in this directory from the reference itself.

The reference's own kernels (sorting.cuh, contactsearch.cuh,
contactmodels.cuh, cohesion.cuh, integration.cuh), compiled for the host by
oracle/Makefile into oracle/_ref, run each seeded input below; the input .bin
and the reference's state after the listed steps are stored as
<case>.bin + <case>.npz.  Run from the repository root where the reference
tree is present:  python tests/golden/make_golden.py  (with the argument
`ns`, only the Navier-Stokes fixture is made).
"""
import os
import sys

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from sphere_b200 import binfile, configs  # noqa: E402
import oracle as O  # noqa: E402

FIELDS = ("x", "vel", "angvel", "angpos", "force", "torque", "xyzsum", "acc", "angacc",
          "es_dot", "es", "ev_dot", "ev", "p", "cellid", "index", "contacts", "delta_t",
          "walls_nx", "walls_mvfd")
STEPS = (1, 5, 20)


def cases():
    d = configs.settling_lattice(n=300, seed=11, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    yield "dense_model2", d
    d = configs.settling_lattice(n=300, seed=12, nx=7, ny=7, nz=7, spacing=0.0195, steps=40,
                                 contactmodel=1)
    d.gamma_n = 30.0
    d.gamma_t = 10.0
    yield "dense_model1", d
    d = configs.settling_lattice(n=320, seed=13, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    configs.shear_setup(d, 0.05, 20e3)
    d.w_x[0] -= 0.002
    d.E = 7e8
    yield "shear_young", d
    d = configs.settling_lattice(n=300, seed=14, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    d.periodic = 0
    d.gamma_n = 20.0
    yield "walls_nonperiodic", d


DARCY_FIELDS = ("darcy_p", "darcy_phi", "darcy_k", "darcy_v", "darcy_f_p", "darcy_nijac_last",
                "x", "vel", "force")


def darcy_cases():
    d = configs.settling_lattice(n=300, seed=15, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    configs.add_top_wall(d, 10e3)
    d.w_x[0] -= 0.002
    configs.init_fluid_darcy(d, mu=1.797e-6, k_c=3.5e-13, tolerance=1e-8, maxiter=2000,
                             bottom_no_flow=True)
    yield "darcy_consolidation", d


NS_FIELDS = ("ns_p", "ns_phi", "ns_dphi", "ns_v", "ns_v_face", "ns_epsilon", "ns_norm", "ns_f_d",
             "ns_f_p", "ns_f_v", "ns_f_sum", "ns_nijac_last", "x", "vel", "force")


def ns_cases():
    """Navier-Stokes (cfd_solver 0): a settling box under a stress-controlled
    wall in a hydrostatic fluid (navierstokes.cuh, device.cu:1213-1898)."""
    d = configs.settling_lattice(n=300, seed=16, nx=7, ny=7, nz=7, spacing=0.0195, steps=40)
    configs.add_top_wall(d, 10e3)
    d.w_x[0] -= 0.002
    configs.init_fluid_ns(d, mu=8.9e-4, hydrostatic=True, tolerance=1e-6, maxiter=2000)
    yield "ns_settling", d


def make_ns():
    for name, d in ns_cases():
        path = os.path.join(HERE, f"{name}.bin")
        binfile.write_bin(d, path)
        ref = O.Reference(path, fluid=True)
        out = {}
        for s in (1, 2, 3):
            ref.step(1)
            for f in NS_FIELDS:
                out[f"{f}@{s}"] = ref.get(f)
        ref.close()
        numpy.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "written")


def main():
    O.build(ref=True)
    if sys.argv[1:] == ["ns"]:
        make_ns()
        return
    make_ns()
    for name, d in darcy_cases():
        path = os.path.join(HERE, f"{name}.bin")
        binfile.write_bin(d, path)
        ref = O.Reference(path, fluid=True)
        out = {}
        for s in (1, 2, 3):
            ref.step(1)
            for f in DARCY_FIELDS:
                a = ref.get(f)
                if f == "force":
                    a = a[:, :3]
                out[f"{f}@{s}"] = a
        ref.close()
        numpy.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "written")
    for name, d in cases():
        path = os.path.join(HERE, f"{name}.bin")
        binfile.write_bin(d, path)
        ref = O.Reference(path)
        out = {}
        done = 0
        for s in STEPS:
            ref.step(s - done)
            done = s
            for f in FIELDS:
                a = ref.get(f)
                if f in ("angvel", "angpos", "force", "torque", "xyzsum", "acc", "angacc"):
                    a = a[:, :3]
                out[f"{f}@{s}"] = a
        ref.close()
        numpy.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "written")


if __name__ == "__main__":
    main()
