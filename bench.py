#!/usr/bin/env python
"""Benchmark of the DEM step: particle-steps/s on one B200.

Workload: the dense-shear configuration -- N = 100,000 spheres, radii
U(0.008, 0.012) m, settled packing, fixed bottom layer, top layer sheared at
1e-4 m/s along x, top wall at sigma0 = 20 kPa, Young's modulus contact
E = 7e8 Pa, mu = 0.5, periodic x/y (seeded synthetic data).

One benchmark "step" is one output interval of INTERVAL DEM time steps (the
unit `sim.run()` advances between two output files).  `value` is
N * DEM steps / device time with the state resident on the GPU, for the
mixed-precision engine by default (its force error against FP64 is measured
in the same run and reported); the plain FP64 drop-in engine is timed in the
same run and reported beside it as `fp64_plain`.  `e2e` is the
same metric through the C ABI with host buffers: every interval uploads the
particle state (positions, velocities, angular velocities) from pinned host
memory, advances INTERVAL DEM steps and reads the state back (positions,
velocities, angular velocities, forces, torques).

`python bench.py --impl reference` times the reference algorithm on the host
cores instead, on a bounded sample of the same workload: the reference's own
kernels compiled for the host (oracle/_ref, one thread; sphere has no CPU DEM
path of its own), or where that build is absent the CPU restatement of the
reference's step (the oracle, OpenMP over all host threads).  The engine's
line carries the latter as `cpu_baseline`.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

INTERVAL = 100          # DEM steps per benchmark step
N_PARTICLES = 100000
# dram__bytes_read.sum + dram__bytes_write.sum of one k_contacts<2,2> launch
# on this workload (mixed precision, N = 1e5), from an ncu --set full
# capture of that kernel: 46.30 MB read + 3.15 MB written (ncu flushes the
# caches before the launch)
CONTACTS_TRAFFIC = 46.30e6 + 3.15e6
# the same for one k_contacts_integrate<2,2> launch (contacts and
# integration in one launch): 43.62 MB read + 10.41 MB written
FUSED_TRAFFIC = 43.62e6 + 10.41e6
SEED = 1


def log(msg):
    print(msg, file=sys.stderr, flush=True)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=0):
        self.samples = []
        self.proc = None
        self.dev = device_index
        self._thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self._thread = threading.Thread(target=self._read, daemon=True)
        self._thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self._thread:
            self._thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
                for i, nm in enumerate(names):
                    if s[5 + i].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(numpy.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(n):
    """The dense-shear workload.  At the benchmark size the settled packing
    is the packaged fixture (sphere_b200/data), so neither arm settles
    anything and the CPU reference arm never touches the GPU engine."""
    from sphere_b200 import configs
    return configs.shear_benchmark(n=n, seed=SEED, log=log)


def workload_config(n):
    """The `config` of both arms' JSON lines: the same workload and the same
    DEM steps per benchmark step."""
    return {"workload": f"dense dry shear, N={n}, radii U(0.008,0.012) m, E=7e8 Pa, "
                        f"mu=0.5, sigma0=20 kPa, shear 1e-4 m/s, periodic x/y",
            "dem_steps_per_step": INTERVAL}


def step_path_name(info):
    """The step path the engine ran (sph_info.step_path)."""
    return {1: "persistent", 2: "per-stage, contacts and integration in one launch"}.get(
        int(info.step_path), "per-stage")


def mean_contacts(eng, n):
    c = eng.get("contacts")
    return float((c != n).sum()) / n


def flush_l2(buf):
    buf.add_(1.0)


def measure(d, precision, args, flush):
    """Device-timed throughput of one precision mode on workload d."""
    import torch
    from sphere_b200.engine import Engine

    n = d.np
    eng = Engine(d, precision=precision, graph_steps=INTERVAL, step_kernel=args.step_kernel)
    for _ in range(args.warmup):
        eng.step(INTERVAL)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        # CUDA events on the engine's stream around the INTERVAL steps
        times.append(eng.step_timed(INTERVAL) * 1e-3)
    step_s = float(numpy.sum(times))
    return eng, {"value": n * INTERVAL * args.steps / step_s,
                 "ms_per_step": 1e3 * step_s / args.steps}


def shear_report(d, eng, info):
    """The shear test's observables after the steps run so far: the
    effective shear stress (python/sphere.py:6406-6432: minus the x forces
    on the fixed particles moving in +x, over the top area) and the dilation
    in mean particle diameters (:6786-6810)."""
    vel = eng.get("vel")
    force = eng.get("force")
    moving = (vel[:, 3] > 0.0) & (vel[:, 0] > 0.0)
    tau = float(-force[moving, 0].sum() / (d.L[0] * d.L[1]))
    w_x = float(eng.get("walls_nx")[0, 3])
    d_bar = float(numpy.mean(d.radius) * 2.0)
    return {"dem_steps": int(info.iter), "shear_stress_pa": tau,
            "dilation_mean_diameters": (w_x - float(d.w_x[0])) / d_bar}


HISTORY_STEPS = 1000


def force_error(d, history_steps=HISTORY_STEPS):
    """Normwise relative force error of the mixed mode against FP64,
    ||F_mixed - F_fp64|| / ||F_fp64||, after one step from the same sheared
    state: the workload is first sheared for history_steps FP64 steps, so the
    contacts carry developed tangential displacements (the FP32 history path
    of the mixed contact law contributes); positions, velocities, walls,
    contact rows and histories are then copied into fresh FP64 and mixed
    engines, which take one step each.  Returns (error, mean occupied slots
    with a non-zero history per particle)."""
    from sphere_b200.engine import Engine
    fields = ("x", "vel", "angvel", "walls_nx", "walls_mvfd", "contacts", "delta_t")
    with Engine(d, precision="fp64") as e:
        e.step(history_steps)
        state = {f: e.get(f) for f in fields}
    out = {}
    for prec in ("fp64", "mixed"):
        with Engine(d, precision=prec) as e:
            for f in fields:
                e.set(f, state[f])
            e.step(1)
            out[prec] = e.get("force")[:, :3]
    a, b = out["mixed"], out["fp64"]
    live = float((numpy.abs(state["delta_t"][:, :3]).sum(axis=1) > 0).sum()) / d.np
    return float(numpy.linalg.norm(a - b) / numpy.linalg.norm(b)), live


def run_gpu(args):
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n = args.particles
    d = workload(n)
    precision = args.precision
    # L2 flush buffer (256 MB, larger than the 126 MB L2)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    # ---- the plain FP64 drop-in (faithful arithmetic), for comparison ----
    plain = None
    if precision != "faithful":
        e_plain, plain = measure(d, "faithful", args, flush)
        e_plain.close()

    # ---- headline mode, device-resident timing: value ----
    sampler = ClockSampler()
    sampler.start()
    torch.cuda.cudart().cudaProfilerStart()   # a profiler captures the timed region only
    eng, head = measure(d, precision, args, flush)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    clocks = sampler.stop()
    value = head["value"]
    zbar = mean_contacts(eng, n)

    # ---- per-kernel timing with CUDA events (on the engine's stream) ----
    prof = eng.profile(200)

    # ---- end to end through the C ABI with pinned host buffers ----
    x = torch.empty((n, 4), dtype=torch.float64).pin_memory()
    vel = torch.empty((n, 4), dtype=torch.float64).pin_memory()
    angvel = torch.empty((n, 4), dtype=torch.float64).pin_memory()
    force = torch.empty((n, 4), dtype=torch.float64).pin_memory()
    torque = torch.empty((n, 4), dtype=torch.float64).pin_memory()
    xa, va, aa, fa, ta = (t.numpy() for t in (x, vel, angvel, force, torque))
    eng.get("x", xa); eng.get("vel", va); eng.get("angvel", aa)
    e2e_times = []
    for _ in range(max(3, args.steps // 2)):
        flush_l2(flush)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.set("x", xa); eng.set("vel", va); eng.set("angvel", aa)
        eng.step(INTERVAL)
        eng.get("x", xa); eng.get("vel", va); eng.get("angvel", aa)
        eng.get("force", fa); eng.get("torque", ta)
        t1 = time.perf_counter()
        e2e_times.append(t1 - t0)
    e2e_value = n * INTERVAL * len(e2e_times) / float(numpy.sum(e2e_times))
    info = eng.info()
    shear = shear_report(d, eng, info)
    eng.close()

    peak, peak_kind = load_peaks()
    # algorithmic bytes of the contact kernel per particle (plain FP64 field
    # widths): sorted pos+r, vel, angvel read 80; force+torque write 48;
    # es_dot, ev_dot, p write 24; es, ev read+write 32; per occupied slot
    # partner id 4 + tangential history 24, read and written (56)
    bytes_per_particle = 184.0 + 56.0 * zbar
    kernel_name = "k_contacts (contact search + forces)"
    traffic = CONTACTS_TRAFFIC if precision == "mixed" else None
    if info.step_path == 2:
        # contacts and integration in one launch: the integration's own
        # fields (fixvel 8; angpos, acc0, angacc0, xyzsum read 96; pos, vel,
        # angvel, angpos, acc, angacc, xyzsum written 168) come on top; its
        # reads of force, torque, pos, vel and angvel are gone
        bytes_per_particle += 272.0
        kernel_name = "k_contacts_integrate (contact search + forces + integration)"
        traffic = FUSED_TRAFFIC if precision == "mixed" else None
    contacts_bytes = n * bytes_per_particle
    achieved = contacts_bytes / (prof.contacts_ms * 1e-3) / 1e9
    # launches of this library's kernels in the timed region: per DEM step
    # k_resort (with the list rebuild), k_contacts, k_integrate (+2 for the
    # shear-stress wall, +2 with bonds) on the per-stage path; k_resort,
    # k_contacts_integrate and k_walls_step with contacts and integration in
    # one launch; one k_persistent per call on the persistent path
    if info.step_path == 1:
        timed_launches = args.steps
    elif info.step_path == 2:
        timed_launches = 3 * INTERVAL * args.steps
    else:
        per_step = 3 + (2 if d.nw > 0 and d.wmode[0] == 3 else 0) + (2 if d.nb0 > 0 else 0)
        timed_launches = per_step * INTERVAL * args.steps
    out = {
        "metric": "particle-steps/s",
        "value": value,
        "unit": "particle-steps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"faithful": "f64", "fp64": "f64", "mixed": "f32+f64"}[precision],
        "data": "synthetic (seeded settled packing)",
        "config": workload_config(n),
        "engine": {"precision": precision, "integrator": "TY3",
                   "mean_contacts_per_particle": zbar,
                   "l2": "flushed between timed steps (256 MB write)"},
        "e2e": {"value": e2e_value, "unit": "particle-steps/s",
                "h2d_bytes_per_step": 3 * 32 * n, "d2h_bytes_per_step": 5 * 32 * n},
        "gpu_launches": timed_launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": traffic,
                     "traffic_unit": "DRAM bytes per launch (ncu, cold caches)",
                     "kernel": kernel_name,
                     "bytes_per_particle": bytes_per_particle,
                     "peak_source": peak_kind},
        "stage_ms_per_dem_step": {"resort": prof.resort_ms, "contacts": prof.contacts_ms,
                                  "bonds": prof.bonds_ms, "integrate": prof.integrate_ms,
                                  "step": prof.step_ms},
        "resorts": int(info.resorts),
        "shear_observables": shear,
        "step_path": {"kernel": step_path_name(info),
                      "threads": int(info.step_threads), "grid": int(info.step_grid),
                      "autotuned": bool(info.tuned)},
        "clocks": clocks,
    }
    if plain is not None:
        out["fp64_plain"] = {"value": plain["value"], "ms_per_step": plain["ms_per_step"],
                             "speedup_of_headline": value / plain["value"]}
    if precision == "mixed":
        err, live = force_error(d)
        out["force_rel_err_vs_fp64"] = err
        out["force_err_state"] = {"history_steps": HISTORY_STEPS,
                                  "slots_with_tangential_history_per_particle": live}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(d, sample_steps=args.cpu_steps)
    if args.darcy_steps > 0:
        out["darcy"] = darcy_leg(args)
    if args.batch_boxes > 0:
        out["batch"] = batch_leg(args)
    if args.large_particles > 0:
        out["large"] = large_leg(args)
    if args.settle_steps > 0:
        out["settle"] = settle_leg(args)
    if args.render:
        out["render"] = render_leg(args, d)
    if args.ns_steps > 0:
        out["navier_stokes"] = ns_leg(args)
    return out


def darcy_leg(args):
    """Darcy-coupled consolidation (40 x 40 x 80 fluid grid, residual
    tolerance 1e-8, top wall stepped 10 -> 20 -> 40 -> 80 kPa): Jacobi
    iterations per fluid step from the previous solution (the reference),
    with the learned warm start, and with its extrapolation alone.  The
    network trains online from the first solve; the comparison uses the
    second half of the steps, exact iteration counts (the first iteration
    whose residual met the tolerance) and the reference's own count (checks
    every 10 iterations)."""
    from sphere_b200 import configs
    from sphere_b200.engine import Engine
    d = configs.darcy_benchmark(n=args.particles, seed=SEED, log=log)
    steps = args.darcy_steps
    loads = [10e3, 20e3, 40e3, 80e3]
    arms = {}
    names = {0: "plain", 1: "warm", 2: "extrapolation"}
    for warm in (0, 1, 2):
        eng = Engine(d, fluid=True, precision="mixed", warm_start=warm)
        mv = eng.get("walls_mvfd")
        exact, quant, ms = [], [], []
        for s in range(steps):
            load = loads[min(len(loads) - 1, s * len(loads) // steps)]
            if mv[0, 3] != load:
                mv[0, 3] = load
                eng.set("walls_mvfd", mv)
            ms.append(eng.step_timed(1))
            exact.append(int(eng.get("darcy_iters_exact")[0]))
            quant.append(int(eng.get("darcy_iters")[0]) + 1)
        stats = eng.get("darcy_warm")
        eng.close()
        h = steps // 2
        arms[names[warm]] = {
            "iters_exact_per_step": float(numpy.mean(exact[h:])),
            "iters_per_step": float(numpy.mean(quant[h:])),
            "ms_per_fluid_step": float(numpy.mean(ms[h:])),
            "predictions": int(stats[0]), "trained": int(stats[1]), "used_network_guess": int(stats[2]),
        }
        log(f"darcy {names[warm]}: {arms[names[warm]]}")
    p, w, x = arms["plain"], arms["warm"], arms["extrapolation"]
    return {
        "workload": f"Darcy consolidation, N={d.np}, fluid grid {int(d.num[0])}x{int(d.num[1])}x{int(d.num[2])}, "
                    "mu_f=1.797e-6 Pa s, k_c=3.5e-13 m^2, beta_f=4.5e-10 1/Pa, tolerance 1e-8, "
                    "top wall 10->20->40->80 kPa",
        "steps": steps, "measured_steps": steps - steps // 2,
        "iters_per_step_plain": p["iters_exact_per_step"],
        "iters_per_step_warm": w["iters_exact_per_step"],
        "iteration_reduction": p["iters_exact_per_step"] / max(w["iters_exact_per_step"], 1e-9),
        "iters_per_step_extrapolation": x["iters_exact_per_step"],
        "iteration_reduction_extrapolation_only": p["iters_exact_per_step"] / max(x["iters_exact_per_step"], 1e-9),
        "plain": p, "warm": w, "extrapolation": x,
    }


def batch_leg(args):
    """The batched ensemble: independent shear boxes (particle counts
    log-uniform in [2000, 20000]) stepped by one persistent launch per call,
    launch shape from the autotuner, replayed as a CUDA graph."""
    from sphere_b200 import configs
    from sphere_b200.engine import Batch
    boxes, meta = configs.batch_shear_boxes(nbox=args.batch_boxes, seed=7)
    total = int(sum(m["n"] for m in meta))
    interval = 100
    with Batch(boxes, precision="mixed") as b:
        b.step(300)                      # autotunes on its first steps
        for _ in range(2):
            b.step(interval)             # captures the graph
        times = [b.step_timed(interval) for _ in range(args.batch_steps)]
        cfg = b.config()
        trials = b.trials()
    step_s = float(numpy.sum(times)) * 1e-3
    return {
        "workload": f"{len(boxes)} shear boxes, {total} particles (counts log-uniform in [2000, 20000]), "
                    "radii U(0.009, 0.011) m, sigma0 in {10..160} kPa, shear U(1e-5, 1e-3) m/s, "
                    "k_n = k_t = 1.16e7 N/m, mu U(0.3, 0.6), mixed precision",
        "particle_steps_per_s": total * interval * len(times) / step_s,
        "ms_per_step": 1e3 * step_s / len(times), "dem_steps_per_step": interval,
        "launch": cfg, "autotuner_trials": len(trials),
        "best_trial_ms_per_step": min(t["ms_per_step"] for t in trials) if trials else None,
    }


def ns_leg(args):
    """Navier-Stokes fluid (cfd_solver 0) coupled to the consolidation
    packing: the settled N-sphere packing on the 40 x 40 x 80 fluid grid
    under the 10 kPa wall, water (mu = 8.9e-4 Pa s, rho_f = 1000 kg/m^3) at
    hydrostatic pressure, the reference's solver defaults (tolerance 1e-3,
    theta 1, beta 0, ndem 1); faithful FP64.  Per DEM step: the time of the
    whole step and of its fluid stage, the projection's Jacobi iterations,
    and the same step of the reference's own kernels built for the host
    (oracle/_ref, one thread) when it is present."""
    import tempfile
    from sphere_b200 import binfile, configs
    from sphere_b200.engine import Engine
    d = configs.darcy_benchmark(n=args.particles, seed=SEED, log=log)
    configs.init_fluid_ns(d, mu=8.9e-4, rho_f=1000.0, hydrostatic=True)
    steps = args.ns_steps
    with Engine(d, fluid=True, precision="faithful") as eng:
        eng.step(3)
        ms, fluid, iters = [], [], []
        for _ in range(steps):
            pr = eng.profile(1)
            ms.append(pr.step_ms)
            fluid.append(pr.fluid_ms)
            iters.append(int(eng.get("darcy_iters")[0]) + 1)
    out = {
        "workload": f"Navier-Stokes fluid, N={d.np}, grid {int(d.num[0])}x{int(d.num[1])}x{int(d.num[2])}, "
                    "water at hydrostatic pressure, tolerance 1e-3, faithful FP64",
        "dem_steps": steps, "ms_per_dem_step": float(numpy.mean(ms)),
        "fluid_ms_per_dem_step": float(numpy.mean(fluid)),
        "jacobi_iters_per_step": float(numpy.mean(iters)),
        "us_per_jacobi_iteration_upper_bound": 1e3 * float(numpy.sum(fluid)) / max(1, int(numpy.sum(iters))),
    }
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        if O.ref_available() and args.ns_ref_steps > 0:
            with tempfile.TemporaryDirectory() as td:
                path = os.path.join(td, "ns.bin")
                binfile.write_bin(d, path)
                ref = O.Reference(path, fluid=True)
                ref.step(1)
                t0 = time.perf_counter()
                ref.step(args.ns_ref_steps)
                sec = (time.perf_counter() - t0) / args.ns_ref_steps
                ref.close()
            out["cpu_reference"] = {"s_per_dem_step": sec, "cores": 1, "kind": "reference",
                                    "sample": f"{args.ns_ref_steps} DEM steps after the first"}
            out["speedup_vs_cpu_reference"] = sec / (1e-3 * out["ms_per_dem_step"])
    except Exception as exc:  # the reference build is optional here
        out["cpu_reference"] = {"unavailable": str(exc)}
    return out


def render_leg(args, d):
    """The ray tracer (``sphere --render``) on the headline packing at the
    reference's defaults: 800 x 800 pixels, pressure colour map."""
    from sphere_b200.engine import Engine
    import time as _t
    with Engine(d, precision="mixed") as eng:
        eng.step(10)
        eng.render(method=1, width=800, height=800)      # warm-up
        t0 = _t.perf_counter()
        reps = 3
        for _ in range(reps):
            eng.render(method=1, width=800, height=800)
        s = (_t.perf_counter() - t0) / reps
    tests = 800 * 800 * d.np
    return {"workload": f"ray-traced image, 800x800 pixels, N={d.np} spheres, pressure colour map",
            "ms_per_image": 1e3 * s, "ray_sphere_tests_per_s": tests / s,
            "note": "wall time of the whole call (state read-back, camera, kernels, image copy)"}


def settle_leg(args):
    """Plain FP64 dry settling (the configuration the reference itself runs):
    10,000 spheres on the first sites of a 22 x 22 x 21 lattice, spacing
    0.025 m, jitter +/-0.002 m, radii U(0.009, 0.011) m, periodic x/y, linear
    contact k_n = k_t = 1.16e7 N/m, mu = 0.5, run for its 20,000 steps from
    the lattice; faithful FP64."""
    from sphere_b200 import configs
    from sphere_b200.engine import Engine
    d = configs.settling_lattice(n=10000, seed=SEED)
    steps = args.settle_steps
    with Engine(d, precision="faithful", graph_steps=100) as eng:
        ms = eng.step_timed(steps)
        info = eng.info()
        zbar = mean_contacts(eng, d.np)
    return {
        "workload": "dry settling, N=10000 on a 22x22x21 lattice (spacing 0.025 m, jitter 0.002 m), "
                    "radii U(0.009, 0.011) m, k_n = k_t = 1.16e7 N/m, mu = 0.5, periodic x/y, "
                    "faithful FP64, from the lattice",
        "dem_steps": steps, "particle_steps_per_s": d.np * steps / (ms * 1e-3),
        "us_per_dem_step": 1e3 * ms / steps, "resorts": int(info.resorts),
        "mean_contacts_per_particle_at_end": zbar,
        "step_path": step_path_name(info),
    }


def large_leg(args):
    """The large polydisperse cohesive packing (4e6 spheres, log-normal
    radii, bonded initial neighbours), mixed precision, per-stage kernels:
    particle-steps/s, and the DRAM-roofline fraction of the sort and of the
    contact stage (algorithmic bytes per particle: hash 32 + sort 16 +
    reorder 180 = 228 per sort; contacts 184 + 56 Z per step)."""
    from sphere_b200 import configs
    from sphere_b200.engine import Engine
    d = configs.large_cohesive_packing(n=args.large_particles, seed=SEED + 3)
    n, nb0 = d.np, d.nb0
    interval = 20
    with Engine(d, precision="mixed", graph_steps=interval) as eng:
        eng.step(2 * interval)
        times = [eng.step_timed(interval) for _ in range(args.large_steps)]
        prof = eng.profile(5)
        sort_ms = eng.time_sort(3)
        zbar = mean_contacts(eng, n)
        info = eng.info()
    # the plain FP64 drop-in (faithful arithmetic) on the same packing
    with Engine(d, precision="faithful", graph_steps=interval) as eng:
        eng.step(2 * interval)
        times_fp64 = [eng.step_timed(interval) for _ in range(args.large_steps)]
    fp64_rate = n * interval * len(times_fp64) / (float(numpy.sum(times_fp64)) * 1e-3)
    peak, peak_kind = load_peaks()
    step_s = float(numpy.sum(times)) * 1e-3
    contacts_bpp = 184.0 + 56.0 * zbar
    contacts_gbs = n * contacts_bpp / (prof.contacts_ms * 1e-3) / 1e9
    sort_gbs = n * 228.0 / (sort_ms * 1e-3) / 1e9
    return {
        "workload": f"large cohesive packing, N={n}, log-normal radii (median 0.01 m, sigma_ln 0.3, "
                    f"clipped to [0.004, 0.03] m), {nb0} bonds (k 1e7, tensile strength 1e5 Pa), "
                    "E=7e8 Pa, mu=0.5, periodic x/y, bottom wall, gravity, mixed precision",
        "particle_steps_per_s": n * interval * len(times) / step_s,
        "ms_per_dem_step": 1e3 * step_s / (interval * len(times)),
        "fp64_plain_particle_steps_per_s": fp64_rate,
        "mixed_over_fp64": n * interval * len(times) / step_s / fp64_rate,
        "mean_contacts_per_particle": zbar,
        "step_path": step_path_name(info),
        "stage_ms_per_dem_step": {"resort": prof.resort_ms, "contacts": prof.contacts_ms,
                                  "bonds": prof.bonds_ms, "integrate": prof.integrate_ms,
                                  "step": prof.step_ms},
        "sort": {"ms": sort_ms, "algorithmic_bytes_per_particle": 228.0, "achieved_gbs": sort_gbs,
                 "frac": sort_gbs / peak},
        "contacts": {"algorithmic_bytes_per_particle": contacts_bpp, "achieved_gbs": contacts_gbs,
                     "frac": contacts_gbs / peak},
        "peak_gbs": peak, "peak_source": peak_kind,
    }


def cpu_baseline(d, sample_steps=3):
    """The oracle (CPU restatement of the reference step, OpenMP) on a
    bounded sample of the same workload."""
    import tempfile
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from sphere_b200 import binfile
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "w.bin")
        binfile.write_bin(d, path)
        orc = O.Oracle(path, precision="faithful")
        orc.step(1)
        t0 = time.perf_counter()
        orc.step(sample_steps)
        t1 = time.perf_counter()
        orc.close()
    cores = os.cpu_count() or 1
    nthreads = int(os.environ.get("OMP_NUM_THREADS", cores))
    return {"value": d.np * sample_steps / (t1 - t0), "unit": "particle-steps/s",
            "cores": nthreads, "kind": "port",
            "sample": f"{sample_steps} DEM steps of the N={d.np} workload after 1 warm-up step"}


# DEM steps per benchmark step of the reference arm when it runs the
# reference's own kernels built for the host: they run one thread at a time
# (about 0.2 s per DEM step of this workload on one core), so a benchmark step
# of INTERVAL DEM steps would make a 30-step run last ten minutes
REF_BUILD_SAMPLE = 10


def run_reference(args):
    """The reference arm: the reference's own FP64 step on the host cores.
    Where the reference's kernels were compiled for the host (oracle/_ref:
    sorting.cuh, contactsearch.cuh, contactmodels.cuh, integration.cuh,
    ... driven one thread at a time, the reference having no CPU DEM path of
    its own), those; otherwise the oracle's restatement of them on all host
    threads.  Each benchmark step times a bounded sample of DEM steps of the
    same workload; the metric is per particle and DEM step."""
    n = args.particles
    d = workload(n)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import tempfile
    import oracle as O
    from sphere_b200 import binfile
    kind = "reference" if O.ref_available() else "port"
    sample_steps = args.ref_sample or (REF_BUILD_SAMPLE if kind == "reference" else INTERVAL)
    times = []
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "w.bin")
        binfile.write_bin(d, path)
        runner = O.Reference(path) if kind == "reference" else O.Oracle(path, precision="faithful")
        # warm-up steps: one DEM step each (the CPU code has no state a
        # longer warm-up would prepare)
        for _ in range(args.warmup):
            runner.step(1)
        for _ in range(args.steps):
            t0 = time.perf_counter()
            rc = runner.step(sample_steps)
            t1 = time.perf_counter()
            if rc:
                raise RuntimeError(f"reference step failed with status {rc}")
            times.append(t1 - t0)
        runner.close()
    total = float(numpy.sum(times))
    value = n * sample_steps * args.steps / total
    if kind == "reference":
        cores = 1
        sample = (f"{sample_steps} DEM steps of the N={n} workload per benchmark step: the "
                  f"reference's own kernels compiled for the host (oracle/_ref), one thread, "
                  f"{sample_steps} instead of {INTERVAL} DEM steps per benchmark step to keep "
                  f"the run within minutes")
    else:
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        sample = (f"{sample_steps} DEM steps of the N={n} workload per benchmark step: the oracle "
                  f"(a C restatement of the reference's FP64 step, pinned bit-exact against the "
                  f"reference's own kernels built for the host), OpenMP on {cores} threads")
    cfg = workload_config(n)
    cfg["dem_steps_per_step"] = sample_steps
    return {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded settled packing)",
        "config": cfg,
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores,
                         "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["faithful", "fp64", "mixed"])
    ap.add_argument("--step-kernel", default="auto",
                    choices=["auto", "stages", "persistent", "stages_staged", "stages_fused"],
                    help="step path of the shear leg: automatic (autotuned), the per-stage "
                         "kernels, the fused persistent kernel, the per-stage kernels with "
                         "the contact search reading neighbour cells staged in shared memory, "
                         "or the per-stage kernels with contacts and integration in one launch")
    ap.add_argument("--particles", type=int, default=N_PARTICLES)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--ref-sample", type=int, default=0,
                    help="DEM steps per benchmark step of the reference arm (0: %d with the "
                         "reference's host build, %d with the oracle port)" % (REF_BUILD_SAMPLE, INTERVAL))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--darcy-steps", type=int, default=200,
                    help="fluid steps per arm of the Darcy leg (0 skips it)")
    ap.add_argument("--batch-boxes", type=int, default=256,
                    help="boxes of the batched-ensemble leg (0 skips it)")
    ap.add_argument("--batch-steps", type=int, default=5)
    ap.add_argument("--large-particles", type=int, default=4_000_000,
                    help="spheres of the large cohesive-packing leg (0 skips it)")
    ap.add_argument("--large-steps", type=int, default=5,
                    help="timed calls of 20 DEM steps in the large leg")
    ap.add_argument("--render", type=int, default=1,
                    help="1: time the ray tracer on the headline packing (0 skips it)")
    ap.add_argument("--settle-steps", type=int, default=20000,
                    help="DEM steps of the 10,000-sphere settling leg (0 skips it)")
    ap.add_argument("--ns-steps", type=int, default=20,
                    help="DEM steps of the Navier-Stokes leg (0 skips it)")
    ap.add_argument("--ns-ref-steps", type=int, default=1,
                    help="steps of the reference's host build timed beside the Navier-Stokes leg")
    ap.add_argument("--legs", default="shear,darcy,batch,large,settle,render,ns",
                    help="comma list of legs to run: shear (the headline), darcy, batch, large, "
                         "settle, render, ns")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0
    if world > 1:
        # replicas only: every rank runs the same single-GPU workload; the
        # timing is the max over ranks (see run_distributed)
        return run_distributed(args, rank, world)
    legs = set(args.legs.split(","))
    if "shear" not in legs:
        # a single side leg (profiling runs): its own JSON object
        out = {}
        if "darcy" in legs and args.darcy_steps > 0:
            out["darcy"] = darcy_leg(args)
        if "batch" in legs and args.batch_boxes > 0:
            out["batch"] = batch_leg(args)
        if "large" in legs and args.large_particles > 0:
            out["large"] = large_leg(args)
        if "settle" in legs and args.settle_steps > 0:
            out["settle"] = settle_leg(args)
        if "render" in legs and args.render:
            out["render"] = render_leg(args, workload(args.particles))
        if "ns" in legs and args.ns_steps > 0:
            out["navier_stokes"] = ns_leg(args)
        print(json.dumps(out), flush=True)
        return 0
    if "darcy" not in legs:
        args.darcy_steps = 0
    if "batch" not in legs:
        args.batch_boxes = 0
    if "large" not in legs:
        args.large_particles = 0
    if "settle" not in legs:
        args.settle_steps = 0
    if "render" not in legs:
        args.render = 0
    if "ns" not in legs:
        args.ns_steps = 0
    print(json.dumps(run_gpu(args)), flush=True)
    return 0


def max_over_ranks(x, device=None):
    """The maximum of a per-rank float over the process group."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def combine_replicas(max_ms, max_e2e_s, world, n, steps):
    """Whole-job throughput of `world` replicas that each stepped n particles
    for steps x INTERVAL DEM steps: device time and end-to-end wall time are
    the maxima over ranks."""
    work = world * n * INTERVAL * steps
    return {"value": work / (max_ms * 1e-3), "ms_per_step": max_ms / steps,
            "e2e_value": work / max_e2e_s}


def run_distributed(args, rank, world):
    """Replicas only: every rank steps its own copy of the headline workload
    (the boxes are independent, nothing is exchanged); the timed K calls are
    bracketed by a barrier and a device synchronisation on both sides, and
    the job's time is the maximum over ranks."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from sphere_b200.engine import Engine
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    n = args.particles
    d = workload(n)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    eng = Engine(d, precision=args.precision, graph_steps=INTERVAL, device=local)
    for _ in range(args.warmup):
        eng.step(INTERVAL)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize()
    dist.barrier()
    times = []
    for _ in range(args.steps):
        flush_l2(flush)
        times.append(eng.step_timed(INTERVAL))
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop() if sampler else None
    # end to end through the C ABI with pinned host buffers (state up,
    # INTERVAL steps, state down), the same bracket
    x = torch.empty((n, 4), dtype=torch.float64).pin_memory().numpy()
    v = torch.empty((n, 4), dtype=torch.float64).pin_memory().numpy()
    w = torch.empty((n, 4), dtype=torch.float64).pin_memory().numpy()
    eng.get("x", x); eng.get("vel", v); eng.get("angvel", w)
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.set("x", x); eng.set("vel", v); eng.set("angvel", w)
        eng.step(INTERVAL)
        eng.get("x", x); eng.get("vel", v); eng.get("angvel", w)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    dist.barrier()
    info = eng.info()
    eng.close()
    max_ms = max_over_ranks(float(numpy.sum(times)), dev)
    max_e2e = max_over_ranks(e2e_s, dev)
    comb = combine_replicas(max_ms, max_e2e, world, n, args.steps)
    if rank == 0:
        per_step = 3 + (2 if d.nw > 0 and d.wmode[0] == 3 else 0)
        if info.step_path == 2:
            per_step = 3
        out = {
            "metric": "particle-steps/s", "value": comb["value"], "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": comb["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"faithful": "f64", "fp64": "f64", "mixed": "f32+f64"}[args.precision],
            "data": "synthetic (seeded settled packing)",
            "config": {"workload": f"dense dry shear, N={n} per GPU (independent replicas)",
                       "dem_steps_per_step": INTERVAL, "precision": args.precision,
                       "parallelism": f"replicas{world}",
                       "l2": "flushed between timed steps (256 MB write)"},
            "e2e": {"value": comb["e2e_value"], "unit": "particle-steps/s",
                    "h2d_bytes_per_step": 3 * 32 * n * world, "d2h_bytes_per_step": 3 * 32 * n * world},
            "gpu_launches": (args.steps if info.step_path == 1
                             else per_step * INTERVAL * args.steps) * world,
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
