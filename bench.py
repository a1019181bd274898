#!/usr/bin/env python3
"""Benchmark: converged RANS solves per hour on one B200 (or N replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c_sa_385] [--precision fp64|mixed] [--line-schedule F,A,S]

A step is one converged solve of the workload (``jaxrans_b200.workloads``; by default
the 2D SA-noft2 NACA 4412 C-grid 385 x 97, Roe + MUSCL minmod, GMRES(30)) from the
freestream, stopped by the reference's own exit test.  ``value`` times the solves with
the start state already in HBM (a device-to-device restart); ``e2e`` times them through
the C ABI from a pinned host state, the final state and forces read back each solve.
With N GPUs each rank runs its own replica of the same solves (the cases are
independent: no collective on the data path) and the whole-job rate is reported.

``--impl reference`` times the CPU restatement of the reference (``oracle``; the
reference itself is JAX, absent here) on a bounded sample of the same workload: each
step one Newton step, extrapolated by the number of Newton steps a converged solve takes.

The default line (config 2, FP64) also carries ``forms``: the north-star forms timed
beside it on bounded samples -- the batched mixed polar ``polar16_uneven`` (19 cases of
uneven grids in one device plan) and a served Poisson stream of 24 mixed requests with
continuous batching -- with their solves/hr, p50/p99 and ratios to the plain FP64 path
(``--no-forms`` skips them).

``--workload wing_ch_4blk`` (or ``wing_ch_4blk_small``) prints a separate line: 3D
pseudo-transient Newton steps per second of the swept, tapered wing on its four-block
C-H grid (3.93M cells), the state resident on the device.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "jax-rans_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

import numpy as np  # noqa: E402

METRIC = "converged RANS solves/hr"
# Newton steps of one converged solve of each workload from the freestream (FP64): the
# device path's own count (the bench line's config.newton_steps_per_solve, which it
# measures every run); the CPU samples, a few Newton steps each, are scaled by it.
STEPS_PER_SOLVE = {"c_sa_385": 680, "o_euler_257": 3840}
# coefficients of the linearisation the J.v tile reads per face and per cell (the
# kernel's JacShape and JCELL): inviscid 4 x 4 per side, the SA convection's 3, the
# viscous tail's derivatives its dependences allow (19 laminar, 33 SA)
LIN_FACE = {"euler": 32, "laminar": 32 + 19, "sa": 35 + 33}
LIN_CELL = {"euler": 0, "laminar": 0, "sa": 7}


def model_of(flow) -> str:
    return "euler" if flow.inviscid else ("sa" if flow.turbulence is not None else "laminar")


def jvp_bytes_per_cell(model: str, nvar: int, fp32_faces: bool = False) -> int:
    """Algorithmic bytes per cell of one J.v tile launch: the coefficients of the two faces
    a cell owns (FP64, or FP32 in the mixed form) and its own, then U (the primitive
    tangent), v and the output, V/dt; viscous: the centre (2); SA: the volume and the two
    face vectors the Green-Gauss source reads (4), all FP64."""
    words = LIN_CELL[model] + 3 * nvar + 1
    if model != "euler":
        words += 2
    if model == "sa":
        words += 1 + 4
    return 8 * words + (4 if fp32_faces else 8) * 2 * LIN_FACE[model]


def residual_bytes_per_cell(model: str, nvar: int) -> int:
    """Algorithmic bytes per cell of one residual tile launch (FP64): U and R, the volume,
    the two face vectors a cell owns (4); viscous: the centre (2); SA: the wall distance."""
    return 8 * (2 * nvar + 1 + 4 + (2 if model != "euler" else 0) + (1 if model == "sa" else 0))


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.is_file():
        return {**json.loads(path.read_text()), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def profiled_traffic(workload: str):
    """dram bytes per launch of the J.v tile from the committed ncu summary, if any."""
    path = ROOT / "profiles" / f"jvp_tile_{workload}.txt"
    if not path.is_file():
        return None
    for ln in path.read_text().splitlines():
        if ln.startswith("dram_bytes_per_launch:"):
            return float(ln.split(":", 1)[1].split()[0])
    return None


def reference_sample(name: str, steps: int, warmup: int, precision: str):
    """Seconds of each of `steps` Newton steps of the CPU restatement (the oracle) of
    workload `name` from the freestream, after `warmup` untimed ones (one process, one
    thread: the pool around it gives each host core its own solve)."""
    from jaxrans_b200.config import freestream_primitive
    from jaxrans_b200.workloads import workload
    from oracle import implicit as im
    from oracle import numerics as nm
    case = workload(name, **{"implicit.precision": precision})
    plan = case.grid()
    flow, num = case.flow, case.numerics
    model = nm.Model(plan, np.array(freestream_primitive(flow)), flow.gamma, num.flux, num.limiter, num.kappa,
                     None if flow.inviscid else flow.mu_inf, flow.sutherland_ratio, flow.turbulence is not None,
                     0.3 if flow.turbulence == "sa_noft2_qcr" else 0.0, num.far_field, plan.distance)
    state = im.NewtonState(nm.initial_state(model), case.implicit.cfl, float("inf"))
    times = []
    with np.errstate(all="ignore"):
        for k in range(warmup + steps):
            t = time.perf_counter()
            state, _ = im.newton_step(state, model, case.implicit)
            if k >= warmup:
                times.append(time.perf_counter() - t)
    return times


def _sample_worker(job):
    return reference_sample(*job)


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_rate(name: str, steps: int, warmup: int, precision: str, steps_per_solve: int) -> dict:
    """The oracle's whole-host throughput on workload `name`: one independent solve per
    host core (a process pool started with spawn, one BLAS thread each), each timed over
    `steps` Newton steps after `warmup`; solves/hr = cores / (mean step x steps per solve)."""
    import multiprocessing
    cores = host_cores()
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    with multiprocessing.get_context("spawn").Pool(cores) as pool:
        times = pool.map(_sample_worker, [(name, steps, warmup, precision)] * cores)
    per_step = statistics.mean(t for ts in times for t in ts)
    value = cores * 3600.0 / (per_step * steps_per_solve)
    sample = (f"{cores} processes (one per host core, one thread each), each one solve of the oracle (NumPy "
              f"FP64, complex-step J.v) from the freestream on {name}: {warmup} untimed and {steps} timed Newton "
              f"steps, {per_step:.2f} s per step on average, scaled by {steps_per_solve} Newton steps per "
              f"converged solve")
    return {"value": value, "unit": "solves/hr", "cores": cores, "kind": "port", "sample": sample,
            "seconds_per_step": per_step}


def run_reference(args) -> int:
    rank, _, world = rank_info()
    if rank != 0:
        return 0
    from jaxrans_b200.workloads import BATCHES, workload
    # a batch is timed on its first case (the oracle runs one case at a time)
    name = BATCHES[args.workload][0][0] if args.workload in BATCHES else args.workload
    n = STEPS_PER_SOLVE[name]
    cpu = cpu_rate(name, args.steps, args.warmup, args.precision, n)
    value, per_step = cpu["value"], cpu.pop("seconds_per_step")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/hr", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per_step * n / cpu["cores"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (generated NACA section and grid)",
            "config": {"workload": args.workload, "cells": workload(name).grid().cells,
                       "newton_steps_per_solve": n, "cores": cpu["cores"]},
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "solves/hr", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --- the 3D wing (a separate line: Newton steps per second of one 3D case) ------------

WING3D_WORKLOADS = ("wing_ch_4blk", "wing_ch_4blk_small")
METRIC3D = "3D pseudo-transient Newton steps/s"


def wing3d_setup(name: str):
    """The 3D workload's case (grid file written to a scratch directory) and plan; on a
    CUDA device the plan's wall distance is computed there."""
    import tempfile
    from jaxrans_b200.workloads import wing3d_case
    with tempfile.TemporaryDirectory() as d:
        case = wing3d_case(name, d)
        plan = case.grid()
    return case, plan


def oracle3d_step_seconds(steps: int, warmup: int):
    """Seconds per Newton step of the 3D oracle (NumPy FP64) on the small wing, from the
    freestream, and that case's cell count: the CPU rate per cell of a bounded sample."""
    from oracle import implicit3d as i3
    from oracle import numerics3d as n3
    from oracle.implicit import NewtonState
    from jaxrans_b200.solver3d import freestream_state3, physics3
    case, plan = wing3d_setup("wing_ch_4blk_small")
    ph = physics3(case)
    model = n3.Model3(plan, ph["q_inf"], ph["gamma"], ph["flux"], ph["limiter"], ph["kappa"], ph["mu_inf"],
                      ph["sutherland"], len(ph["q_inf"]) == 6, plan.distance)
    state = NewtonState(freestream_state3(case, plan), case.implicit.cfl, math.inf)
    times = []
    for k in range(warmup + steps):
        t0 = time.perf_counter()
        state, _ = i3.newton_step(state, model, case.implicit)
        if k >= warmup:
            times.append(time.perf_counter() - t0)
    return statistics.mean(times), plan.cells


def jvp3d_bytes_per_cell(nvar: int) -> int:
    """Algorithmic bytes per cell of one 3D J.v (every launch of jr_jvp3d: primitive canvas,
    ghost stages, face phase, cell phase): U and v read, J.v written (3 nvar), the volume,
    the three face vectors a cell owns (9), the centre (3) and the wall distance, FP64."""
    return 8 * (3 * nvar + 1 + 9 + 3 + 1)


def roofline3d(kern: dict, nvar: int, cells: int, peaks: dict) -> dict:
    """The 3D J.v's achieved HBM bandwidth (its algorithmic bytes over the CUDA-event time of
    the whole jr_jvp3d sequence) against the measured copy bandwidth."""
    per_cell = jvp3d_bytes_per_cell(nvar)
    achieved = per_cell * cells / (kern["jvp3d"] * 1e-3) / 1e9
    return {"kernel": "jvp3d (primitive canvas, ghost stages, face phase, cell phase)", "bound": "hbm",
            "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
            "traffic": None, "algorithmic_bytes_per_cell": per_cell, "algorithmic_bytes_per_launch": per_cell * cells,
            "launch_ms": kern["jvp3d"], "peak_source": peaks.get("source", "measured")}


def run_wing3d(args) -> int:
    """``--workload wing_ch_4blk``: K pseudo-transient Newton steps of the 3D wing
    (``jr_newton_steps3d``, GMRES with the line preconditioner, host-driven: the step
    synchronises for its scalars, so it is timed by the host clock between device
    synchronisations) with the state resident; ``e2e`` the same steps through
    ``DevicePlan3.newton_steps`` from and back to a host state."""
    rank, local, world = rank_info()
    if args.impl == "reference":
        if rank != 0:
            return 0
        from jaxrans_b200.workloads import wing3d_cells
        per_step, cells = oracle3d_step_seconds(max(1, min(args.steps, 2)), 1)
        total = wing3d_cells(args.workload)
        value = cells / (per_step * total)
        sample = (f"Newton steps of the 3D oracle (NumPy FP64, complex-step J.v) on the wing_ch_4blk_small grid "
                  f"({cells} cells), {per_step:.1f} s each, scaled by cells to the {total}-cell workload")
        print(json.dumps({"impl": "reference", "metric": METRIC3D, "value": value, "unit": "steps/s",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated wing and grid)",
                          "config": {"workload": args.workload, "cells": total},
                          "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "port",
                                           "sample": sample},
                          "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    import ctypes as C
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from jaxrans_b200.build import build
    from jaxrans_b200.solver3d import device3_for, freestream_state3
    build()
    case, plan = wing3d_setup(args.workload)
    dev = device3_for(case, plan)
    U0 = freestream_state3(case, plan)
    U_dev = torch.from_numpy(U0).to("cuda")
    cfl, res, hist = C.c_double(case.implicit.cfl), C.c_double(math.inf), np.zeros(1)

    def device_step():
        rc = dev.lib.jr_newton_steps3d(dev.handle, U_dev.data_ptr(), 1, C.byref(cfl), C.byref(res), hist.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"jr_newton_steps3d failed ({rc}): {dev.lib.jr_last_error().decode()}")

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        device_step()
    launches = C.c_int64()
    dev.lib.jr_launches3d(C.byref(launches))
    before = launches.value
    barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            device_step()
        torch.cuda.synchronize()
        seconds = time.perf_counter() - t0
    dev.lib.jr_launches3d(C.byref(launches))
    launched = launches.value - before
    kern3 = dev.time_kernels(U_dev.cpu().numpy(), 5)
    U_host, c2, r2 = U0.copy(), case.implicit.cfl, math.inf
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        U_host, c2, r2, _ = dev.newton_steps(U_host, 1, c2, r2)
    torch.cuda.synchronize()
    e2e_seconds = time.perf_counter() - t0
    seconds, e2e_seconds = max_over_ranks([seconds, e2e_seconds], dist, "cuda")
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            per_step, cells = oracle3d_step_seconds(1, 0)   # NumPy: no warm-up to amortise
            cpu = {"value": cells / (per_step * plan.cells), "unit": "steps/s", "cores": 1, "kind": "port",
                   "sample": f"one Newton step of the 3D oracle on the wing_ch_4blk_small grid ({cells} cells), "
                             f"{per_step:.1f} s, scaled by cells"}
        value = world * args.steps / seconds
        bytes_per_step = int(U0.nbytes)
        print(json.dumps({
            "metric": METRIC3D, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * seconds / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated wing and grid)",
            "config": {"workload": args.workload, "cells": plan.cells, "canvas": list(plan.shape),
                       "blocks": len(plan.mesh), "nvar": int(U0.shape[0]),
                       "krylov_subspace": case.implicit.krylov_subspace,
                       "preconditioner": case.implicit.preconditioner, "precision": case.implicit.precision,
                       "l2": "inputs larger than L2" if U0.nbytes > 126e6 else "inputs smaller than L2, no flush",
                       "timer": "host clock between device synchronisations (the 3D step is host-driven)"},
            "e2e": {"value": world * args.steps / e2e_seconds, "unit": "steps/s",
                    "h2d_bytes_per_step": bytes_per_step, "d2h_bytes_per_step": bytes_per_step},
            "gpu_launches": launched, "kernel_ms": kern3,
            "roofline": roofline3d(kern3, int(U0.shape[0]), plan.cells, measured_peaks()),
            "cpu_baseline": cpu, "clocks": clocks.summary()}),
            flush=True)
    if dist is not None:
        dist.destroy_process_group()
    dev.close()
    return 0


def roofline_of(kern: dict, model: str, nvar: int, cells: int, peaks: dict, kernel: str = "jvp_tile",
                fp32_faces: bool = False) -> dict:
    """A tile kernel's achieved HBM bandwidth: its algorithmic bytes per launch over its
    CUDA-event launch time, against the measured copy bandwidth (fp32_faces: the J.v of
    the mixed form, its face coefficients in FP32)."""
    per_cell = (jvp_bytes_per_cell(model, nvar, fp32_faces) if kernel == "jvp_tile"
                else residual_bytes_per_cell(model, nvar))
    achieved = per_cell * cells / (kern[kernel] * 1e-3) / 1e9
    return {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": None, "algorithmic_bytes_per_cell": per_cell,
            "algorithmic_bytes_per_launch": per_cell * cells, "launch_ms": kern[kernel],
            "peak_source": peaks.get("source", "measured")}


def measure_forms(fp64_value: float, fp64_forces, peaks: dict, served_requests: int = 24) -> dict:
    """The north-star forms beside the plain FP64 line, each bounded to a few minutes:

    * batched, mixed: the 19 cases of ``polar16_uneven`` (16 angles on the 385 x 97 grid and
      the 257, 513 and 769 uneven grids) in one device plan, FP32 line preconditioner and
      Krylov basis, each case leaving the launches at its own exit; solves/hr of the whole
      batch (device clock), the cases' exit times (p50, p99), |dCL|, |dCD| of its 8 deg
      case against the FP64 line's forces, and the J.v and residual tiles' rooflines over
      the batch's 819k cells (each tile timed live with CUDA events on the batch);
    * config 3's whole batch (``polar64_uneven``, 2.59M cells), mixed: the tiles' kernel
      times and rooflines after one Newton step (the batch is not solved);
    * served: a seeded Poisson stream (20 requests/s) of ``served_requests`` SA requests of
      the config-4 distribution (van Albada), mixed, continuous batching with up to
      ``served_requests`` slots per grid size; solves/hr over the stream's wall time,
      p50/p99 latency from arrival; the first three requests also solved one at a time on
      the plain FP64 path (solves/hr, |dCL|, |dCD| against the served results).
    """
    import dataclasses
    import torch
    from jaxrans_b200.batch import batch_device, run_batch_blocks, start_batch
    from jaxrans_b200.serve import Server, poisson_requests, summary
    from jaxrans_b200.solver import march
    from jaxrans_b200.workloads import BATCHES, batch_workload, workload
    out = {}
    # batched, mixed
    cases = batch_workload("polar16_uneven", **{"implicit.precision": "mixed"})
    made, grids = {}, []
    for (w, _), c in zip(BATCHES["polar16_uneven"], cases):
        if w not in made:
            made[w] = c.grid()
        grids.append(made[w])
    dev = batch_device(cases, grids, autotune=True)
    start_batch(dev, cases, grids)
    stream = torch.cuda.ExternalStream(dev.stream_handle())
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    monitors, seconds, _ = run_batch_blocks(cases, dev)
    s1.record(stream)
    torch.cuda.synchronize()
    wall = s0.elapsed_time(s1) / 1e3
    for k in range(len(cases)):   # the finished cases back in the launches, for the kernel times
        dev.enable(k, True)
    kern = dev.time_kernels(10)
    dev.close()
    batch_cells = sum(g.cells for g in grids)
    lat = [m.seconds * wall / seconds for m in monitors]
    k8 = [round(c.flow.alpha_deg, 6) for c in cases].index(8.0)
    f8 = monitors[k8].forces
    value = 3600.0 * len(cases) / wall
    out["batched_mixed"] = {
        "workload": "polar16_uneven", "cases": len(cases), "cells": sum(g.cells for g in grids),
        "solves_per_hr": value, "ratio_to_fp64_line": value / fp64_value, "seconds": wall,
        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
        "newton_steps_slowest": max(m.iterations for m in monitors),
        "exits": {r: sum(m.reason == r for m in monitors) for r in sorted({m.reason for m in monitors})},
        "alpha8_vs_fp64_line": {"dcl": abs(f8.cl - fp64_forces["cl"]), "dcd": abs(f8.cd - fp64_forces["cd"]),
                                "note": "settled (minmod) states: the state the forces settle on depends "
                                        "on the path, by about 5e-4 in CL between FP64 runs too"},
        "kernel_ms": kern,
        "roofline": roofline_of(kern, "sa", 5, batch_cells, peaks, fp32_faces=True),
        "roofline_residual": roofline_of(kern, "sa", 5, batch_cells, peaks, kernel="residual_tile")}
    # config 3's whole batch (64 angles and the three uneven grids, 2.59M cells), mixed: the
    # tiles' rooflines at that size, after one Newton step from the freestream
    cases = batch_workload("polar64_uneven", **{"implicit.precision": "mixed"})
    made, grids = {}, []
    for (w, _), c in zip(BATCHES["polar64_uneven"], cases):
        if w not in made:
            made[w] = c.grid()
        grids.append(made[w])
    dev = batch_device(cases, grids, autotune=True)
    start_batch(dev, cases, grids)
    dev.newton_steps(1)
    kern = dev.time_kernels(5)
    dev.close()
    cells3 = sum(g.cells for g in grids)
    out["config3_batch_kernels"] = {
        "workload": "polar64_uneven", "cases": len(cases), "cells": cells3, "precision": "mixed",
        "kernel_ms": kern, "roofline": roofline_of(kern, "sa", 5, cells3, peaks, fp32_faces=True),
        "roofline_residual": roofline_of(kern, "sa", 5, cells3, peaks, kernel="residual_tile")}
    # served, mixed, continuous batching
    template = workload("c_sa_385", **{"implicit.precision": "mixed", "convective_fluxes.limiter": "van_albada"})
    requests = poisson_requests(served_requests, template, 20.0, seed=0)
    server = Server(max_slots=served_requests, workers=4)
    t = time.perf_counter()
    served = server.serve(requests)
    wall = time.perf_counter() - t
    server.close()
    summ = summary(served, wall)
    plain_s, dcl, dcd = 0.0, [], []
    for x in served[:3]:
        c = x.request.case
        plain = dataclasses.replace(c, implicit=dataclasses.replace(c.implicit, precision="fp64"))
        grid = plain.grid()
        t = time.perf_counter()
        r = march(plain, grid)
        plain_s += time.perf_counter() - t
        dcl.append(abs(x.forces.cl - r.forces.cl))
        dcd.append(abs(x.forces.cd - r.forces.cd))
    plain_rate = 3600.0 * 3 / plain_s
    out["served_mixed"] = {
        "requests": served_requests, "rate_per_s": 20.0, "seed": 0, "limiter": "van_albada",
        "solves_per_hr": summ["solves_per_hr"], "p50_s": summ["p50_s"], "p99_s": summ["p99_s"],
        "exits": summ["exits"], "seconds": wall,
        "plain_fp64_first3": {"solves_per_hr": plain_rate, "max_dcl": max(dcl), "max_dcd": max(dcd)},
        "ratio_to_plain_fp64_first3": summ["solves_per_hr"] / plain_rate}
    return out


def max_over_ranks(values, dist, device):
    """Each value's maximum over the ranks (the slowest replica times the job); the
    values themselves without a process group."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def whole_job_rate(steps: int, n_cases: int, world: int, seconds: float) -> float:
    """Solves per hour of the whole job: every rank solved steps x n_cases cases in at
    most `seconds` (independent replicas, no collective on the data path)."""
    return 3600.0 * steps * n_cases * world / seconds


def load_job(args):
    """The cases of the workload (one, or a named batch), their grids (one per distinct
    workload) and the device plan."""
    from jaxrans_b200.batch import batch_device
    from jaxrans_b200.solver import device_for
    from jaxrans_b200.workloads import BATCHES, batch_workload, workload
    prec = {"implicit.precision": args.precision}
    if args.workload in BATCHES:
        cases = batch_workload(args.workload, **prec)
        names = [w for w, _ in BATCHES[args.workload]]
    else:
        cases = [workload(args.workload, **prec)]
        names = [args.workload]
    made = {}
    grids = []
    for name, case in zip(names, cases):
        if name not in made:
            made[name] = case.grid()
        grids.append(made[name])
    dev = (batch_device(cases, grids, autotune=False) if len(cases) > 1
           else device_for(cases[0], grids[0], autotune=False))
    if args.line_schedule:
        f, a, s = (int(x) for x in args.line_schedule.split(","))
        dev.line_schedule(f, a, s)
        args.schedule = {"line_factor_threads": f, "line_apply_threads": a, "line_apply_stage": s, "by": "hand"}
    else:
        args.schedule = dict(dev.autotune(), by="autotuner")
    return cases, grids, dev


def run_device(args) -> int:
    import torch
    rank, local, world = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from jaxrans_b200.batch import run_batch_blocks
    from jaxrans_b200.build import build
    from jaxrans_b200.solver import freestream_state
    build()
    cases, grids, dev = load_job(args)
    n_cases = len(cases)
    cfl = cases[0].implicit.cfl
    U0 = np.concatenate([freestream_state(c, g).ravel() for c, g in zip(cases, grids)])
    U0_pinned = torch.from_numpy(U0).pin_memory()
    U0_dev = U0_pinned.to("cuda")
    stream = torch.cuda.ExternalStream(dev.stream_handle())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    torch.cuda.synchronize()
    kps = dev.kernels_per_step()

    def barrier():
        if dist is not None:
            dist.barrier()

    def enable_all():
        if n_cases > 1:
            for k in range(n_cases):
                dev.enable(k, True)

    def device_solve():
        dev.set_state_device(U0_dev, cfl)
        enable_all()
        return run_batch_blocks(cases, dev)[0]

    def host_solve():
        dev.set_state(U0_pinned.numpy() if n_cases > 1 else U0_pinned.numpy().reshape(dev.shape), cfl)
        enable_all()
        out = run_batch_blocks(cases, dev)[0]
        U, _, _, _ = dev.get_state()
        return out, U

    for _ in range(args.warmup):
        device_solve()
    # timed: device-resident restarts
    launched0 = dev.launch_count()
    starts, ends, solves = [], [], []
    with Clocks(local) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            torch.cuda.synchronize()
            barrier()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            solves.append(device_solve())
            e.record(stream)
            torch.cuda.synchronize()
            starts.append(s)
            ends.append(e)
    per_step = [s.elapsed_time(e) / 1e3 for s, e in zip(starts, ends)]
    total = sum(per_step)
    launched = dev.launch_count() - launched0
    # e2e: host state in, state and forces out, through the C ABI
    e2e_times = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        barrier()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        out, U = host_solve()
        e.record(stream)
        torch.cuda.synchronize()
        e2e_times.append(s.elapsed_time(e) / 1e3)
    e2e_total = sum(e2e_times)
    total, e2e_total = max_over_ranks([total, e2e_total], dist, "cuda")
    value = whole_job_rate(args.steps, n_cases, world, total)
    e2e_value = whole_job_rate(args.steps, n_cases, world, e2e_total)
    # every case's latency: its exit within its batch, on the device clock of the batch
    latencies = [m.seconds * (step_t / max(mm.seconds for mm in mons))
                 for mons, step_t in zip(solves, per_step) for m in mons]
    iters = [m.iterations for mons in solves for m in mons]
    blocks = [max(len(m.blocks) for m in mons) for mons in solves]
    steps_run = [max(m.iterations for m in mons) for mons in solves]
    # the Newton steps' kernels (skipped Krylov cycles not counted) and, per block, the
    # ghost fill, force and exit-test kernels of the device monitor: all counted by the plan
    launches = launched
    kern = dev.time_kernels(20)
    peaks = measured_peaks()
    nvar = cases[0].flow.nvar
    model = model_of(cases[0].flow)
    cells = sum(g.cells for g in grids)
    roofline = roofline_of(kern, model, nvar, cells, peaks)
    roofline["traffic"] = profiled_traffic(args.workload)
    last = solves[-1]
    config = {"workload": args.workload, "cases": n_cases, "cells": cells, "nvar": nvar,
              "precision": args.precision, "newton_steps_per_solve": int(np.median(iters)),
              "exit_reasons": sorted({m.reason for mons in solves for m in mons}),
              "l2": "flushed (256 MB write) per step", "parallelism": f"replicas x{world}",
              "kernels_per_newton_step_max": kps, "line_schedule": args.schedule}
    if n_cases == 1:
        config["canvas"] = list(grids[0].shape)
        f = last[0].forces
        config["forces"] = {"cl": f.cl, "cd": f.cd, "cm": f.cm}
    else:
        config["batch"] = "every case in one device plan: one captured graph per Newton step for all"
        config["newton_steps_per_batch"] = int(max(steps_run))
    block_iters = cases[0].block_iters
    result = {
        "metric": METRIC, "value": value, "unit": "solves/hr", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32",
        "data": "synthetic (generated NACA sections and grids, freestream start)",
        "config": config,
        "latency_s": {"p50": float(np.percentile(latencies, 50)), "p99": float(np.percentile(latencies, 99))},
        "e2e": {"value": e2e_value, "unit": "solves/hr", "h2d_bytes_per_step": int(U0.nbytes),
                # the state, every step's |R| and every block's force sample of every case
                "d2h_bytes_per_step": int(U0.nbytes + max(len(m.blocks) for m in out) * 8 * n_cases
                                          * (block_iters + 3))},
        "gpu_launches": launches,
        "roofline": roofline,
        "roofline_residual": roofline_of(kern, model, nvar, cells, peaks, kernel="residual_tile"),
        "kernel_ms": kern,
    }
    if rank == 0:
        result["clocks"] = clocks.summary()
        if world == 1 and n_cases == 1 and not args.no_forms and args.workload == "c_sa_385" \
                and args.precision == "fp64":
            result["forms"] = measure_forms(value, config["forces"], peaks)
        if world == 1 and not args.no_cpu_baseline:
            from jaxrans_b200.workloads import BATCHES
            name = BATCHES[args.workload][0][0] if args.workload in BATCHES else args.workload
            # scaled by this run's own Newton steps per solve (the reference arm, a separate
            # process, uses STEPS_PER_SOLVE, this count as last measured)
            per_solve = int(np.median(iters)) if n_cases == 1 else STEPS_PER_SOLVE[name]
            cpu = cpu_rate(name, args.steps, args.warmup, args.precision, per_solve)
            cpu.pop("seconds_per_step")
            result["cpu_baseline"] = cpu
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    dev.close()
    return 0


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=("b200", "reference"))
    p.add_argument("--workload", default="c_sa_385",
                   choices=sorted(STEPS_PER_SOLVE) + ["polar64_uneven", "polar16_uneven"] + list(WING3D_WORKLOADS))
    p.add_argument("--precision", default="fp64", choices=("fp64", "mixed"))
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-forms", action="store_true",
                   help="skip the batched and served mixed forms timed beside the default FP64 line")
    p.add_argument("--line-schedule", default=None, metavar="F,A,S",
                   help="line factor threads, line solve threads, solve form (0 global, 1-4 staged) instead of "
                        "the autotuner's pick (for runs under a profiler, where its timings do not hold)")
    args = p.parse_args(argv)
    if args.warmup < 3:
        raise SystemExit("--warmup must be at least 3")
    if args.workload in WING3D_WORKLOADS:
        return run_wing3d(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_device(args)


if __name__ == "__main__":
    raise SystemExit(main())
