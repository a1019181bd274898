"""A few Newton steps of a named workload from its freestream: a short, fixed program
to run under a profiler.

    python -m jaxrans_b200.profile [WORKLOAD] [--precision fp64|mixed] [--steps N]
                                   [--time] [--line-schedule F,A,S] [--applies N]

Prints the residual norms of the steps; ``--time`` also prints the live CUDA-event times
of the hot kernels (``jr_time_kernels``); ``--line-schedule`` replaces the autotuner's
choice by the line factor's and line solve's threads per chain and the solve's form
(``jr_line_schedule``: S = 0 global, 1..4 staged; the autotuner is then not run);
``--applies N`` then factors the line preconditioner at the state and applies it to N
seeded random right-hand sides through the C ABI (one factor and one solve launch each,
outside any graph).
"""

from __future__ import annotations

import argparse
import sys

import numpy as np

from .batch import batch_device
from .solver import device_for, freestream_state
from .workloads import BATCHES, batch_workload, workload


def main(argv=None) -> int:
    p = argparse.ArgumentParser(prog="python -m jaxrans_b200.profile", description=__doc__.splitlines()[0])
    p.add_argument("workload", nargs="?", default="c_sa_385", help="a workload or a batch name")
    p.add_argument("--precision", default="fp64", choices=("fp64", "mixed"))
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--time", action="store_true")
    p.add_argument("--line-schedule", default=None, metavar="F,A,S")
    p.add_argument("--applies", type=int, default=0)
    args = p.parse_args(argv)
    prec = {"implicit.precision": args.precision}
    if args.workload in BATCHES:
        cases = batch_workload(args.workload, **prec)
        made = {}
        grids = []
        for (name, _), case in zip(BATCHES[args.workload], cases):
            if name not in made:
                made[name] = case.grid()
            grids.append(made[name])
        dev = batch_device(cases, grids, autotune=not args.line_schedule)
        for k, (c, g) in enumerate(zip(cases, grids)):
            dev.set_case_state(k, freestream_state(c, g), c.implicit.cfl)
    else:
        case = workload(args.workload, **prec)
        plan = case.grid()
        dev = device_for(case, plan, autotune=not args.line_schedule)
        dev.set_state(freestream_state(case, plan), case.implicit.cfl)
    if args.line_schedule:
        f, a, s = (int(x) for x in args.line_schedule.split(","))
        dev.line_schedule(f, a, s)
    first = min(3, args.steps)
    if first > 0:
        print(dev.newton_steps(first))
    if args.steps > first:
        print(dev.newton_steps(args.steps - first))
    if args.applies > 0:
        U, cfl = dev.get_state()[:2]
        rng = np.random.default_rng(0)
        for _ in range(args.applies):
            z = dev.precondition(U, float(np.max(cfl)), rng.standard_normal(np.shape(U)))
        print("|z| of the last solve", float(np.linalg.norm(z)))
    if args.time:
        for name, ms in dev.time_kernels(20).items():
            print(f"{name:18s} {1e3 * ms:9.2f} us")
    dev.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
