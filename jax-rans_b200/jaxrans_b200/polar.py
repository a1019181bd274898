"""A polar: one case at many angles of attack, batched on the GPU
(``src/jaxrans/polar.py``).

    python -m jaxrans_b200.polar CASE_DIR --alpha START STOP STEP
                                 [--set file.section.key=value ...] [--out DIR]

The angle of attack enters the solver only through the freestream vector, so every angle
is a case of one device batch on the same grid (``jaxrans_b200.batch``): one captured
graph steps all angles, each with its own CFL ramp, rejections and exit.  Output: the
reference's ``polar.dat`` table and ``polar_metadata.json``.
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import sys
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .batch import run_batch
from .case import Case, CaseError, load_case
from .plan import Plan
from .solver import Result, Timing

# largest CL range over the last quarter of a run for it to count as settled
# (src/jaxrans/simulation.py:40)
SETTLED_CL_SPREAD = 1e-4


@dataclass(frozen=True)
class Polar:
    """One ``Result`` per angle, and the timing of the batch (``src/jaxrans/polar.py:43-72``)."""

    case: Case
    alphas: np.ndarray
    results: list
    timing: Timing

    def table(self) -> np.ndarray:
        """Rows ``alpha, CL, CD, CD friction, CM, orders, iterations, CL spread, settled``."""
        return np.array([[a, r.forces.cl, r.forces.cd, r.forces.cd_friction, r.forces.cm,
                          r.history.orders_dropped, r.history.n_iters, r.cl_spread,
                          float(r.cl_spread <= SETTLED_CL_SPREAD)]
                         for a, r in zip(self.alphas, self.results)])

    def write(self, directory: str | Path) -> Path:
        directory = Path(directory)
        directory.mkdir(parents=True, exist_ok=True)
        np.savetxt(directory / "polar.dat", self.table(),
                   header="alpha_deg cl cd cd_friction cm orders_dropped iterations cl_spread settled",
                   fmt=["%.4f", "%.8f", "%.8f", "%.8f", "%.8f", "%.3f", "%d", "%.3e", "%d"])
        (directory / "polar_metadata.json").write_text(json.dumps({
            "case": self.case.name, "alphas": self.alphas.tolist(), "timing": self.timing.record(),
            "settled_cl_spread": SETTLED_CL_SPREAD,
            "exits": [r.history.reason for r in self.results],
        }, indent=2, default=float))
        return directory


def at_alpha(case: Case, alpha: float) -> Case:
    """``case`` at angle of attack ``alpha`` degrees (``src/jaxrans/polar.py:75-77``)."""
    flow = dataclasses.replace(case.flow, alpha_deg=float(alpha))
    return dataclasses.replace(case, flow=flow, name=f"{case.name}_a{alpha:+.2f}")


def run_polar(case: Case, alphas, grid: Plan | None = None, devices: int | None = None,
              progress=None, release: bool = True) -> Polar:
    """``case`` at every angle of ``alphas`` (degrees) at once on one GPU;
    ``progress(iteration, CL per angle)`` per block (``src/jaxrans/polar.py:80-121``)."""
    if devices is not None and devices > 1:
        raise ValueError("a polar runs on one GPU in jaxrans_b200 (run one polar per GPU)")
    grid = case.grid() if grid is None else grid
    alphas = np.asarray(alphas, dtype=float)
    cases = [at_alpha(case, a) for a in alphas]
    results: list[Result] = run_batch(cases, [grid] * len(cases), progress=progress, release=release)
    return Polar(case, alphas, results, results[0].timing)


def main(argv: list[str] | None = None) -> int:
    parser = argparse.ArgumentParser(prog="python -m jaxrans_b200.polar", description=__doc__.splitlines()[0])
    parser.add_argument("case_dir")
    parser.add_argument("--alpha", nargs=3, type=float, required=True, metavar=("START", "STOP", "STEP"))
    parser.add_argument("--set", action="append", default=[], metavar="file.section.key=value")
    parser.add_argument("--out", default=None)
    parser.add_argument("--quiet", action="store_true")
    args = parser.parse_args(argv)
    try:
        case = load_case(args.case_dir, tuple(args.set))
    except CaseError as e:
        print(f"error: {e}", file=sys.stderr)
        return 2
    start, stop, step = args.alpha
    alphas = np.arange(start, stop + 0.5 * step, step)

    def progress(iteration, cl):
        if not args.quiet:
            print(f"{iteration:6d}  CL " + " ".join(f"{c:+.5f}" for c in cl), flush=True)

    polar = run_polar(case, alphas, progress=progress)
    out = polar.write(args.out or f"{case.name}_polar")
    if not args.quiet:
        for row in polar.table():
            print(f"alpha {row[0]:+7.2f}  CL {row[1]:+.6f}  CD {row[2]:+.6f}  CM {row[4]:+.6f}")
        print(f"wrote {out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
