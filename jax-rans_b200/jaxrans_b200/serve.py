"""Serving: a request loop with continuous batching.

Requests (2D cases, each with its own section, grid size and flow) arrive over time.
Pools of device slots (each a device batch, ``jr_batch_create``) hold the requests of one
grid size.  A request is admitted as soon as it has arrived and a slot of its grid size
is free: the slot's static tables are overwritten with the request's grid
(``jr_case_load``), its state reset to the request's freestream, and it joins the next
block of Newton steps.  When every slot of its size is taken, another pool of that size
is made if the free device memory allows (``Admission``: a share of the free memory,
keeping room for the grid sizes not seen yet); otherwise the request waits, and while a
request waits for memory, pools that have gone idle and whose size has no request
waiting are released, so the memory moves to the sizes in demand.  Every pool steps all
its live slots with one captured graph per Newton step, on its own stream, so the pools'
work overlaps on the device.  After each block the host runs each live request's exit
test (``jaxrans_b200.solver.CaseMonitor``, the exit test of a single run); a finished
request frees its slot at once.  States and preconditioner factors stay resident on the
device for the whole life of a request.

A request's result is the same as the same case run alone: slots never interact, and
each slot's reductions are split as for a single case.
"""

from __future__ import annotations

import copy
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .case import Case
from .plan import Plan
from .solver import CaseMonitor, ConvergenceHistory, Forces, freestream_state

# C-grid sizes (nodes) of the served requests: cells round the airfoil, along each wake
# side, normal to the wall
GRID_CLASSES = {
    (193, 49): (128, 32, 48),
    (385, 97): (256, 64, 96),
    (513, 129): (344, 84, 128),
    (769, 193): (512, 128, 192),
}


@dataclass
class Request:
    """A case and its arrival time (seconds from the start of the stream)."""

    id: int
    case: Case
    arrival: float
    grid_key: tuple = ()


@dataclass
class Served:
    """A finished request: its exit, forces, history, and its times on the server."""

    request: Request
    reason: str
    forces: Forces
    history: ConvergenceHistory
    U: np.ndarray
    admitted: float
    finished: float

    @property
    def latency(self) -> float:
        """Seconds from arrival to result."""
        return self.finished - self.request.arrival


def request_case(template: Case, airfoil: str, size: tuple, mach: float, alpha: float, reynolds: float,
                 name: str, classes: dict = GRID_CLASSES) -> Case:
    """``template`` (its numerics, model and boundary conditions) on a C-grid of ``size``
    nodes round ``airfoil`` at the given flow."""
    from .case import parse_case
    around, wake, normal = classes[size]
    doc = copy.deepcopy(template.raw["case"])
    num = copy.deepcopy(template.raw["numerical"])
    doc["general"] = {"case_name": name}
    doc["domain"] = dict(doc["domain"], airfoil=airfoil, cells_airfoil=around, cells_wake=wake,
                         cells_normal=normal)
    doc["freestream"] = dict(doc["freestream"], mach=float(mach), alpha_deg=float(alpha), reynolds=float(reynolds))
    return parse_case(doc, num)


def poisson_requests(n: int, template: Case, rate: float = 20.0, seed: int = 0,
                     classes: dict = GRID_CLASSES) -> list[Request]:
    """``n`` requests with Poisson arrivals of mean ``rate`` per second: NACA 4-digit
    sections of max camber 0-6 %, camber position 20-50 %, thickness 6-24 %, a C-grid
    size from ``sizes``, M uniform on [0.15, 0.78], alpha uniform on [-5, 15] deg, Re
    log-uniform on [1e6, 2e7]; all from ``seed``."""
    rng = np.random.default_rng(seed)
    sizes = tuple(classes)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        camber = int(rng.integers(0, 7))
        position = int(rng.integers(2, 6)) if camber else 0
        thickness = int(rng.integers(6, 25))
        airfoil = f"naca{camber}{position}{thickness:02d}"
        size = sizes[int(rng.integers(0, len(sizes)))]
        mach = float(rng.uniform(0.15, 0.78))
        alpha = float(rng.uniform(-5.0, 15.0))
        reynolds = float(10.0 ** rng.uniform(6.0, np.log10(2e7)))
        case = request_case(template, airfoil, size, mach, alpha, reynolds, f"req{i:04d}", classes)
        out.append(Request(i, case, t, size))
    return out


def case_bytes(plan: Plan, nvar: int, m: int, mixed: bool) -> int:
    """Device bytes one slot of this grid takes (work vectors, basis, line factor)."""
    n_vec = nvar * plan.NI * plan.NJ
    tb = 4 if mixed else 8
    rows = int(plan.chains.lengths.sum()) + 16 * plan.chains.cells.shape[0]
    return 11 * n_vec * 8 + (m + 1) * n_vec * tb + rows * (80 + 5 + 104) * tb + 32 * plan.NI * plan.NJ * 8


@dataclass
class Pool:
    """The slots of one grid size: a device batch and who holds each slot."""

    key: tuple
    dev: object
    slots: int
    holder: list = field(default_factory=list)     # Request or None per slot
    monitor: list = field(default_factory=list)    # CaseMonitor or None per slot
    admitted: list = field(default_factory=list)

    def free_slot(self):
        for k, h in enumerate(self.holder):
            if h is None:
                return k
        return None

    @property
    def live(self) -> bool:
        return any(h is not None for h in self.holder)


@dataclass
class Admission:
    """The serving loop's use of device memory: how many slots a new pool gets, and which
    idle pools give their memory back.

    A new pool of grid size ``key`` gets ``memory_fraction`` of the free memory, shared
    with the grid sizes (of ``n_classes``) that have no pool yet, in slots of
    ``per_slot`` bytes, at most ``max_slots``; none (the request waits) when not one slot
    fits.  While some request waits for memory (``starved`` sizes), the pools with no
    live slot whose size has no request waiting (``waiting`` sizes) are released."""

    max_slots: int = 64
    memory_fraction: float = 0.8
    n_classes: int = 4

    def new_pool_slots(self, free: int, per_slot: int, key, keys_with_pools) -> int:
        unseen = max(0, self.n_classes - len(set(keys_with_pools) | {key}))
        share = self.memory_fraction * free / (1 + unseen)
        return int(max(0, min(self.max_slots, share // max(1, per_slot))))

    @staticmethod
    def releasable(pools, starved, waiting) -> list:
        if not starved:
            return []
        return [p for p in pools if not p.live and p.key not in waiting]


def build_grid(case: Case) -> Plan:
    """A request's grid and plan tables (run in a worker process)."""
    return case.grid()


class Server:
    """Continuous batching of requests over pools of device slots, pools per grid size
    made and released by the free device memory (``Admission``).

    ``max_slots`` caps a pool; ``memory_fraction`` of the free device memory, shared by
    the grid sizes still without a pool, bounds it when the pool is made.  Each request's
    grid is generated on the host by a pool of ``workers`` processes from the moment it
    arrives, while the device steps the admitted ones."""

    def __init__(self, max_slots: int = 64, memory_fraction: float = 0.8, block_iters: int | None = None,
                 n_classes: int = len(GRID_CLASSES), workers: int = 4):
        self.admission = Admission(max_slots, memory_fraction, n_classes)
        self.workers = workers
        self.block_iters = block_iters
        self.pools: list[Pool] = []
        self.made = 0        # pools made over the stream
        self.released = 0    # idle pools released for sizes waiting on memory

    def free_pool(self, key) -> tuple:
        """A pool of grid size ``key`` with a free slot, and the slot (or (None, None))."""
        for pool in self.pools:
            if pool.key == key:
                slot = pool.free_slot()
                if slot is not None:
                    return pool, slot
        return None, None

    def make_pool(self, req: Request, plan: Plan) -> Pool | None:
        """Another pool of the request's grid size, as large as the free memory allows;
        None when not one slot fits."""
        import torch
        from .batch import batch_device
        imp = req.case.implicit
        per = case_bytes(plan, req.case.flow.nvar, imp.krylov_subspace, imp.precision == "mixed")
        free, _ = torch.cuda.mem_get_info()
        slots = self.admission.new_pool_slots(free, per, req.grid_key, {p.key for p in self.pools})
        if slots < 1:
            if not self.pools:   # nothing to wait for: the request can never be admitted
                raise MemoryError(f"a request of grid size {req.grid_key} needs {per} bytes of device memory; "
                                  f"{free} are free")
            return None
        dev = batch_device([req.case] * slots, [plan] * slots)
        for k in range(slots):
            dev.enable(k, False)
        pool = Pool(req.grid_key, dev, slots, [None] * slots, [None] * slots, [0.0] * slots)
        self.pools.append(pool)
        self.made += 1
        return pool

    def release(self, pool: Pool) -> None:
        pool.dev.close()
        self.pools.remove(pool)
        self.released += 1

    def slots_by_size(self) -> dict:
        out: dict = {}
        for p in self.pools:
            out[p.key] = out.get(p.key, 0) + p.slots
        return out

    def admit(self, pool: Pool, slot: int, req: Request, plan: Plan, now: float) -> None:
        c = req.case
        pool.dev.load_case(slot, plan, c.flow, c.numerics, c.implicit, c.grid_spec.reference_length,
                           tuple(c.grid_spec.moment_centre[:2]))
        pool.dev.set_case_state(slot, freestream_state(c, plan), c.implicit.cfl, float("inf"))
        pool.dev.enable(slot, True)
        pool.holder[slot] = req
        pool.monitor[slot] = CaseMonitor(c)
        pool.admitted[slot] = now

    def serve(self, requests: list[Request], realtime: bool = True) -> list[Served]:
        """Run the stream to its end; ``realtime`` releases each request at its arrival on
        the wall clock, otherwise every request is there at the start."""
        import multiprocessing
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(self.workers, mp_context=multiprocessing.get_context("spawn")) as workers:
            return self._serve(requests, realtime, workers)

    def _serve(self, requests, realtime, workers) -> list[Served]:
        import torch
        block = self.block_iters or requests[0].case.block_iters
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        grids: dict = {}
        done: list[Served] = []
        hist_buf: dict = {}
        t0 = time.perf_counter()

        def clock():
            return time.perf_counter() - t0

        while pending or any(p.live for p in self.pools):
            t = clock() if realtime else float("inf")
            for req in pending:
                if req.arrival > t:
                    break
                if req.id not in grids:
                    grids[req.id] = workers.submit(build_grid, req.case)
            # admit, in arrival order, every arrived request whose grid is ready and that
            # finds a free slot of its size, or memory for another pool of it
            starved = set()
            for req in [r for r in pending if r.id in grids and grids[r.id].done()]:
                plan = grids[req.id].result()
                pool, slot = self.free_pool(req.grid_key)
                if pool is None and req.grid_key not in starved:
                    pool = self.make_pool(req, plan)
                    slot = pool.free_slot() if pool is not None else None
                if pool is None:
                    starved.add(req.grid_key)
                    continue
                self.admit(pool, slot, req, plan, clock())
                pending.remove(req)
                del grids[req.id]
            waiting = {r.grid_key for r in pending if r.arrival <= t}
            for pool in self.admission.releasable(self.pools, starved, waiting):
                hist_buf.pop(id(pool), None)
                self.release(pool)
            live = [p for p in self.pools if p.live]
            if not live:
                time.sleep(0.01)
                continue
            # one block of every live pool, each on its own stream: the pools overlap
            for p in live:
                buf = hist_buf.get(id(p))
                if buf is None:
                    buf = hist_buf[id(p)] = torch.empty((block, p.slots), dtype=torch.float64, device="cuda")
                p.dev.newton_steps_async(block, buf)
            for p in live:
                p.dev.sync()
                hist = hist_buf[id(p)].cpu().numpy()
                forces = np.atleast_2d(p.dev.forces())
                finished_at = clock()
                for k, req in enumerate(p.holder):
                    if req is None:
                        continue
                    mon = p.monitor[k]
                    if mon.feed(hist[:, k], forces[k]):
                        U = p.dev.case_state(k)[0]
                        res = mon.residual()
                        history = ConvergenceHistory(res, mon.reason, int(res.size))
                        done.append(Served(req, mon.reason, mon.forces, history, U, p.admitted[k], finished_at))
                        p.dev.enable(k, False)
                        p.holder[k] = None
                        p.monitor[k] = None
        return sorted(done, key=lambda s: s.request.id)

    def close(self) -> None:
        for p in self.pools:
            p.dev.close()
        self.pools.clear()


def summary(served: list[Served], wall: float) -> dict:
    lat = np.array([s.latency for s in served])
    return {"requests": len(served), "solves_per_hr": 3600.0 * len(served) / wall,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "exits": {r: int(sum(s.reason == r for s in served)) for r in sorted({s.reason for s in served})}}


def main(argv=None) -> int:
    """Serve a seeded Poisson stream of SA requests and print a JSON summary; with
    ``--plain`` also solve the first requests one at a time on the plain FP64 path and
    compare rates and forces."""
    import argparse
    import dataclasses
    import json
    from .solver import march
    from .workloads import workload
    ap = argparse.ArgumentParser(prog="python -m jaxrans_b200.serve", description=main.__doc__)
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="mixed", choices=("fp64", "mixed"))
    ap.add_argument("--limiter", default="van_albada", help="the requests' MUSCL limiter")
    ap.add_argument("--max-slots", type=int, default=64)
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--plain", type=int, default=0, metavar="N",
                    help="also solve the first N requests alone on the plain FP64 path")
    args = ap.parse_args(argv)
    template = workload("c_sa_385", **{"implicit.precision": args.precision,
                                       "convective_fluxes.limiter": args.limiter})
    requests = poisson_requests(args.requests, template, args.rate, args.seed)
    server = Server(max_slots=args.max_slots, workers=args.workers)
    t = time.perf_counter()
    served = server.serve(requests)
    wall = time.perf_counter() - t
    out = summary(served, wall)
    out.update({"rate_per_s": args.rate, "seed": args.seed, "precision": args.precision, "limiter": args.limiter,
                "wall_s": wall, "slots": {f"{k[0]}x{k[1]}": n for k, n in server.slots_by_size().items()},
                "pools_made": server.made, "pools_released": server.released,
                "per_class": {f"{k[0]}x{k[1]}": summary([x for x in served if x.request.grid_key == k], wall)
                              for k in server.slots_by_size()}})
    server.close()
    if args.plain:
        seconds, dcl, dcd, rows = 0.0, [], [], []
        for x in served[: args.plain]:
            c = x.request.case
            plain = dataclasses.replace(c, implicit=dataclasses.replace(c.implicit, precision="fp64"))
            grid = plain.grid()
            t = time.perf_counter()
            r = march(plain, grid)
            seconds += time.perf_counter() - t
            dcl.append(abs(x.forces.cl - r.forces.cl))
            dcd.append(abs(x.forces.cd - r.forces.cd))
            rows.append({"id": x.request.id, "served": x.reason, "plain": r.history.reason,
                         "dcl": dcl[-1], "dcd_counts": 1e4 * dcd[-1]})
        out["plain_fp64"] = {"requests": args.plain, "solves_per_hr": 3600.0 * args.plain / seconds,
                             "seconds": seconds, "max_dcl": max(dcl), "max_dcd_counts": 1e4 * max(dcd),
                             "rows": rows}
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
