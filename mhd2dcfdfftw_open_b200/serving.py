"""Serving: simulation jobs admitted continuously onto one GPU.

A job is one periodic domain (grid size, d_i, resistivity and viscosity,
step count, initial condition) advanced by the fused RK3 steps of
libmhdgpu.so, with the reference's CFL time-step control (calcDt,
timeAdvance.c:38-153) unless the job fixes dt.  Each job owns a context: its
fields stay on the device from admission to completion, and its kernels run
on the context's own CUDA stream.

`Server` keeps `slots` worker threads.  A request that arrives while others
run is admitted as soon as a slot is free and the HBM budget holds its
footprint (first come, first served: a request that does not fit waits, and
the ones behind it wait with it).  The admitted jobs' kernels run
concurrently on their streams, so small grids fill the GPU together.  Every
job's arithmetic is independent of the others (no shared scratch, no
atomics), so a job returns the same fields alone and in the mix.

Requests of the ensemble and serving workloads are drawn by `draw_requests`:
sizes from a list (probability proportional to 1/cells for serving), the
Orszag-Tang or the turbulence generator by seed parity, d_i ~ U[0, 0.1],
eta = nu ~ logU[1e-4, 1e-3], Hall = 1, CFL 0.3, Poisson arrivals.

    python -m mhd2dcfdfftw_open_b200.serving --requests 200 --rate 20 --slots 32

prints one JSON line: p50/p99 completion latency, sustained cell-updates/s,
and the same stream run plain FP64 one job at a time (--baseline).
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import threading
import time

import numpy as np

from . import ic
from .solver import Domain

SERVING_SIZES = ((128, 128), (256, 256), (512, 512), (1024, 1024), (2048, 2048))
ENSEMBLE_SIZES = ((128, 128), (256, 128), (256, 256), (512, 256), (512, 512),
                  (1024, 512), (1024, 1024))


def footprint_bytes(nx: int, ny: int, nvar: int = 8) -> int:
    """Device bytes of one context: the reference's field arrays (uu, dudx,
    dudy, dudt, dudtRK of nvar fields; 24 more fields of second derivatives,
    divB terms and the electric field and its derivatives) plus 8 MiB for
    tables, reductions and allocation rounding."""
    return (5 * nvar + 24) * nx * ny * 8 + (8 << 20)


@dataclasses.dataclass
class Request:
    rid: int
    nx: int
    ny: int
    steps: int
    di: float = 0.0
    eta: float = 1e-4
    nu: float = 1e-4
    kind: str = "ot"          # "ot" (Orszag-Tang) or "turbulence"
    seed: int = 1
    dt_fixed: float = 0.0     # <= 0: CFL control
    dt0: float = 1e-4         # first dt of CFL control
    mixed: bool = False       # mixed-precision fused steps
    arrival: float = 0.0      # seconds after the stream started
    keep_state: bool = False  # return the final fields

    def build(self):
        if self.kind == "ot":
            return ic.orszag_tang(self.nx, self.ny, di=self.di, eta=self.eta, nu=self.nu,
                                  Hall=1, cfl=0.3)
        return ic.alfvenic_turbulence(self.nx, self.ny, seed=self.seed, di=self.di,
                                      eta=self.eta, nu=self.nu, mmax=min(16, self.ny // 8),
                                      Hall=1, cfl=0.3)


@dataclasses.dataclass
class Result:
    rid: int
    cells: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    dt: float
    energy: float
    uu: np.ndarray | None = None
    error: str | None = None
    cross_helicity: float = float("nan")
    positive: bool = True     # every cell's density and pressure > 0 at the end

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    def record(self) -> dict:
        """The job's JSON record: size, steps, time step, energy and cross
        helicity at the end, latency, and its own cell-updates/s while admitted."""
        busy = self.finished - self.admitted
        return {"rid": self.rid, "cells": self.cells, "steps": self.steps, "dt": self.dt,
                "energy": self.energy, "cross_helicity": self.cross_helicity,
                "latency_s": self.latency, "queued_s": self.admitted - self.arrival,
                "cell_updates_per_s": self.cells * self.steps / busy if busy > 0 else None,
                "positive": self.positive, "error": self.error}


class Server:
    """Continuous batching of simulation jobs on one GPU."""

    def __init__(self, budget_bytes: float = 150e9, slots: int = 8, device: int = 0,
                 chunk: int = 0):
        self.budget = float(budget_bytes)
        self.device = device
        self.chunk = chunk  # steps per library call (0: the whole job)
        self._cv = threading.Condition()
        self._queue: list[Request] = []
        self._reserved = 0.0
        self._stop = False
        self._t0 = None
        self.results: list[Result] = []
        self._workers = [threading.Thread(target=self._work, daemon=True) for _ in range(slots)]
        for w in self._workers:
            w.start()

    def clock(self) -> float:
        return time.perf_counter() - self._t0

    def start_clock(self):
        with self._cv:
            self._t0 = time.perf_counter()

    def submit(self, req: Request):
        if footprint_bytes(req.nx, req.ny) > self.budget:
            raise ValueError(f"request {req.rid}: {req.nx}x{req.ny} exceeds the HBM budget")
        with self._cv:
            if self._t0 is None:
                self._t0 = time.perf_counter()
            self._queue.append(req)
            self._cv.notify_all()

    def _take(self):
        with self._cv:
            while True:
                if self._queue:
                    head = self._queue[0]
                    fp = footprint_bytes(head.nx, head.ny)
                    if self._reserved + fp <= self.budget:
                        self._queue.pop(0)
                        self._reserved += fp
                        return head, fp
                elif self._stop:
                    return None, 0
                self._cv.wait()

    def _work(self):
        while True:
            req, fp = self._take()
            if req is None:
                return
            admitted = self.clock()
            res = None
            try:
                res = self._run(req, admitted)
            finally:
                # the reservation is returned whatever happened to the job,
                # so a queued head request can always be admitted later
                with self._cv:
                    self._reserved -= fp
                    if res is None:
                        res = Result(req.rid, req.nx * req.ny, req.steps, req.arrival, admitted,
                                     self.clock(), 0.0, float("nan"), None,
                                     "worker failed before recording a result")
                    self.results.append(res)
                    self._cv.notify_all()

    def _run(self, req: Request, admitted: float) -> Result:
        try:
            p, uu = req.build()
            with Domain(p, uu, device=self.device) as d:
                d.set_precision(req.mixed)
                dt = req.dt0
                left = req.steps
                while left > 0:
                    n = left if self.chunk <= 0 else min(left, self.chunk)
                    dt = d.steps(n, req.dt_fixed, dt=dt, fused=True)
                    left -= n
                diag = d.diagnostics()
                out = d.get("uu") if req.keep_state else None
            # a state that left the finite numbers is this job's error, not the
            # server's; a finite state with a non-positive density or pressure
            # (which the reference also carries on with) is flagged, not failed
            err = None if diag["finite"] else "non-finite state (NaN or Inf) at the end of the job"
            return Result(req.rid, req.nx * req.ny, req.steps, req.arrival, admitted,
                          self.clock(), dt, diag["energy"], out, err, diag["cross_helicity"],
                          diag["positive"])
        except Exception as exc:  # reported per job, the server keeps serving
            return Result(req.rid, req.nx * req.ny, req.steps, req.arrival, admitted,
                          self.clock(), 0.0, float("nan"), None, str(exc))

    def cancel(self, rid: int) -> bool:
        """Withdraw a request that has not been admitted yet; False when it
        is running, finished or unknown."""
        with self._cv:
            for i, q in enumerate(self._queue):
                if q.rid == rid:
                    self._queue.pop(i)
                    self._cv.notify_all()
                    return True
        return False

    def drain(self):
        """Wait for every submitted job, then stop the workers."""
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for w in self._workers:
            w.join()


    def load_bytes(self) -> float:
        """Current load: footprint bytes of the running jobs plus those of
        the queued requests, read under the server's lock."""
        with self._cv:
            return self._reserved + sum(footprint_bytes(q.nx, q.ny) for q in self._queue)


class Router:
    """Several GPUs of one node: one Server per device, each request placed
    whole on the device with the least current load (footprint bytes of its
    running and queued jobs; ties to the lower device).  Jobs never span
    devices, so no collective is involved; results are gathered on the host."""

    def __init__(self, devices, budget_bytes: float = 150e9, slots: int = 8,
                 server_cls=None):
        cls = server_cls or Server
        self.servers = [cls(budget_bytes, slots, d) for d in devices]
        self._lock = threading.Lock()
        self.placement: dict = {}

    def start_clock(self):
        for s in self.servers:
            s.start_clock()

    def clock(self) -> float:
        return self.servers[0].clock()

    def submit(self, req: Request):
        with self._lock:
            loads = [s.load_bytes() for s in self.servers]
            k = min(range(len(self.servers)), key=lambda i: (loads[i], i))
            self.placement[req.rid] = self.servers[k].device
            # submitted under the router's lock, so the next placement sees it
            self.servers[k].submit(req)

    def drain(self):
        for s in self.servers:
            s.drain()
        return [r for s in self.servers for r in s.results]


def pretune(requests, device=0):
    """Autotune the x-pass tiling once per grid shape of the stream, each on an
    idle GPU before the stream starts; the library keeps the choice for every
    later context of that shape in this process."""
    seen = set()
    for r in requests:
        if (r.nx, r.ny) in seen:
            continue
        seen.add((r.nx, r.ny))
        p, uu = r.build()
        with Domain(p, uu, device=device) as d:
            d.autotune()
    return sorted(seen)


def run_stream(requests, budget_bytes=150e9, slots=8, device=0, realtime=True, devices=None):
    """Feed `requests` to a Server (or, with `devices`, a Router over those
    GPUs) at their arrival times (realtime) or all at once; return (results,
    wall seconds)."""
    srv = Router(devices, budget_bytes, slots) if devices else Server(budget_bytes, slots, device)
    srv.start_clock()
    for r in sorted(requests, key=lambda q: q.arrival):
        if realtime:
            wait = r.arrival - srv.clock()
            if wait > 0:
                time.sleep(wait)
        else:
            r.arrival = srv.clock()
        srv.submit(r)
    results = srv.drain() if devices else (srv.drain() or srv.results)
    wall = max(x.finished for x in results) if results else 0.0
    return sorted(results, key=lambda x: x.rid), wall


def summarize(results, wall):
    """Stream statistics.  `cell_updates_per_s` counts every job the GPU ran;
    `finite_cell_updates_per_s` counts only the jobs that ended with a finite
    state (no error), and its latencies are over those jobs alone."""
    lat = np.array([r.latency for r in results])
    ok = [r for r in results if not r.error]
    lat_ok = np.array([r.latency for r in ok])
    work = float(sum(r.cells * r.steps for r in results))
    work_ok = float(sum(r.cells * r.steps for r in ok))
    nonfinite = sum(1 for r in results if r.error and "non-finite" in r.error)
    nonpositive = sum(1 for r in results if not r.error and not r.positive)
    return {"jobs": len(results), "failed": sum(1 for r in results if r.error),
            "nonfinite": nonfinite, "finite_but_nonpositive": nonpositive,
            "p50_latency_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "cell_updates": work, "wall_s": wall,
            "cell_updates_per_s": work / wall if wall > 0 else None,
            "finite_jobs": len(ok), "finite_cell_updates": work_ok,
            "finite_cell_updates_per_s": work_ok / wall if wall > 0 else None,
            "finite_p50_latency_s": float(np.percentile(lat_ok, 50)) if len(lat_ok) else None,
            "finite_p99_latency_s": float(np.percentile(lat_ok, 99)) if len(lat_ok) else None}


def draw_requests(n, seed=5, rate=20.0, sizes=SERVING_SIZES, inverse_cells=True,
                  steps=(100, 2000), mixed=True):
    """Seeded request stream: sizes (probability proportional to 1/cells when
    inverse_cells), generator by seed parity, d_i ~ U[0, 0.1], eta = nu ~
    logU[1e-4, 1e-3], steps ~ U[steps], Poisson arrivals at `rate` per
    second (rate <= 0: all at time 0)."""
    rng = np.random.default_rng(seed)
    w = np.array([1.0 / (a * b) if inverse_cells else 1.0 for a, b in sizes])
    w /= w.sum()
    t = 0.0
    out = []
    for i in range(n):
        nx, ny = sizes[rng.choice(len(sizes), p=w)]
        s = int(rng.integers(steps[0], steps[1] + 1))
        di = float(rng.uniform(0.0, 0.1))
        eta = float(10 ** rng.uniform(-4, -3))
        js = int(rng.integers(1, 1 << 30))
        if rate > 0:
            t += float(rng.exponential(1.0 / rate))
        out.append(Request(i, int(nx), int(ny), s, di=di, eta=eta, nu=eta,
                           kind="ot" if js % 2 == 0 else "turbulence", seed=js,
                           mixed=mixed, arrival=t))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--slots", type=int, default=32)
    ap.add_argument("--gpus", type=int, default=1, help="route jobs over this many GPUs")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--steps-min", type=int, default=100)
    ap.add_argument("--steps-max", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--fp64", action="store_true", help="serve in FP64 instead of mixed")
    ap.add_argument("--ensemble", action="store_true",
                    help="ensemble sizes, uniform, all submitted at once")
    ap.add_argument("--baseline", action="store_true",
                    help="also run the same stream plain FP64, one job at a time")
    ap.add_argument("--records", default="", help="write one JSON record per job to this file")
    a = ap.parse_args(argv)
    sizes = ENSEMBLE_SIZES if a.ensemble else SERVING_SIZES
    rate = 0.0 if a.ensemble else a.rate
    reqs = draw_requests(a.requests, a.seed, rate, sizes, not a.ensemble,
                         (a.steps_min, a.steps_max), mixed=not a.fp64)
    for dev in range(max(1, a.gpus)):
        pretune(reqs, dev)  # the served stream and the baseline share the tiling
    res, wall = run_stream(reqs, a.budget_gb * 1e9, a.slots, realtime=rate > 0,
                           devices=list(range(a.gpus)) if a.gpus > 1 else None)
    if a.records:
        with open(a.records, "w") as f:
            for r in res:
                f.write(json.dumps(r.record()) + "\n")
    out = {"workload": "ensemble" if a.ensemble else "serving", "requests": a.requests,
           "rate_per_s": rate, "slots": a.slots, "precision": "fp64" if a.fp64 else "mixed",
           "served": summarize(res, wall)}
    if a.baseline:
        base = draw_requests(a.requests, a.seed, rate, sizes, not a.ensemble,
                             (a.steps_min, a.steps_max), mixed=False)
        bres, bwall = run_stream(base, a.budget_gb * 1e9, 1, realtime=rate > 0)
        out["baseline_fp64_one_at_a_time"] = summarize(bres, bwall)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
