"""Serving cavity requests on one GPU: Poisson arrivals, admission against a device-memory budget, continuous
batching, and the time-to-solution of every request.

A request is a cavity (grid size, Reynolds number, lid shape) with its initial noise, to be run until its
clock reaches `t_end`.  The server advances every running cavity `chunk` steps per round.  Running cavities of
the same grid size are stepped as one batch (`cavity_batch_*`: one launch per kernel for all of them); a batch
is rebuilt when a request joins or leaves its group.  While a round's steps run on the GPU, the host admits
waiting requests in arrival order, as long as their estimated device bytes (`cavity_estimate_bytes`) fit in
the budget, and sets them up (solver creation and the initial projection); they join at the next round.  A
request finishes at the end of the first round in which its clock reaches `t_end`; its time to solution is
that moment minus its arrival.  With `batched=False, max_running=1` the same loop serves one request at a time through its own graph
(the plain form the batched server is compared with).
"""
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import workloads
from .api import Batch, Cavity, estimate_bytes

# grid sizes of the serving mix: cubes and one elongated cavity (nx, ny, nz)
SERVING_SIZES = ((32, 32, 32), (64, 64, 64), (64, 64, 128), (96, 96, 96), (128, 128, 128))


@dataclass
class Request:
    id: int
    arrival: float                 # seconds after the start of the run
    settings: dict
    t_end: float
    noise: float = 1e-3
    seed: int = 0
    fields: tuple = None           # the initial noise (v, w) the request arrives with; generated if None

    def initial_fields(self, shapes):
        if self.fields is None:
            return workloads.initial_noise(shapes, self.noise, self.seed)
        return self.fields


@dataclass
class Result:
    id: int
    cells: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    time: float

    @property
    def time_to_solution(self):
        return self.finished - self.arrival


def serving_requests(count, rate, seed=0, sizes=SERVING_SIZES, re_range=(100.0, 5000.0), t_end=5.0, cfl=0.5,
                     with_fields=False):
    """`count` requests with Poisson arrivals at `rate` per second: size uniform over `sizes`, Re log-uniform in
    `re_range`, lid half uniform and half regularised, uniform grid, adaptive dt at `cfl`.  `with_fields`: each
    request carries its initial noise (as a client would send it), instead of the server drawing it."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(count):
        t += float(rng.exponential(1.0 / rate))
        nx, ny, nz = sizes[int(rng.integers(len(sizes)))]
        re = float(math.exp(rng.uniform(math.log(re_range[0]), math.log(re_range[1]))))
        lid = 'uniform' if rng.random() < 0.5 else 'regularised'
        s = workloads.settings(nx, re, nz=nz, lid=lid, cfl=cfl)
        s['ny'] = ny
        req = Request(id=k, arrival=t, settings=s, t_end=t_end, seed=k)
        if with_fields:
            req.fields = workloads.initial_noise({'v': (nz, ny + 1, nx), 'w': (nz + 1, ny, nx)}, req.noise, req.seed)
        out.append(req)
    return out


@dataclass
class _Running:
    request: Request
    cavity: Cavity
    admitted: float
    bytes: int
    key: tuple = field(default=())


class Server:
    def __init__(self, budget_bytes=120e9, precision='mixed', chunk=8, batched=True, max_running=None,
                 library=None):
        self.budget = float(budget_bytes)
        self.precision = precision
        self.chunk = int(chunk)
        self.batched = batched
        self.max_running = max_running
        self.library = library

    def run(self, requests, on_finish=None):
        """Serve `requests` in real time; returns one Result per request, in id order.  `on_finish(request,
        cavity)`, if given, sees each cavity at its final state before it is released."""
        waiting = sorted(requests, key=lambda r: r.arrival)
        running = []
        batches = {}                  # size key -> (members' ids, Batch)
        results = {}
        in_use = 0.0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        def admit():
            nonlocal in_use
            while waiting and waiting[0].arrival <= now():
                if self.max_running is not None and len(running) + len(joining) >= self.max_running:
                    return
                req = waiting[0]
                need = float(estimate_bytes(req.settings, self.precision, self.library))
                if (running or joining) and in_use + need > self.budget:
                    return
                waiting.pop(0)
                cav = Cavity(req.settings, precision=self.precision, library=self.library)
                cav.initialize(*req.initial_fields(cav.shapes))
                joining.append(_Running(req, cav, now(), need, (cav.nx, cav.ny, cav.nz)))
                in_use += need

        joining = []
        try:
            while waiting or running or joining:
                running += joining
                joining = []
                if not running:
                    time.sleep(max(0.0, min(waiting[0].arrival - now(), 0.05)))
                    admit()
                    continue
                # one round: every running cavity advances `chunk` steps; requests that arrive meanwhile are set up
                # on the host (and their own streams) while the round runs, and join the next one
                if self.batched:
                    groups = {}
                    for r in running:
                        groups.setdefault(r.key, []).append(r)
                    for key in list(batches):
                        if key not in groups or batches[key][0] != [r.request.id for r in groups[key]]:
                            batches.pop(key)[1].close()
                    for key, members in groups.items():
                        if key not in batches:
                            batches[key] = ([r.request.id for r in members], Batch([r.cavity for r in members]))
                    for _, b in batches.values():
                        b.step_async(self.chunk)
                    admit()
                    reports = {}
                    for ids, b in batches.values():
                        for i, rep in zip(ids, b.sync()):
                            reports[i] = rep
                else:
                    for r in running:
                        r.cavity.step_async(self.chunk)
                    admit()
                    reports = {r.request.id: r.cavity.sync() for r in running}
                t_round = now()
                still = []
                for r in running:
                    rep = reports[r.request.id]
                    if rep['time'] >= r.request.t_end:
                        results[r.request.id] = Result(r.request.id, r.cavity.n_cell, r.request.arrival, r.admitted,
                                                       t_round, rep['steps'], rep['time'])
                        in_use -= r.bytes
                        key = r.key
                        if key in batches:
                            batches.pop(key)[1].close()
                        if on_finish is not None:
                            on_finish(r.request, r.cavity)
                        r.cavity.close()
                    else:
                        still.append(r)
                running = still
        finally:
            for _, b in batches.values():
                b.close()
            for r in running + joining:
                r.cavity.close()
        return [results[k] for k in sorted(results)]


def summary(results):
    """p50 / p99 time to solution (s) and the cell-updates per second of the whole run."""
    tts = np.array([r.time_to_solution for r in results])
    span = max(r.finished for r in results) - min(r.arrival for r in results)
    work = sum(r.cells * r.steps for r in results)
    return {'requests': len(results), 'p50_s': float(np.percentile(tts, 50)), 'p99_s': float(np.percentile(tts, 99)),
            'mean_s': float(tts.mean()), 'span_s': span, 'cell_updates_per_s': work / span}
