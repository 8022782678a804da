"""Serving cavity requests on one GPU: Poisson arrivals, admission against a device-memory budget, continuous
batching, and the time-to-solution of every request.

A request is a cavity (grid size, Reynolds number, lid shape) with its initial noise, to be run until its
clock reaches `t_end`.  The server advances every running cavity `chunk` steps per round.  Running cavities of
the same grid size share slot batches (`cavity_batch_create_slots`: one launch per kernel for all slots, one
CUDA graph per batch built once); a request takes a free slot (`cavity_batch_set_member`) and gives it back when
it finishes, so joining and leaving rebuild nothing.  While a round's steps run on the GPU, the host admits
waiting requests in arrival order, as long as their estimated device bytes (`cavity_estimate_bytes`) fit in
the budget, and a set-up thread creates them and runs their initial projection on their own streams; they join
the first round after their set-up is done.  A request finishes at the end of the first round in which its
clock reaches `t_end`; its time to solution is that moment minus its arrival.  With `batched=False, max_running=1` the same loop serves one request at a time through its own graph
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
    batch: object = None          # the slot batch it runs in (batched serving)
    slot: int = -1


def _set_up(request, precision, library):
    """Create and initialise a request's cavity (runs on the set-up thread)."""
    cav = Cavity(request.settings, precision=precision, library=library)
    try:
        cav.initialize(*request.initial_fields(cav.shapes))
    except Exception:
        cav.close()
        raise
    return cav


class Server:
    """`batched`: running cavities of one grid size share slot batches of `slots` slots (one CUDA graph per
    batch, built once; a request takes a free slot when its set-up is done and frees it when it finishes, with no
    graph rebuilt).  Otherwise every cavity steps through its own graphs.  `setup_threads` threads create and
    initialise admitted requests while the GPU runs the round (0: on the serving thread)."""

    def __init__(self, budget_bytes=120e9, precision='mixed', chunk=8, batched=True, max_running=None,
                 library=None, slots=8, setup_threads=1):
        self.budget = float(budget_bytes)
        self.precision = precision
        self.chunk = int(chunk)
        self.batched = batched
        self.max_running = max_running
        self.library = library
        self.slots = int(slots)
        self.setup_threads = int(setup_threads)

    def run(self, requests, on_finish=None):
        """Serve `requests` in real time; returns one Result per request, in id order.  `on_finish(request,
        cavity)`, if given, sees each cavity at its final state before it is released."""
        from concurrent.futures import ThreadPoolExecutor
        waiting = sorted(requests, key=lambda r: r.arrival)
        running = []
        setting_up = []               # (request, admitted time, bytes, future or cavity)
        batches = {}                  # size key -> [Batch]
        results = {}
        in_use = 0.0
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        pool = ThreadPoolExecutor(self.setup_threads) if self.setup_threads > 0 else None

        def admit():
            nonlocal in_use
            while waiting and waiting[0].arrival <= now():
                if self.max_running is not None and len(running) + len(setting_up) >= self.max_running:
                    return
                req = waiting[0]
                need = float(estimate_bytes(req.settings, self.precision, self.library))
                if (running or setting_up) and in_use + need > self.budget:
                    return
                waiting.pop(0)
                job = (pool.submit(_set_up, req, self.precision, self.library) if pool
                       else _set_up(req, self.precision, self.library))
                setting_up.append((req, now(), need, job))
                in_use += need

        def join(block):
            """Cavities whose set-up is done start running (in slot batches when batched)."""
            still = []
            for req, admitted, need, job in setting_up:
                if pool and not block and not job.done():
                    still.append((req, admitted, need, job))
                    continue
                cav = job.result() if pool else job
                r = _Running(req, cav, admitted, need, (cav.nx, cav.ny, cav.nz))
                if self.batched:
                    group = batches.setdefault(r.key, [])
                    for b in group:
                        free = b.free_slots()
                        if free:
                            b.set_member(free[0], cav)
                            r.batch, r.slot = b, free[0]
                            break
                    else:
                        b = Batch([cav], capacity=self.slots)
                        group.append(b)
                        r.batch, r.slot = b, 0
                running.append(r)
            setting_up[:] = still

        try:
            while waiting or running or setting_up:
                join(block=not running)
                if not running:
                    time.sleep(max(0.0, min(waiting[0].arrival - now(), 0.05)) if waiting else 0.0)
                    admit()
                    continue
                # one round: every running cavity advances `chunk` steps; requests that arrive meanwhile are set up
                # on the set-up thread while the round runs, and join the next one
                if self.batched:
                    live = [b for group in batches.values() for b in group if b.cavities]
                    for b in live:
                        b.step_async(self.chunk)
                    admit()
                    reports = {}
                    for b in live:
                        for cav, rep in zip(b.slots, b.sync()):
                            if cav is not None:
                                reports[id(cav)] = rep
                else:
                    for r in running:
                        r.cavity.step_async(self.chunk)
                    admit()
                    reports = {id(r.cavity): r.cavity.sync() for r in running}
                t_round = now()
                still = []
                for r in running:
                    rep = reports[id(r.cavity)]
                    if rep['time'] >= r.request.t_end:
                        results[r.request.id] = Result(r.request.id, r.cavity.n_cell, r.request.arrival, r.admitted,
                                                       t_round, rep['steps'], rep['time'])
                        in_use -= r.bytes
                        if r.batch is not None:
                            r.batch.set_member(r.slot, None)
                        if on_finish is not None:
                            on_finish(r.request, r.cavity)
                        r.cavity.close()
                    else:
                        still.append(r)
                running = still
                # batches left empty are released
                for key in list(batches):
                    keep = []
                    for b in batches[key]:
                        if b.cavities:
                            keep.append(b)
                        else:
                            b.close()
                    batches[key] = keep
        finally:
            for group in batches.values():
                for b in group:
                    b.close()
            for r in running:
                r.cavity.close()
            for req, admitted, need, job in setting_up:
                try:
                    (job.result() if pool else job).close()
                except Exception:
                    pass
            if pool:
                pool.shutdown(wait=True)
        return [results[k] for k in sorted(results)]


def summary(results):
    """p50 / p99 time to solution (s) and the cell-updates per second of the whole run."""
    tts = np.array([r.time_to_solution for r in results])
    span = max(r.finished for r in results) - min(r.arrival for r in results)
    work = sum(r.cells * r.steps for r in results)
    return {'requests': len(results), 'p50_s': float(np.percentile(tts, 50)), 'p99_s': float(np.percentile(tts, 99)),
            'mean_s': float(tts.mean()), 'span_s': span, 'cell_updates_per_s': work / span}
