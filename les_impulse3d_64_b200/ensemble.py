"""Many independent cavities advanced together on one GPU.

Each cavity is a handle of the C ABI (`cavity_create`) with its own CUDA stream and step graphs; stepping
enqueues graph launches on every cavity's stream before waiting for any of them, so the small, latency-bound
kernels of different cavities run concurrently and fill the device.  Results do not depend on the mix: each
cavity's kernels read and write only its own buffers and control block, and its reductions have a fixed order.
"""
import time

import numpy as np

from . import workloads
from .api import Cavity


class Ensemble:
    def __init__(self, cases, library=None):
        """`cases`: dicts with `settings`, `noise`, `seed` and `precision` (see workloads.ensemble_cases)."""
        self.cases = list(cases)
        self.cavities = []
        try:
            for case in self.cases:
                cav = Cavity(case['settings'], precision=case.get('precision', 'mixed'), library=library)
                self.cavities.append(cav)
                cav.initialize(*workloads.initial_noise(cav.shapes, case['noise'], case['seed']))
        except Exception:
            self.close()
            raise
        self.cells = [c.n_cell for c in self.cavities]

    def advance(self, steps, chunk=8):
        """Advance every cavity by `steps` steps, `chunk` queued per cavity between waits; returns the reports
        of the last step."""
        done = 0
        reports = None
        while done < steps:
            n = min(chunk, steps - done)
            for cav in self.cavities:
                cav.step_async(n)
            reports = [cav.sync() for cav in self.cavities]
            done += n
        return reports

    def timed(self, steps, warmup=2, chunk=8):
        """Wall time of `steps` steps of every cavity after `warmup`; returns (seconds, cell-updates/s)."""
        self.advance(warmup, chunk)
        t0 = time.perf_counter()
        self.advance(steps, chunk)
        dt = time.perf_counter() - t0
        return dt, sum(self.cells) * steps / dt

    def device_bytes(self):
        return sum(c.device_bytes() for c in self.cavities)

    def fields(self, index, names=('u', 'v', 'w', 'phi')):
        return {k: self.cavities[index].field(k) for k in names}

    def close(self):
        for cav in self.cavities:
            cav.close()
        self.cavities = []
