"""Many independent cavities advanced together on one GPU.

Two ways of stepping them:

* batched (the default): cavities of the same precision form are grouped into batches (`cavity_batch_create`),
  whatever their grid sizes.  One CUDA graph steps a whole batch, and each of its kernel launches covers every
  cavity of the batch through a work list of (cavity, block) entries, so a step of B cavities costs the launches
  of one.  Cavities whose launch sequences differ (the tensor-core transforms of the mixed form from 128^3 cells
  up, for instance) go to separate batches, by size, which run on their own streams, concurrently.
  `group='size'` batches by grid size only.
* per cavity (`batched=False`): every cavity steps through its own stream and graphs; the graph launches of all
  cavities are enqueued before waiting for any, so small, latency-bound kernels of different cavities overlap.

Results do not depend on the mix or on the way of stepping: each cavity's kernels read and write only its own
buffers and control block, and its reductions have a fixed order.
"""
import time

from . import workloads
from .api import Batch, Cavity


class Ensemble:
    def __init__(self, cases, library=None, batched=True, group='precision'):
        """`cases`: dicts with `settings`, `noise`, `seed` and `precision` (see workloads.ensemble_cases);
        `group`: 'precision' (one batch per precision form where the launch sequences agree) or 'size'."""
        self.cases = list(cases)
        self.cavities = []
        self.batches = []
        self.groups = []              # member indices of each batch
        try:
            for case in self.cases:
                cav = Cavity(case['settings'], precision=case.get('precision', 'mixed'), library=library)
                self.cavities.append(cav)
                cav.initialize(*workloads.initial_noise(cav.shapes, case['noise'], case['seed']))
            if batched:
                by_size, by_form = {}, {}
                for i, (case, cav) in enumerate(zip(self.cases, self.cavities)):
                    form = case.get('precision', 'mixed')
                    by_size.setdefault((cav.nx, cav.ny, cav.nz, form), []).append(i)
                    by_form.setdefault(form, []).append(i)
                groups = list(by_size.values())
                if group == 'precision':
                    groups = []
                    for form, members in by_form.items():
                        sizes = [k for k in by_size if k[3] == form]
                        if len(sizes) > 1 and self._try_batch(members):
                            continue
                        groups += [by_size[k] for k in sizes]
                for members in groups:
                    self.batches.append(Batch([self.cavities[i] for i in members]))
                    self.groups.append(members)
        except Exception:
            self.close()
            raise
        self.cells = [c.n_cell for c in self.cavities]

    def _try_batch(self, members):
        """One batch of cavities of different sizes; False when their launch sequences differ."""
        try:
            batch = Batch([self.cavities[i] for i in members])
        except RuntimeError as exc:
            if 'launch sequences differ' in str(exc):
                return False
            raise
        self.batches.append(batch)
        self.groups.append(members)
        return True

    def advance(self, steps, chunk=8):
        """Advance every cavity by `steps` steps, `chunk` queued per cavity (or batch) between waits; returns the
        reports of the last step, in case order."""
        done = 0
        reports = None
        while done < steps:
            n = min(chunk, steps - done)
            if self.batches:
                for b in self.batches:
                    b.step_async(n)
                reports = [None] * len(self.cavities)
                for b, members in zip(self.batches, self.groups):
                    for i, r in zip(members, b.sync()):
                        reports[i] = r
            else:
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
        for b in self.batches:
            b.close()
        self.batches = []
        self.groups = []
        for cav in self.cavities:
            cav.close()
        self.cavities = []
