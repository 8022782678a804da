"""The workloads' host side on the CPU: the run protocol's order of calls (main.py:342-363: step, probes, a kick
when one is due, then the statistics), the kick and initial noise, the stretched grid's first cell, and the C4
ensemble's cases.  A recording stand-in plays the solver."""
import math

import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads


class Recorder:
    """Stands in for a solver binding: logs every call run_protocol makes."""

    def __init__(self, n=8):
        self.shapes = {'u': (n, n, n + 1), 'v': (n, n + 1, n), 'w': (n + 1, n, n), 'phi': (n, n, n)}
        self.calls = []
        self.steps = 0
        self.ke = 1.0

    def step(self):
        self.steps += 1
        self.calls.append(('step', self.steps))
        return {'dt': 0.01 * self.steps, 'time': 0.01 * self.steps * (self.steps + 1) / 2, 'dt_reason': 'CFL',
                'phi_passes': 1}

    def probes(self):
        self.calls.append(('probes', self.steps))
        return np.full(16, self.steps, dtype=np.float32)

    def diagnostics(self):
        return {'kinetic_energy': self.ke}

    def kick(self, noise, amplitude, passes):
        self.calls.append(('kick', self.steps, amplitude, passes, float(noise[0].ravel()[0])))
        self.ke *= 2

    def add_statistics(self, weight):
        self.calls.append(('stats', self.steps, weight))
        return np.zeros(4)


WORKLOAD = dict(name='protocol', steps=6, kicks=((2, 1e-2), (4, 5e-3)), stats_from=3, seed=7)


def test_protocol_order_kicks_and_statistics_window():
    sim = Recorder()
    seen = []
    run = workloads.run_protocol(sim, WORKLOAD, snapshots=(3, 6), on_snapshot=lambda n, s: seen.append(n))
    kinds = [c[0] for c in sim.calls]
    # every step is followed by its probes; kicks follow steps 2 and 4; statistics from step 4 (n > stats_from)
    assert kinds == ['step', 'probes', 'step', 'probes', 'kick', 'step', 'probes', 'step', 'probes', 'kick',
                     'stats', 'step', 'probes', 'stats', 'step', 'probes', 'stats']
    kicks = [c for c in sim.calls if c[0] == 'kick']
    assert [(c[1], c[2], c[3]) for c in kicks] == [(2, 1e-2, workloads.KICK_PASSES), (4, 5e-3, workloads.KICK_PASSES)]
    # each kick draws its own noise: kick k of the run from seed + 1000 + k - 1
    first = [workloads.kick_noise(sim.shapes, WORKLOAD['seed'], k)[0].ravel()[0] for k in (1, 2)]
    assert [c[4] for c in kicks] == pytest.approx(first)
    stats = [c for c in sim.calls if c[0] == 'stats']
    assert [(c[1], c[2]) for c in stats] == [(4, 0.04), (5, 0.05), (6, 0.06)]      # weight = that step's dt
    assert seen == [3, 6]
    assert run['kick_ke'].tolist() == [[1.0, 2.0], [2.0, 4.0]]
    assert run['probes'].shape == (6, 16) and run['probes'][:, 0].tolist() == [1, 2, 3, 4, 5, 6]
    assert list(run['dt_reason']) == ['CFL'] * 6 and run['centreline'].shape[0] == 3


def test_noise():
    shapes = Recorder(6).shapes
    v, w = workloads.initial_noise(shapes, 1e-3, 5)
    assert v.shape == shapes['v'] and w.shape == shapes['w']
    assert np.std(v) == pytest.approx(1e-3, rel=0.2)
    v2, _ = workloads.initial_noise(shapes, 1e-3, 5)
    assert np.array_equal(v, v2)
    a = workloads.kick_noise(shapes, 0, 1)
    b = workloads.kick_noise(shapes, 0, 2)
    assert [x.shape for x in a] == [shapes[c] for c in 'uvw']
    assert not np.array_equal(a[0], b[0])


def test_stretched_first_cell():
    # a two-sided tanh grid: the wall cell shrinks as beta grows and tends to L / n as beta -> 0
    n = 64
    cells = [workloads.dx_wall_for_beta(n, b) for b in (1e-6, 0.5, 1.5, 2.0)]
    assert cells[0] == pytest.approx(1.0 / n, rel=1e-6)
    assert all(a > b for a, b in zip(cells, cells[1:]))
    assert workloads.C2['settings']['grid_dx_wall'] == pytest.approx(workloads.dx_wall_for_beta(64, 1.5))
    assert workloads.C2['settings']['grid_stretch'] == 1


def test_ensemble_cases():
    cases = workloads.ensemble_cases(count=400, seed=0)
    assert cases == workloads.ensemble_cases(count=400, seed=0)
    sizes = [c['settings']['nx'] for c in cases]
    assert set(sizes) == {24, 32, 48, 64}
    assert [c['settings']['grid_stretch'] for c in cases] == [k % 2 for k in range(400)]
    re = np.array([1.0 / c['settings']['nu'] for c in cases])
    assert re.min() >= 100.0 * (1 - 1e-9) and re.max() <= 2000.0 * (1 + 1e-9)
    assert np.mean(np.log(re) < math.log(math.sqrt(100.0 * 2000.0))) == pytest.approx(0.5, abs=0.06)
    assert all(c['precision'] == 'mixed' and c['seed'] == k for k, c in enumerate(cases))
