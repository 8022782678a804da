"""Queued steps with their per-step outputs on the device give the same probe values and statistics sums as
the reference's per-step calls (solver_step, solver_probes, solver_add_statistics with the step's dt)."""
import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Cavity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_queued_outputs_match_per_step_calls(precision):
    s = workloads.settings(24, 1000.0, beta=1.5, cfl=0.5)
    steps = 12
    a = Cavity(s, precision=precision)
    b = Cavity(s, precision=precision)
    try:
        for c in (a, b):
            c.initialize(*workloads.initial_noise(c.shapes, 1e-3, 4))
        probes_a = []
        for _ in range(steps):
            rep = a.step()
            probes_a.append(a.probes())
            a.add_statistics(rep['dt'])
        b.step_outputs_async(5, statistics=True)
        b.step_outputs_async(steps - 5, statistics=True)
        rep_b, probes_b = b.sync_outputs()
        assert rep_b == a.report()
        assert probes_b.shape == (steps, 2 * a.config.n_probes)
        assert np.array_equal(np.array(probes_a), probes_b)
        assert np.array_equal(a.statistics(), b.statistics())
    finally:
        a.close()
        b.close()
