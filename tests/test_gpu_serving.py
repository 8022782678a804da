"""The serving loop: every request of a Poisson stream completes at its end time, and a request served in the
batched mix ends in exactly the state of the same cavity stepped alone for the same number of steps."""
import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Cavity
from les_impulse3d_64_b200.serve import Server, serving_requests, summary

pytestmark = pytest.mark.gpu

SIZES = ((16, 16, 16), (24, 24, 24), (16, 16, 24))


@pytest.mark.parametrize('batched', [True, False])
def test_serving_matches_alone(batched):
    reqs = serving_requests(10, rate=200.0, seed=7, sizes=SIZES, t_end=0.03)
    finals = {}

    def keep(req, cav):
        finals[req.id] = {k: cav.field(k) for k in ('u', 'v', 'w', 'phi')}

    results = Server(budget_bytes=2e9, precision='mixed', chunk=4, batched=batched).run(reqs, on_finish=keep)
    assert [r.id for r in results] == list(range(10))
    for r in results:
        assert r.time >= 0.03 and r.steps >= 1 and r.finished >= r.arrival
    s = summary(results)
    assert s['p99_s'] >= s['p50_s'] > 0
    for k in (0, 4, 9):
        req, res = reqs[k], results[k]
        cav = Cavity(req.settings, precision='mixed')
        try:
            cav.initialize(*workloads.initial_noise(cav.shapes, req.noise, req.seed))
            cav.step_async(res.steps)
            rep = cav.sync()
            assert rep['steps'] == res.steps and rep['time'] == res.time
            for name, a in finals[k].items():
                assert np.array_equal(a, cav.field(name)), (k, name)
        finally:
            cav.close()


def test_admission_respects_the_budget():
    """A budget that holds one cavity at a time serves the stream one by one, in arrival order."""
    reqs = serving_requests(4, rate=1000.0, seed=3, sizes=((16, 16, 16),), t_end=0.01)
    from les_impulse3d_64_b200.api import estimate_bytes
    one = estimate_bytes(reqs[0].settings, 'mixed')
    results = Server(budget_bytes=1.5 * one, precision='mixed', chunk=2).run(reqs)
    for a, b in zip(results, results[1:]):
        assert b.admitted >= a.finished - 1e-3
