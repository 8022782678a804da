"""The serving loop: every request of a Poisson stream completes at its end time, and a request served in the
batched mix ends in the state of the same cavity stepped alone for the same number of steps: bit for bit when
served one graph per cavity; to rounding (1e-6 relative in the FP32 fields) in slot batches, whose column
kernels split a cavity's z-range into fewer chunks than a cavity alone, so that its sums (norms, the potential's
mean) add the same values in another grouping.  Slot batches take cavities in and out without a rebuild."""
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
            assert rep['steps'] == res.steps and abs(rep['time'] - res.time) <= 1e-9 * res.time
            for name, a in finals[k].items():
                b = cav.field(name)
                if batched:
                    err = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
                    assert err <= 1e-6, (k, name, err)
                else:
                    assert np.array_equal(a, b), (k, name)
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


@pytest.mark.parametrize('precision, fdm', [('fp64', 'dmma'), ('mixed', 'dmma'), ('mixed', 'tc')])
def test_slot_batch_takes_members_in_and_out(precision, fdm, monkeypatch):
    """A batch of three slots: A starts alone in it; B, stepped once on its own (the other state parity), joins;
    A leaves, the batch steps with its first slot empty (the first block of every launch then belongs to an
    empty slot, which must still end each refinement loop), and C joins that slot.  Each cavity's state after its
    steps in the batch equals that of a twin stepped the same number of steps alone, to rounding.  Both transform
    paths: FP64 DMMA, and the mixed form's tensor-core transforms (CAVITY_FDM=tc)."""
    from les_impulse3d_64_b200.api import Batch
    monkeypatch.setenv('CAVITY_FDM', fdm)
    s = workloads.settings(24, 800.0, beta=1.5, cfl=0.5)
    tol = 1e-12 if precision == 'fp64' else 1e-6

    def make(seed):
        c = Cavity(s, precision=precision)
        c.initialize(*workloads.initial_noise(c.shapes, 1e-3, seed))
        return c

    a, b, c = make(1), make(2), make(3)
    twins = {k: make(seed) for k, seed in (('a', 1), ('b', 2), ('c', 3))}
    steps = {'a': 0, 'b': 0, 'c': 0}
    batch = Batch([a], capacity=3)
    try:
        assert batch.free_slots() == [1, 2]
        batch.step_async(2); batch.sync(); steps['a'] += 2
        b.step(); steps['b'] += 1
        batch.set_member(1, b)
        batch.step_async(3); reps = batch.sync(); steps['a'] += 3; steps['b'] += 3
        assert reps[2] is None and reps[0]['steps'] == 5 and reps[1]['steps'] == 4
        batch.set_member(0, None)
        batch.step_async(2); reps = batch.sync(); steps['b'] += 2
        assert reps[0] is None and reps[1]['steps'] == 6
        batch.set_member(0, c)
        batch.step_async(2); batch.sync(); steps['b'] += 2; steps['c'] += 2
        for name, cav in (('a', a), ('b', b), ('c', c)):
            twin = twins[name]
            twin.step_async(steps[name])
            assert twin.sync()['steps'] == cav.report()['steps'] == steps[name]
            for k in ('u', 'v', 'w', 'phi'):
                x, y = cav.field(k), twin.field(k)
                err = float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-30))
                assert err <= tol, (name, k, err)
        with pytest.raises(RuntimeError, match='already in another slot'):
            batch.set_member(2, b)
        other = Cavity(workloads.settings(16, 800.0), precision=precision)
        try:
            with pytest.raises(RuntimeError, match='grid size differs'):
                batch.set_member(2, other)
        finally:
            other.close()
    finally:
        batch.close()
        for cav in [a, b, c, *twins.values()]:
            cav.close()
