"""Several cavities advanced together (concurrent streams) give each cavity exactly the result it has alone."""
import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('batched', [True, False])
def test_ensemble_matches_alone(batched):
    """Batched (one graph per group of same-size cavities) or per-cavity stepping: bit-identical to each cavity
    stepped alone."""
    cases = workloads.ensemble_cases(count=9, seed=3, sizes=(12, 16, 24), re_range=(100.0, 2000.0))
    for k, c in enumerate(cases):          # batches mixing uniform and stretched grids, in both forms
        c['precision'] = 'mixed' if k < 5 else 'fp64'
    ens = Ensemble(cases, batched=batched)
    try:
        assert not batched or len(ens.batches) < len(cases)
        ens.advance(5, chunk=3)
        together = [ens.fields(i) for i in range(len(cases))]
    finally:
        ens.close()
    for i in (0, 3, 5, 8):
        alone = Ensemble([cases[i]], batched=False)
        try:
            alone.advance(5, chunk=1)
            f = alone.fields(0)
        finally:
            alone.close()
        for k in f:
            assert np.array_equal(f[k], together[i][k]), (i, k)


def test_many_mixed_cavities_set_up_and_converge():
    """128 mixed-form cavities created back to back, each initialised (a projection from noise) and stepped:
    every pressure solve converges.  Creating many solvers keeps the default stream busy with set-up copies;
    each solver's first kernels must still see its uploaded operators."""
    cases = workloads.ensemble_cases(count=128, seed=5, sizes=(32, 48, 64))
    ens = Ensemble(cases)
    try:
        reports = ens.advance(2, chunk=2)
        for rep in reports:
            assert rep['steps'] == 2 and rep['phi_rel'] <= 1e-9
    finally:
        ens.close()
