"""Several cavities advanced together (concurrent streams) give each cavity exactly the result it has alone."""
import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('batched', [True, False])
def test_ensemble_matches_alone(batched):
    """Batched (one graph for the cavities of each precision form, whatever their sizes) or per-cavity stepping:
    bit-identical to each cavity stepped alone."""
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


@pytest.mark.parametrize('group', ['precision', 'size'])
def test_large_mixed_size_batch_matches_alone(group):
    """48 cavities of three sizes in one batch: few z-chunks per cavity in the column kernels, where a cavity alone
    fills the device with its own.  Its reductions (norms, the mean of the potential) then add the same values in another grouping, so
    each cavity ends equal to itself alone to rounding: 1e-6 relative in the FP32 fields of the mixed form."""
    cases = workloads.ensemble_cases(count=48, seed=7, sizes=(16, 24, 32), re_range=(100.0, 2000.0))
    ens = Ensemble(cases, group=group)
    try:
        assert len(ens.batches) == (1 if group == 'precision' else 3)
        ens.advance(4, chunk=2)
        together = [ens.fields(i) for i in range(len(cases))]
    finally:
        ens.close()
    for i in (0, 17, 47):
        alone = Ensemble([cases[i]], batched=False)
        try:
            alone.advance(4, chunk=1)
            f = alone.fields(0)
        finally:
            alone.close()
        for k in f:
            err = float(np.abs(f[k] - together[i][k]).max() / max(np.abs(f[k]).max(), 1e-30))
            assert err <= 1e-6, (i, k, err)


BATCH_RUN = r'''
import sys
import numpy as np
sys.path[:0] = [{root!r}]
from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.ensemble import Ensemble
cases = workloads.ensemble_cases(count=6, seed=13, sizes=(24, 40, 64), re_range=(100.0, 2000.0))
for k, c in enumerate(cases):
    c['precision'] = 'mixed' if k % 2 else 'fp64'
ens = Ensemble(cases, group='precision')
ens.advance(3, chunk=3)
np.savez({path!r}, **{{f'{{i}}_{{k}}': v for i in range(len(cases)) for k, v in ens.fields(i).items()}})
ens.close()
print('ok')
'''


def test_batch_pass_tiles_per_cta(tmp_path):
    """A batch of cavities of three sizes in both forms whose paired FP64 passes take one tile per CTA, or four
    (CAVITY_PAIR_PER, read once per process: a child process each): the same fields bit for bit."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    out = {}
    for per in ('1', '4'):
        path = str(tmp_path / f'per{per}.npz')
        env = dict(os.environ, CAVITY_PAIR_PER=per)
        res = subprocess.run([sys.executable, '-c', BATCH_RUN.format(root=str(root), path=path)], env=env,
                             capture_output=True, text=True, timeout=600)
        assert res.returncode == 0 and 'ok' in res.stdout, res.stdout + res.stderr
        out[per] = np.load(path)
    for k in out['1'].files:
        assert np.array_equal(out['1'][k], out['4'][k]), k


@pytest.mark.parametrize('form', ['0', '2'])
def test_batch_pass_forms_agree(form):
    """A batch of cavities of three sizes with its FP64 passes as six launches (CAVITY_FDM_FUSED=0, the large and
    the small transform tile) or as three paired launches (=2, the default when no axis exceeds 64 cells): the
    same fields bit for bit as the default batch."""
    import os
    cases = workloads.ensemble_cases(count=12, seed=11, sizes=(16, 24, 40), re_range=(100.0, 2000.0))
    for k, c in enumerate(cases):
        c['precision'] = 'mixed' if k % 2 else 'fp64'

    def run(env):
        old = os.environ.pop('CAVITY_FDM_FUSED', None)
        os.environ.update(env)
        try:
            ens = Ensemble(cases, group='precision')
        finally:
            os.environ.pop('CAVITY_FDM_FUSED', None)
            if old is not None:
                os.environ['CAVITY_FDM_FUSED'] = old
        try:
            ens.advance(3, chunk=3)
            return [ens.fields(i) for i in range(len(cases))]
        finally:
            ens.close()

    ref = run({})
    got = run({'CAVITY_FDM_FUSED': form})
    for i in range(len(cases)):
        for k in ref[i]:
            assert np.array_equal(ref[i][k], got[i][k]), (i, k)


def test_batch_with_an_axis_beyond_the_paired_pass():
    """A batch whose members include one with 80 cells per axis runs every member's FP64 passes as six launches
    (the paired pass takes at most 64 per axis, and a batch's members share their launches); each member ends equal
    to itself alone, which runs the paired pass when it fits, to rounding."""
    cases = workloads.ensemble_cases(count=3, seed=17, sizes=(24, 80), re_range=(100.0, 2000.0))
    cases[0]['settings'] = workloads.settings(80, 500.0, beta=1.5, cfl=0.5)
    for c in cases:
        c['precision'] = 'fp64'
    ens = Ensemble(cases, group='precision')
    try:
        assert len(ens.batches) == 1
        ens.advance(3, chunk=3)
        together = [ens.fields(i) for i in range(len(cases))]
    finally:
        ens.close()
    for i in range(len(cases)):
        alone = Ensemble([cases[i]], batched=False)
        try:
            alone.advance(3, chunk=1)
            f = alone.fields(0)
        finally:
            alone.close()
        for k in f:
            err = float(np.abs(f[k] - together[i][k]).max() / max(np.abs(f[k]).max(), 1e-30))
            assert err <= 1e-10, (i, k, err)


def test_batch_part_times_are_ordinary_steps():
    """cavity_batch_part_times times a batch's parts (sweep, start with the guess residual, first pass, finish)
    through an instrumented copy of its graph: every part takes time, the steps it takes leave the cavities bit for
    bit where plain batched steps leave them, and the plain graph steps on correctly afterwards."""
    cases = workloads.ensemble_cases(count=4, seed=19, sizes=(16, 24), re_range=(100.0, 2000.0))
    ens_a, ens_b = Ensemble(cases, group='precision'), Ensemble(cases, group='precision')
    try:
        assert len(ens_a.batches) == 1
        times = ens_a.batches[0].part_times(3)
        assert set(times) == {'sweep', 'start', 'first_pass', 'finish'} and all(t > 0 for t in times.values())
        ens_b.advance(3, chunk=3)
        for e in (ens_a, ens_b):
            e.advance(2, chunk=2)
        for i in range(len(cases)):
            fa, fb = ens_a.fields(i), ens_b.fields(i)
            for k in fa:
                assert np.array_equal(fa[k], fb[k]), (i, k)
    finally:
        ens_a.close()
        ens_b.close()
