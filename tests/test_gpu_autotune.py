"""The autotuner (cavity_autotune): it leaves the cavity's state as it was, picks one of its candidates, and the
steps it then runs equal an untuned cavity's: bit for bit when the sweep kernel is fixed (CAVITY_SWEEP=tile: the
other choices only change launch shapes), to rounding when the tuner may also pick the march sweep (1e-12 in
FP64, 1e-6 in the FP32 fields of the mixed form); the choice is written to CAVITY_TUNE_FILE."""
import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Cavity

pytestmark = pytest.mark.gpu
FIELDS = ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')


@pytest.mark.parametrize('sweep', ['tile', None])
@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_autotune_keeps_state_and_results(precision, sweep, tmp_path, monkeypatch):
    tune_file = tmp_path / 'tune.txt'
    monkeypatch.setenv('CAVITY_TUNE_FILE', str(tune_file))
    if sweep:
        monkeypatch.setenv('CAVITY_SWEEP', sweep)
    s = workloads.settings(48, 1000.0, nz=40, beta=1.5, cfl=0.5)
    a, b = Cavity(s, precision=precision), Cavity(s, precision=precision)
    try:
        for cav in (a, b):
            cav.initialize(*workloads.initial_noise(cav.shapes, 1e-3, 4))
            for _ in range(3):
                cav.step()
        before = {k: a.field(k) for k in FIELDS}
        rep = a.report()
        chunks, tile, fused, ms = a.autotune(steps=3)
        # chunks: 0 with the default tile sweep (nothing to choose), 1 .. nz/4 with the march sweep; FP64
        # transforms below 128^3 in both forms: the size rule (when no candidate beat it), 64 x 64 or 32 x 32 tiles,
        # the latter possibly in one launch, or the three paired launches
        assert ms > 0 and 0 <= chunks <= 40 // 4 and (tile, fused) in ((0, -1), (64, 0), (32, 0), (32, 1), (0, 2))
        assert a.report() == rep
        for k in FIELDS:
            assert np.array_equal(a.field(k), before[k]), k
        tol = 0.0 if sweep else (1e-12 if precision == 'fp64' else 1e-6)
        for _ in range(4):
            ra, rb = a.step(), b.step()
            assert ra['steps'] == rb['steps'] and ra['phi_passes'] == rb['phi_passes']
            assert abs(ra['time'] - rb['time']) <= tol * rb['time']
        for k in FIELDS:
            x, y = a.field(k), b.field(k)
            if sweep:
                assert np.array_equal(x, y), k
            else:
                assert float(np.abs(x - y).max()) <= tol * max(float(np.abs(y).max()), 1e-30), k
    finally:
        a.close()
        b.close()
    line = tune_file.read_text().strip().splitlines()[-1]
    assert line.startswith('48 48 40 1 ') and line.split('|')[1].split()[:3] == [str(chunks), str(tile), str(fused)]
