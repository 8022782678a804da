"""Checkpoints keep everything that decides the following steps: continuing from a loaded checkpoint is
bit-identical to never having stopped, from a host or a device copy; restarting through the fields alone (the
reference's path, which drops the potential history and the dt lag) is not."""
import numpy as np
import pytest

from les_impulse3d_64_b200 import workloads
from les_impulse3d_64_b200.api import Cavity

pytestmark = pytest.mark.gpu

FIELDS = ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')


def state(cav):
    return {k: cav.field(k) for k in FIELDS}


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_checkpoint_continues_bit_identically(precision):
    s = workloads.settings(24, 1000.0, beta=1.5, cfl=0.5, dt_lag=1)
    cav = Cavity(s, precision=precision)
    try:
        cav.initialize(*workloads.initial_noise(cav.shapes, 1e-3, 2))
        for _ in range(6):
            cav.step()
        host = cav.checkpoint()
        import torch
        dev = torch.empty(cav.checkpoint_bytes(), dtype=torch.uint8, device='cuda')
        cav.checkpoint(dev.data_ptr())
        for _ in range(5):
            r_ref = cav.step()
        ref = state(cav)
        for ck in (host, dev.data_ptr()):
            cav.restore(ck)
            assert cav.report()['steps'] == 6
            for _ in range(5):
                r = cav.step()
            assert r == r_ref
            for k, a in state(cav).items():
                assert np.array_equal(a, ref[k]), k
        # the reference's restart: fields and clock only (history and dt lag cleared)
        cav.restore(host)
        saved = state(cav)
        rep = cav.report()
        fresh = Cavity(s, precision=precision)
        try:
            fresh.initialize()
            for k in ('u', 'v', 'w', 'mx', 'my', 'mz'):
                fresh.set_field(k, saved[k])
            fresh.set_field('phi', saved['phi'])
            fresh.set_clock(rep['time'], rep['steps'], rep['dt'])
            for _ in range(5):
                fresh.step()
            assert any(not np.array_equal(fresh.field(k), ref[k]) for k in ('u', 'v', 'w', 'phi'))
        finally:
            fresh.close()
    finally:
        cav.close()


def test_checkpoint_rejects_another_grid():
    a = Cavity(workloads.settings(16, 500.0), precision='fp64')
    b = Cavity(workloads.settings(24, 500.0), precision='fp64')
    try:
        a.initialize()
        ck = a.checkpoint()
        with pytest.raises(RuntimeError, match='grid size or precision'):
            b.restore(ck)
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize('change', [dict(beta=2.0), dict(re=2000.0), dict(lid='uniform'), dict(impulse_order=2)])
def test_checkpoint_rejects_other_settings(change):
    """Same grid size and precision, but another stretching, Re, lid or impulse order: the saved dt lag,
    CFL state and potential history belong to another run, so the load is refused."""
    base = dict(beta=1.5, re=1000.0, lid='regularised', impulse_order=4)
    other = dict(base, **change)
    a = Cavity(workloads.settings(16, base['re'], beta=base['beta'], lid=base['lid'],
                                  impulse_order=base['impulse_order']), precision='fp64')
    b = Cavity(workloads.settings(16, other['re'], beta=other['beta'], lid=other['lid'],
                                  impulse_order=other['impulse_order']), precision='fp64')
    try:
        a.initialize()
        ck = a.checkpoint()
        with pytest.raises(RuntimeError, match='other settings'):
            b.restore(ck)
        b.initialize()
        b.restore(b.checkpoint())      # its own checkpoint still loads
    finally:
        a.close()
        b.close()
