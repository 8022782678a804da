"""Host-side fault injection shared by the CPU (oracle) and GPU tests: each scenario makes the solver fail
through its inputs only (no device fault), checks the reference's error message, and that the solver stays
usable afterwards."""
import numpy as np
import pytest

from cases import base_settings, random_state


def infinite_velocity(make):
    """An infinite face velocity makes the CFL rate infinite: the step refuses to start (backend.cu:890)."""
    sim = make(base_settings(nx=8, ny=8, nz=6, adaptive_dt=1, dt_max=0.05))
    try:
        sim.initialize()
        state = random_state(sim.shapes, 3, True)
        for k, a in state.items():
            sim.set_field(k, a)
        before = {k: sim.field(k) for k in ('u', 'mx', 'phi')}
        bad = state['v'].copy()
        bad[2, 3, 4] = np.inf
        sim.set_field('v', bad)
        with pytest.raises(RuntimeError, match=r'^velocity is NaN/inf: the solution has blown up$'):
            sim.step()
        assert sim.report()['steps'] == 0
        # the failed step left the state alone; a finite velocity steps again
        sim.set_field('v', state['v'])
        assert np.array_equal(sim.field('u'), before['u']) and np.array_equal(sim.field('mx'), before['mx'])
        rep = sim.step()
        assert rep['steps'] == 1 and np.isfinite(sim.field('u')).all()
    finally:
        sim.close()


def nan_face_velocity(make):
    """One NaN face velocity: the CFL rate's max over the face pair drops it (fmaxf, backend.cu:469-471), so the
    failure surfaces in the pressure solve of the first stage."""
    sim = make(base_settings(nx=8, ny=8, nz=6, adaptive_dt=1, dt_max=0.05))
    try:
        sim.initialize()
        state = random_state(sim.shapes, 3, True)
        state['v'][2, 3, 4] = np.nan
        for k, a in state.items():
            sim.set_field(k, a)
        with pytest.raises(RuntimeError, match=r'^pressure solve: right-hand side is NaN/inf \(the run has blown up\)$'):
            sim.step()
        assert sim.report()['steps'] == 0
    finally:
        sim.close()


def nan_impulse(make):
    sim = make(base_settings(nx=8, ny=8, nz=6, adaptive_dt=0, dt_fixed=0.01))
    try:
        sim.initialize()
        state = random_state(sim.shapes, 4, True)
        state['my'][3, 3, 3] = np.inf
        for k, a in state.items():
            sim.set_field(k, a)
        with pytest.raises(RuntimeError, match=r'^pressure solve: right-hand side is NaN/inf \(the run has blown up\)$'):
            sim.step()
        assert sim.report()['steps'] == 0
    finally:
        sim.close()


def no_convergence(make):
    """fdm_max_passes = 0: the projection of the initial noise cannot reach FDM_RTOL."""
    sim = make(base_settings(nx=8, ny=8, nz=6, fdm_max_passes=0))
    try:
        v = 0.01 * np.ones(sim.shapes['v'])
        with pytest.raises(RuntimeError, match=r'^pressure solve: residual 1\.00e\+00 > FDM_RTOL after 0 passes$'):
            sim.initialize(v, None)
    finally:
        sim.close()


def tight_tolerance(make):
    """fdm_rtol below what one pass reaches with fdm_max_passes = 1."""
    sim = make(base_settings(nx=8, ny=8, nz=6, fdm_max_passes=1, fdm_rtol=1e-30))
    try:
        v = 0.01 * np.cos(np.arange(np.prod(sim.shapes['v']))).reshape(sim.shapes['v'])
        with pytest.raises(RuntimeError, match=r'^pressure solve: residual .* > FDM_RTOL after 1 passes$'):
            sim.initialize(v, None)
    finally:
        sim.close()


SCENARIOS = {'infinite_velocity': infinite_velocity, 'nan_face_velocity': nan_face_velocity, 'nan_impulse': nan_impulse, 'no_convergence': no_convergence,
             'tight_tolerance': tight_tolerance}
