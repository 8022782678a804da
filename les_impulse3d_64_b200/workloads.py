"""Seeded synthetic cavity workloads (the benchmark configurations, with their seeds and mappings).

No public dataset is involved: every input is generated here from `numpy.random.default_rng(seed)`.
Mappings onto the reference's settings (Config fields):

* Reynolds number -> nu = U L / Re.
* tanh clustering parameter beta -> grid_dx_wall = L/2 (1 + tanh(beta (2/n - 1)) / tanh(beta)), the first
  cell of the stretched grid with that beta; grid_max_aspect = 0 (no cap).
* "regularised lid" -> lid_shaped = 1 (the reference's (1 - s^18)^2 corner-smoothed lid); the polynomial
  lid 16 x^2(1-x)^2 z^2(1-z)^2 -> lid_shaped = 2 (an addition of this build).
* Gaussian initial noise of amplitude a -> a * U * standard_normal on v and w (u gets none), passed through
  solver_initialize like the reference's run script does with its uniform noise (main.py:130-137).
* kicks at given steps -> solver_kick with standard-normal noise on u, v, w, amplitude a, and
  KICK_CELLS // 2 = 10 smoothing passes (main.py:352-356).
"""
import math

import numpy as np

DEFAULTS = dict(length=1.0, u_lid=1.0, lz=1.0, lid_ramp_t=0.0, reinit_r=0.98, impulse_order=4,
                impulse_order4_ramp=1.0, phi_extrapolate=1, fdm_rtol=1e-9, fdm_max_passes=8, dt_lag=0,
                dt_max=4e-3, diffusion_limit=2.0, cfl_target=0.4, dt_fixed=2e-3, grid_max_aspect=0.0,
                grid_dx_wall=0.001)

PROBES4 = ((0.5, 0.5), (0.8, 0.8), (0.2, 0.2), (0.9, 0.1))
PROBES8 = PROBES4 + ((0.5, 0.9), (0.5, 0.1), (0.1, 0.5), (0.9, 0.5))


def dx_wall_for_beta(n, beta, length=1.0):
    """First cell of an n-cell two-sided tanh grid with clustering parameter beta."""
    return length / 2 * (1 + math.tanh(beta * (2.0 / n - 1)) / math.tanh(beta))


def settings(n, re, nz=None, beta=None, lid='regularised', adaptive=True, cfl=0.5, dt_fixed=2e-3, probes=PROBES8,
             **changes):
    s = dict(DEFAULTS)
    s.update(nx=n, ny=n, nz=nz or n, nu=1.0 / re, lid_shaped={'uniform': 0, 'regularised': 1, 'polynomial': 2}[lid],
             adaptive_dt=int(adaptive), cfl_target=cfl, dt_fixed=dt_fixed, probes=probes)
    if beta is None:
        s['grid_stretch'] = 0
    else:
        s['grid_stretch'] = 1
        s['grid_dx_wall'] = dx_wall_for_beta(n, beta)
    s.update(changes)
    return s


# C1: plain FP64, 32^3 uniform, Re 400, polynomial lid, fixed dt 2e-3, 500 steps, noise 1e-4, 4 probes
C1 = dict(name='c1_32cube_re400', settings=settings(32, 400.0, lid='polynomial', adaptive=False, dt_fixed=2e-3,
                                                    probes=PROBES4),
          steps=500, noise=1e-4, seed=0, kicks=(), stats_from=None, beta=None)
# C2: plain FP64 at the repo's size, 64^3 stretched (beta 1.5), Re 1000, regularised lid, CFL 0.5, 2000 steps,
# noise 1e-3, kicks 1e-2 at steps 500 and 1000, mid-span statistics from step 1000, 8 probes
C2 = dict(name='c2_64cube_re1000', settings=settings(64, 1000.0, beta=1.5, cfl=0.5), steps=2000, noise=1e-3, seed=0,
          kicks=((500, 1e-2), (1000, 1e-2)), stats_from=1000, beta=1.5)
# C3: mixed precision, 128^3 stretched (beta 2.0), Re 3200, CFL 0.5, 1000 steps, noise 1e-3
C3 = dict(name='c3_128cube_re3200', settings=settings(128, 3200.0, beta=2.0, cfl=0.5), steps=1000, noise=1e-3,
          seed=0, kicks=(), stats_from=None, precision='mixed', beta=2.0)

# 256^3 stretched (beta 2.0), Re 3200, mixed: the size at which the stencil kernels' HBM roofline is measured
C6 = dict(name='c6_256cube_re3200', settings=settings(256, 3200.0, beta=2.0, cfl=0.5), steps=100, noise=1e-3,
          seed=0, kicks=(), stats_from=None, precision='mixed', beta=2.0)

WORKLOADS = {w['name']: w for w in (C1, C2, C3, C6)}


def initial_noise(shapes, amplitude, seed, u_lid=1.0):
    """Seeded Gaussian noise on v and w (u has none)."""
    rng = np.random.default_rng(seed)
    v = amplitude * u_lid * rng.standard_normal(shapes['v'])
    w = amplitude * u_lid * rng.standard_normal(shapes['w'])
    return v, w


def kick_noise(shapes, seed, number):
    """Standard-normal kick noise on u, v, w for kick `number` (1-based)."""
    rng = np.random.default_rng(seed + 1000 + number - 1)
    return [rng.standard_normal(shapes[c]) for c in 'uvw']


def run_protocol(sim, workload, steps=None, snapshots=(), on_snapshot=None):
    """Drive a solver through a workload's run, step by step, in the order of the reference's run script
    (main.py:342-363): one step, then the probes, then a kick if one is due, then the statistics.

    Kicks and the statistics window are indexed by step number (the configs give them so; main.py keys them
    on time): kick (n, amp) follows step n, and every step n > stats_from adds the mid-span field with weight
    dt.  `sim` is any binding of the solver ABI (the B200 build, the oracle, the reference).
    `on_snapshot(n, sim)` is called after step n for every n in `snapshots`.

    Returns per-step arrays: dt, time, dt_reason, phi_passes, probes (steps x 2 n_probes, float32), the KE
    before and after each kick, and the centreline samples of the statistics steps."""
    steps = workload['steps'] if steps is None else steps
    kicks = dict(workload.get('kicks', ()))
    stats_from = workload.get('stats_from')
    out = dict(dt=[], time=[], dt_reason=[], phi_passes=[], probes=[], kick_ke=[], centreline=[])
    for n in range(1, steps + 1):
        rep = sim.step()
        out['dt'].append(rep['dt'])
        out['time'].append(rep['time'])
        out['dt_reason'].append(rep['dt_reason'])
        out['phi_passes'].append(rep['phi_passes'])
        out['probes'].append(sim.probes())
        if n in kicks:
            before = sim.diagnostics()['kinetic_energy']
            sim.kick(kick_noise(sim.shapes, workload['seed'], sorted(kicks).index(n) + 1), kicks[n], KICK_PASSES)
            out['kick_ke'].append((before, sim.diagnostics()['kinetic_energy']))
        if stats_from is not None and n > stats_from:
            out['centreline'].append(sim.add_statistics(rep['dt']))
        if n in snapshots and on_snapshot is not None:
            on_snapshot(n, sim)
    res = {k: np.asarray(v) for k, v in out.items()}
    res['dt_reason'] = np.asarray(out['dt_reason'], dtype=object)
    return res


# smoothing passes of a kick: KICK_CELLS // 2 with the run script's 20-cell eddies (main.py:54, 356)
KICK_PASSES = 10


def ensemble_cases(count=256, seed=0, sizes=(24, 32, 48, 64), re_range=(100.0, 2000.0), noise=1e-3):
    """C4: `count` cavities, sizes drawn uniformly from `sizes`, half uniform and half stretched (beta 1.5),
    Re log-uniform in `re_range`, independent noise seeds; mixed form, CFL 0.5."""
    rng = np.random.default_rng(seed)
    cases = []
    for k in range(count):
        n = int(rng.choice(sizes))
        re = float(np.exp(rng.uniform(np.log(re_range[0]), np.log(re_range[1]))))
        beta = 1.5 if k % 2 else None
        cases.append(dict(name=f'cavity{k:03d}', settings=settings(n, re, beta=beta, cfl=0.5), noise=noise, seed=k,
                          precision='mixed'))
    return cases


C4 = dict(name='c4_ensemble256', steps=1000, cases=ensemble_cases)
