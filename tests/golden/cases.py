"""Seeded parity cases for the cavity solver ABI, shared by the fixture generator and the tests.

A case is a settings dict plus a short script of ABI calls (create, set fields or initialize, steps,
kick, getters).  `run_case` plays the script through any build of the ABI (the reference's backend.cu
built under oracle/_ref, the CPU oracle, or the B200 build) and returns every output as a flat dict of
NumPy arrays, so outputs of different builds compare key by key.

Inputs come from a splitmix64 hash of (seed, index): integer arithmetic only, so the same inputs are
produced on any machine and NumPy version without storing them.
"""
import numpy as np

MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def seeded_uniform(shape, seed):
    """Uniform values in [-1, 1) from splitmix64(seed * golden + index)."""
    n = int(np.prod(shape))
    with np.errstate(over='ignore'):
        x = np.arange(n, dtype=np.uint64) + np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return ((x >> np.uint64(11)).astype(np.float64) * 2.0 ** -53 * 2.0 - 1.0).reshape(shape)


def base_settings(**changes):
    """Settings of the reference's run script (main.py:19-70) mapped to Config names, then `changes`."""
    s = dict(nx=12, ny=12, nz=8, lid_shaped=1, impulse_order=4, adaptive_dt=0, dt_lag=0, phi_extrapolate=1,
             fdm_max_passes=8, grid_stretch=0, length=1.0, u_lid=1.0, nu=1.0 / 400.0, lz=1.0, lid_ramp_t=0.0,
             reinit_r=0.98, impulse_order4_ramp=1.0, grid_dx_wall=0.001, grid_max_aspect=0.0, dt_fixed=0.02,
             dt_max=0.004, cfl_target=0.4, diffusion_limit=2.0, fdm_rtol=1e-9,
             probes=((0.5, 0.5), (0.8, 0.8), (0.2, 0.2), (0.9, 0.1)))
    s.update(changes)
    return s


def zero_walls(name, a):
    """Zero the faces of field `name` that lie on a wall (arrays are [z, y, x])."""
    a = a.copy()
    if name in ('u', 'mx'):
        a[..., 0] = a[..., -1] = 0
    elif name in ('v', 'my'):
        a[:, 0, :] = a[:, -1, :] = 0
    elif name in ('w', 'mz'):
        a[0] = a[-1] = 0
    return a


def random_state(shapes, seed, walls=True, phi_scale=0.1, gauge=0.3):
    """O(1) random velocity, impulse = velocity + gauge*noise, small random potential."""
    out = {}
    for k, (c, mc) in enumerate((('u', 'mx'), ('v', 'my'), ('w', 'mz'))):
        u = seeded_uniform(shapes[c], seed + 10 * k)
        m = u + gauge * seeded_uniform(shapes[c], seed + 10 * k + 5)
        out[c] = zero_walls(c, u) if walls else u
        out[mc] = zero_walls(mc, m) if walls else m
    out['phi'] = phi_scale * seeded_uniform(shapes['phi'], seed + 99)
    return out


CASES = {
    # one step from O(1) random fields: every term of the right-hand side matters
    'one_step_o4_uniform': dict(
        settings=base_settings(nx=12, ny=12, nz=8, dt_fixed=0.02, nu=0.01),
        script=[('set_state', 1, True), ('steps', 1), ('outputs',)]),
    # stretched grid, odd nz (one mid-span layer), 4th-order ramp over 2 cells, uniform lid, random wall faces,
    # adaptive CFL dt; the second step uses the warm start from the first
    'two_steps_o4_stretched': dict(
        settings=base_settings(nx=12, ny=12, nz=9, grid_stretch=1, grid_dx_wall=0.03, lid_shaped=0,
                               impulse_order4_ramp=2.0, adaptive_dt=1, dt_max=1.0, nu=0.002),
        script=[('set_state', 2, False), ('steps', 2), ('outputs',)]),
    # 2nd order, aspect-capped stretching, lagged dt with growth cap, lid ramp, faster lid
    'three_steps_o2_lag': dict(
        settings=base_settings(nx=8, ny=8, nz=6, grid_stretch=1, grid_dx_wall=0.02, grid_max_aspect=3.0,
                               impulse_order=2, adaptive_dt=1, dt_lag=1, dt_max=0.05, nu=0.02, lid_ramp_t=0.1,
                               u_lid=2.0),
        script=[('set_state', 3, True), ('steps', 3), ('outputs',)]),
    # initial noise -> projection, a short run with probes, statistics and a kick
    'run_with_kick': dict(
        settings=base_settings(nx=16, ny=16, nz=6, grid_stretch=1, grid_dx_wall=0.01, grid_max_aspect=4.0,
                               adaptive_dt=1, dt_lag=1, dt_max=0.01, nu=1.0 / 1000.0, lid_ramp_t=0.05),
        script=[('initialize', 4, 0.01), ('steps', 3), ('kick', 5, 0.02, 2), ('steps', 3),
                ('statistics_steps', 3), ('outputs',)]),
}


def run_case(make_solver, case):
    """Play `case` through a solver made by `make_solver(settings)`; returns {key: ndarray}."""
    sim = make_solver(case['settings'])
    out = {}
    nstep = 0

    def record_report(tag, rep):
        out[f'{tag}.steps'] = np.array(rep['steps'])
        out[f'{tag}.time'] = np.array(rep['time'])
        out[f'{tag}.dt'] = np.array(rep['dt'])
        out[f'{tag}.cfl'] = np.array(rep['cfl'])
        out[f'{tag}.phi_rel'] = np.array(rep['phi_rel'])
        out[f'{tag}.dt_reason'] = np.array(['fixed_DT', 'DT_MAX', 'CFL', 'viscous'].index(rep['dt_reason']))
        out[f'{tag}.phi_passes'] = np.array(rep['phi_passes'])

    try:
        for op in case['script']:
            kind = op[0]
            if kind == 'set_state':
                _, seed, walls = op
                sim.initialize()
                for name, a in random_state(sim.shapes, seed, walls).items():
                    sim.set_field(name, a)
            elif kind == 'initialize':
                _, seed, amp = op
                v = amp * seeded_uniform(sim.shapes['v'], seed)
                w = amp * seeded_uniform(sim.shapes['w'], seed + 1)
                sim.initialize(v, w)
                out['init.u'] = sim.field('u')
                out['init.v'] = sim.field('v')
                out['init.w'] = sim.field('w')
                out['init.phi'] = sim.field('phi')
            elif kind in ('steps', 'statistics_steps'):
                for _ in range(op[1]):
                    old_t = sim.report()['time']
                    rep = sim.step()
                    nstep += 1
                    record_report(f'step{nstep}', rep)
                    out[f'step{nstep}.probes'] = sim.probes()
                    if kind == 'statistics_steps':
                        out[f'step{nstep}.centreline'] = sim.add_statistics(rep['time'] - old_t)
            elif kind == 'kick':
                _, seed, amp, passes = op
                noise = [seeded_uniform(sim.shapes[c], seed + k) for k, c in enumerate('uvw')]
                sim.kick(noise, amp, passes)
                out['kick.u'] = sim.field('u')
                out['kick.mx'] = sim.field('mx')
            elif kind == 'outputs':
                for name in ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi'):
                    out[f'final.{name}'] = sim.field(name)
                for key, val in sim.diagnostics().items():
                    out[f'diag.{key}'] = np.array(val)
                out['final.probes'] = sim.probes()
                out['final.midplane'] = sim.midplane()
                q, colour = sim.q_volume(True)
                out['final.q'], out['final.colour_w'] = q, colour
                out['final.colour_speed'] = sim.q_volume(False)[1]
                out['final.centreline'] = sim.add_statistics(0.5)
                for key, val in sim.statistics().items():
                    out[f'stats.{key}'] = val
                for axis in 'xyz':
                    out[f'grid.{axis}.faces'], out[f'grid.{axis}.centres'] = sim.grid[axis]
        record_report('final', sim.report())
    finally:
        sim.close()
    return out
