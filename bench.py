#!/usr/bin/env python
"""Benchmark of the cavity time step on B200: cell-updates/s per SSP-RK3 step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2_64cube_re1000]

A step is one full time step of the solver (3 RK stages, each with its pressure projection) of the seeded
synthetic workload; the default workload is the plain FP64 form on the 64^3 tanh-stretched cavity (Re 1000,
regularised lid, adaptive dt at CFL 0.5, noise 1e-3).  `value` is device time (CUDA events on the solver's
stream around each step, the L2 cache flushed by a 256 MiB write before each timed step), max over ranks;
`e2e` is the same metric through the reference-facing C ABI (`solver_*`) from host buffers, wall clock,
host<->device copies included.  With N > 1 (torchrun) every rank advances its own replica cavity (the step has
no collective); `value` counts all ranks' cells.

--impl reference times the reference's algorithm on the host cores: the OpenMP FP64 restatement under oracle/
(the reference ships no CPU path), on the same workload, and adds the reference's own backend.cu (built from
its source under oracle/_ref) on the GPU where that build is present.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=50)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', choices=('ours', 'reference'), default='ours')
    ap.add_argument('--workload', default='c2_64cube_re1000')
    ap.add_argument('--precision', choices=('fp64', 'mixed'), default=None)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-batched', action='store_true',
                    help='skip the batched mixed-form sub-measurements of the default line')
    ap.add_argument('--no-serving', action='store_true', help='skip the served-stream sub-measurement of the default line')
    ap.add_argument('--serving-requests', type=int, default=200, help='requests of the default line\'s served stream')
    ap.add_argument('--serving-t-end', type=float, default=0.2, help='end time of each request of that stream')
    ap.add_argument('--count', type=int, default=256, help='cavities of the c4_ensemble workload')
    ap.add_argument('--chunk', type=int, default=8, help='steps queued per cavity between waits (ensemble)')
    ap.add_argument('--requests', type=int, default=64, help='requests of the c5_serving stream')
    ap.add_argument('--rate', type=float, default=50.0, help='Poisson arrival rate (1/s) of c5_serving')
    ap.add_argument('--t-end', type=float, default=0.1, help='simulated end time of each c5_serving request')
    return ap.parse_args()


# ------------------------------------------------------------------------------------------ ranks
class Ranks:
    """torch.distributed plumbing for N replicas (barrier and max over ranks); identity at N = 1.

    One process per GPU: with torchrun, LOCAL_RANK's GPU becomes this process's device 0 before CUDA starts.
    `backend` is 'nccl' on GPUs; 'gloo' runs the same plumbing on CPU (tests).
    """

    def __init__(self, backend='nccl'):
        self.world = int(os.environ.get('WORLD_SIZE', '1'))
        self.rank = int(os.environ.get('RANK', '0'))
        self.local = int(os.environ.get('LOCAL_RANK', '0'))
        self.backend = backend
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            kw = {}
            if backend == 'nccl':
                os.environ['CUDA_VISIBLE_DEVICES'] = str(self.local)
                torch.cuda.set_device(0)
                kw['device_id'] = torch.device('cuda', 0)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
            self.dist, self.torch = dist, torch

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x):
        if self.world == 1:
            return x
        t = self.torch.tensor([float(x)], device='cuda' if self.backend == 'nccl' else 'cpu')
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# ------------------------------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled through NVML every 2 ms during the timed region."""
    REASONS = {0x4: 'sw_power_cap', 0x8: 'hw_slowdown', 0x20: 'sw_thermal_slowdown', 0x40: 'hw_thermal_slowdown',
               0x80: 'hw_power_brake_slowdown'}

    def __init__(self, index=0, period=0.002):
        self.index, self.period = index, period
        self.samples, self.max_mhz, self.reasons = [], None, set()
        self._stop = threading.Event()
        self.nvml = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception:
            self.nvml = None
        return self

    def _run(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                for bit, name in self.REASONS.items():
                    if bits & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __exit__(self, *exc):
        if self.nvml:
            self._stop.set()
            self.thread.join(timeout=2)

    def summary(self):
        return {'sm_mhz': statistics.median(self.samples) if self.samples else None, 'sm_max_mhz': self.max_mhz,
                'reasons': sorted(self.reasons), 'samples': len(self.samples)}


# ------------------------------------------------------------------------------------------ helpers
def measured_peaks():
    p = ROOT / 'MEASURED_PEAKS.json'
    if p.is_file():
        d = json.loads(p.read_text())
        return float(d['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


def profile_traffic(workload):
    """DRAM bytes per momentum-sweep launch from the committed ncu summary (None if absent)."""
    p = ROOT / 'profiles' / f'momentum_sweep_{workload}.md'
    if not p.is_file():
        return None
    for line in p.read_text().splitlines():
        if line.startswith('traffic_bytes_per_launch:'):
            return float(line.split(':', 1)[1])
    return None


def sweep_kernel_name(precision):
    """The momentum-sweep kernel the library runs: the shared-memory tile kernel in the FP64 form and its packed
    two-cells-per-thread variant in the mixed form, unless CAVITY_SWEEP selects another."""
    kind = os.environ.get('CAVITY_SWEEP', '')
    if kind == 'face':
        return 'momentum_kernel'
    if kind == 'march':
        return 'sweep_march_kernel'
    if kind == 'tile' or precision == 'fp64':
        return 'sweep_tile_kernel'
    return 'sweep_pair_kernel'


def momentum_bytes(settings, field_bytes):
    """Algorithmic HBM bytes of one momentum-sweep launch: per component 4 face arrays (read u, m and the RK
    base or write it, write the new impulse), each element once."""
    nx, ny, nz = settings['nx'], settings['ny'], settings['nz']
    faces = (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
    return 4 * faces * field_bytes


def cell_kernel_bytes(settings, field_bytes):
    """Algorithmic HBM bytes of one launch of each cell kernel of a step's projection, each array element once:
    projection start (read m and, in every stage, two potentials and two history increments; write rhs, base,
    guess and in stage 0 phi0 for the other two: 3f + 56 per cell), residual (read phi and rhs, write r: 24 per
    cell) and finish (read phi, m and base, write u, phi and the history increment: 6f + 32 per cell)."""
    nx, ny, nz = settings['nx'], settings['ny'], settings['nz']
    cells = nx * ny * nz
    faces = (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
    return {'projection_start': faces * field_bytes + 56 * cells, 'guess_residual': 24 * cells,
            'finish': 2 * faces * field_bytes + 32 * cells}


def gemm_peak_tflops(kind):
    """Measured tensor-core GEMM rate of this GPU through cuBLAS (torch.matmul), the denominator of the transforms'
    roofline: 'fp64' (DGEMM, 8192^3) or 'tf32' (FP32 GEMM with TF32 tensor cores, 16384^3); best of 5."""
    import torch
    n = 8192 if kind == 'fp64' else 16384
    dtype = torch.float64 if kind == 'fp64' else torch.float32
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = kind == 'tf32'
    try:
        a = torch.randn(n, n, device='cuda', dtype=dtype)
        b = torch.randn(n, n, device='cuda', dtype=dtype)
        torch.matmul(a, b)
        best = None
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def uses_tensor_cores(settings, precision):
    """Whether the library runs a cavity's transforms on tcgen05 (the mixed form from 128^3 cells up, nx a multiple
    of 4, unless CAVITY_FDM says otherwise): the rule of Solver's constructor."""
    fdm = os.environ.get('CAVITY_FDM', '')
    cells = settings['nx'] * settings['ny'] * settings['nz']
    return precision == 'mixed' and settings['nx'] % 4 == 0 and (fdm == 'tc' or (fdm != 'dmma' and cells >= 1 << 21))


def transforms_roofline(settings, ms_per_pass, tc, peak_gbs, launches=6):
    """The six transforms of a pressure pass: FLOP/s against the measured cuBLAS rate of their arithmetic (FP64
    DMMA against DGEMM; the mixed form's 3xTF32 tensor-core products, counted three times, against TF32 GEMM), and
    bytes against HBM.  Six launches move 16 B per cell per transform (an 8-byte read and write; the first reads
    the FP64 residual, the last updates the FP64 potential) plus 8 B of 1/lambda; the three paired launches of
    the FP64 pass (`launches` = 3) keep every second intermediate on chip: 8 B in and out each, 8 B of 1/lambda
    and 8 B of the potential read."""
    nx, ny, nz = settings['nx'], settings['ny'], settings['nz']
    cells = nx * ny * nz
    flops = 4.0 * (nx + ny + nz) * cells * (3 if tc else 1)
    paired = not tc and launches == 3
    nbytes = (3 * 16 + 16 if paired else 6 * 16 + 8) * cells
    s = ms_per_pass / 1e3
    peak = gemm_peak_tflops('tf32' if tc else 'fp64')
    name = ('tc2_transform_kernel / tc_transform_kernel (tcgen05 3xTF32)' if tc else
            'pair_xy/pair_z/pair_yx_kernel (FP64 DMMA, two transforms per launch)' if paired else
            'dgemm_mma_kernel (FP64 DMMA)')
    return {'kernel': name, 'launches_per_pass': launches,
            'ms_per_pass': ms_per_pass, 'flops_per_pass': flops, 'achieved_tflops': flops / s / 1e12,
            'peak_tflops': peak, 'peak_kind': 'measured cuBLAS ' + ('TF32' if tc else 'DGEMM') + ' on this GPU',
            'tensor_frac': flops / s / 1e12 / peak, 'bytes_per_pass': nbytes, 'achieved_gbs': nbytes / s / 1e9,
            'hbm_frac': nbytes / s / 1e9 / peak_gbs}


def cpu_oracle_rate(workload, steps_budget_s=12.0, max_steps=40, warmup=1):
    """The FP64 OpenMP oracle on this host: cell-updates/s over a bounded number of steps after `warmup`."""
    from les_impulse3d_64_b200 import workloads
    from les_impulse3d_64_b200.api import Solver
    sys.path.insert(0, str(ROOT / 'oracle'))
    import build_oracle
    build_oracle.build_oracle()
    w = workloads.WORKLOADS[workload]
    sim = Solver(w['settings'], library=ROOT / 'oracle' / 'libcavity_oracle.so')
    try:
        sim.initialize(*workloads.initial_noise(sim.shapes, w['noise'], w['seed']))
        for _ in range(max(1, warmup)):               # warm-up (first-touch of the arrays)
            sim.step()
        t0 = time.perf_counter()
        n = 0
        while n < max_steps and (n < 2 or time.perf_counter() - t0 < steps_budget_s):
            sim.step()
            n += 1
        dt = time.perf_counter() - t0
    finally:
        sim.close()
    cells = w['settings']['nx'] * w['settings']['ny'] * w['settings']['nz']
    return cells * n / dt, n, dt


def reference_gpu_rate(workload, steps, warmup):
    """The reference's own backend.cu (oracle/_ref build) on this GPU through its C ABI, wall clock."""
    lib = ROOT / 'oracle' / '_ref' / 'libcavity_solver.so'
    if not lib.is_file():
        return None
    from les_impulse3d_64_b200 import workloads
    from les_impulse3d_64_b200.api import Solver
    w = workloads.WORKLOADS[workload]
    sim = Solver(w['settings'], library=lib)
    try:
        sim.initialize(*workloads.initial_noise(sim.shapes, w['noise'], w['seed']))
        for _ in range(warmup):
            sim.step()
        t0 = time.perf_counter()
        for _ in range(steps):
            sim.step()
        dt = time.perf_counter() - t0
    finally:
        sim.close()
    cells = w['settings']['nx'] * w['settings']['ny'] * w['settings']['nz']
    return {'value': cells * steps / dt, 'unit': 'cell-updates/s', 'steps': steps,
            'what': "reference backend.cu built unchanged for sm_100a, driven through its C ABI, wall clock"}


# ------------------------------------------------------------------------------------------ arms
def workload_config(args, w, precision, world):
    """The `config` of a bench line, the same dict in both arms."""
    s = w['settings']
    return {'workload': args.workload, 'grid': [s['nx'], s['ny'], s['nz']], 'precision': precision,
            'stretch_beta': w.get('beta'), 're': round(1.0 / s['nu']),
            'l2': 'GPU steps: flushed before each timed step (256 MiB write)', 'parallelism': f'replicas x{world}'}


def batched_rates(steps, warmup, chunk=8):
    """Sub-measurements of the default line: the mixed form batched (wall clock over all cavities, steps queued
    `chunk` at a time): 64 cavities of the C2 cavity (64^3, beta 1.5, Re 1000; seeds 0..63), and the C4 ensemble
    (256 cavities of 24^3..64^3)."""
    from les_impulse3d_64_b200 import workloads
    from les_impulse3d_64_b200.ensemble import Ensemble
    c2 = workloads.C2
    out = {}
    for name, cases in (('batched_mixed_64cube',
                         [dict(name=f'c2_{k}', settings=c2['settings'], noise=c2['noise'], seed=k, precision='mixed')
                          for k in range(64)]),
                        ('c4_ensemble_mixed', workloads.ensemble_cases(count=256))):
        ens = Ensemble(cases)
        try:
            dt, rate = ens.timed(steps, warmup=warmup, chunk=chunk)
            out[name] = {'value': rate, 'unit': 'cell-updates/s', 'cavities': len(cases), 'cells': sum(ens.cells),
                         'steps': steps, 'seconds': dt, 'timing': 'wall clock over all cavity streams'}
        finally:
            ens.close()
    return out


def serving_sample(requests, rate, t_end, chunk=8):
    """The C5 stream (sizes 32^3 .. 128^3, Re log-uniform in [100, 5000], half uniform and half regularised
    lids, Poisson arrivals at `rate`), `requests` requests to `t_end`, served in real time twice: by the mixed
    form in slot batches, and by the plain FP64 form one request at a time through its own graphs."""
    from les_impulse3d_64_b200.serve import Server, serving_requests, summary
    reqs = serving_requests(requests, rate, seed=0, t_end=t_end, with_fields=True)
    ours = summary(Server(budget_bytes=120e9, precision='mixed', chunk=chunk).run(reqs))
    plain = summary(Server(budget_bytes=120e9, precision='fp64', chunk=chunk, batched=False, max_running=1).run(reqs))
    return {'requests': requests, 'rate_per_s': rate, 't_end': t_end, 'chunk': chunk,
            'sizes': '32^3, 64^3, 64x64x128, 96^3, 128^3', 'budget_bytes': 120e9,
            'served_mixed_slot_batches': ours, 'plain_fp64_one_at_a_time': plain,
            'p50_ratio': plain['p50_s'] / ours['p50_s'], 'p99_ratio': plain['p99_s'] / ours['p99_s'],
            'throughput_ratio': ours['cell_updates_per_s'] / plain['cell_updates_per_s']}


def run_ours(args, ranks):
    from les_impulse3d_64_b200 import _build, workloads
    from les_impulse3d_64_b200.api import Cavity, Solver
    if ranks.rank == 0 and not _build.LIBRARY.is_file():
        raise SystemExit('libcavity_solver.so is not built (python __graft_entry__.py)')
    w = workloads.WORKLOADS[args.workload]
    precision = args.precision or w.get('precision', 'fp64')
    s = w['settings']
    cells = s['nx'] * s['ny'] * s['nz']
    field_bytes = 8 if precision == 'fp64' else 4

    # device-timed steps
    cav = Cavity(s, precision=precision)
    cav.initialize(*workloads.initial_noise(cav.shapes, w['noise'], w['seed']))
    passes0 = cav.pressure_passes()
    ranks.barrier()
    with ClockSampler(ranks.local) as clocks:
        ms, kms = cav.time_steps(args.warmup, args.steps, flush_l2=True)
    ktimes = cav.kernel_times()
    passes = cav.pressure_passes() - passes0
    device_bytes = cav.device_bytes()
    per_pass = (cav.kernels_per_step(1) - cav.kernels_per_step(0)) // 3       # transforms + residual
    launches = args.steps * cav.kernels_per_step(0) + per_pass * passes_in_timed(passes, args, cav)
    cav.close()
    total_ms = ranks.max(float(ms.sum()))
    value = replica_rate(ranks.world, cells, args.steps, total_ms)

    # end to end through the reference-facing ABI with host buffers
    sim = Solver(s, precision=precision)
    v, wn = workloads.initial_noise(sim.shapes, w['noise'], w['seed'])
    sim.initialize(v, wn)
    for _ in range(args.warmup):
        sim.step()
    # the 7 output arrays are the caller's, allocated and touched before the timed region (a caller that reads
    # fields repeatedly reuses its buffers): the copies into them are timed, the first-touch page faults of new
    # host memory are not
    names = ('u', 'v', 'w', 'mx', 'my', 'mz', 'phi')
    fields = [np.ones(sim.shapes[k], dtype=np.float64 if k == 'phi' else np.float32) for k in names]
    ranks.barrier()
    t0 = time.perf_counter()
    sim.initialize(v, wn)
    for _ in range(args.steps):
        sim.step()
        sim.probes()
    for k, f in zip(names, fields):
        sim.field(k, out=f)
    e2e_s = ranks.max(time.perf_counter() - t0)
    sim.close()
    h2d = (v.nbytes + wn.nbytes) / args.steps
    d2h = 48 + 8 * s.get('n_probes', len(s['probes'])) + sum(f.nbytes for f in fields) / args.steps

    # the same, with the steps queued and their probe values kept on the device until one sync
    # (cavity_step_outputs_async / cavity_sync_outputs) instead of a blocking probe read per step
    cav = Cavity(s, precision=precision)
    cav.initialize(v, wn)
    cav.step_outputs_async(args.warmup)
    cav.sync_outputs()
    qfields = [np.ones_like(f) for f in fields]
    ranks.barrier()
    t0 = time.perf_counter()
    cav.initialize(v, wn)
    cav.step_outputs_async(args.steps)
    cav.sync_outputs()
    for k, f in zip(names, qfields):
        cav.field(k, out=f)
    queued_s = ranks.max(time.perf_counter() - t0)
    cav.close()
    del qfields

    peak, peak_kind = measured_peaks()
    kernel_s = float(kms.sum()) / 1e3 / (3 * args.steps)
    achieved = momentum_bytes(s, field_bytes) / kernel_s / 1e9
    # the other stencil kernels of the step, timed by events in the same graph (their launches in all stages)
    cell_kernels = {}
    for name, nbytes in cell_kernel_bytes(s, field_bytes).items():
        launch_s = ranks.max(ktimes[name]) / 1e3 / 3
        gbs = nbytes / launch_s / 1e9 if launch_s > 0 else None
        cell_kernels[name] = {'ms_per_launch': launch_s * 1e3, 'bytes_per_launch': nbytes, 'achieved_gbs': gbs,
                              'frac': gbs / peak if gbs else None}
    line = {
        'metric': 'cell-updates/s per RK3 step', 'value': value, 'unit': 'cell-updates/s', 'n_gpus': ranks.world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total_ms / args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64' if precision == 'fp64' else 'f32',
        'data': 'synthetic (seeded Gaussian initial noise, numpy default_rng)',
        'config': workload_config(args, w, precision, ranks.world),
        'device_bytes': device_bytes,
        'e2e': {'value': ranks.world * cells * args.steps / e2e_s, 'unit': 'cell-updates/s',
                'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h},
        'e2e_queued_outputs': {'value': ranks.world * cells * args.steps / queued_s, 'unit': 'cell-updates/s',
                               'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h},
        'gpu_launches': launches,
        'pressure_passes_per_stage': passes / (3 * (2 * args.steps + args.warmup)) if args.steps else None,
        'roofline': {'kernel': sweep_kernel_name(precision), 'bound': 'hbm', 'achieved': achieved, 'peak': peak,
                     'peak_kind': peak_kind, 'unit': 'GB/s', 'frac': achieved / peak,
                     'traffic': profile_traffic(args.workload), 'ms_per_launch': kernel_s * 1e3},
        'stencil_kernels': cell_kernels,
        'transforms': transforms_roofline(s, ranks.max(ktimes['transforms']) / 3, uses_tensor_cores(s, precision), peak,
                                          per_pass - 1),
        'clocks': clocks.summary(),
    }
    if not args.no_batched and args.workload == 'c2_64cube_re1000':
        # the mixed form batched against this line's plain FP64 value (device time, single cavity)
        ranks.barrier()
        sub = batched_rates(args.steps, max(3, args.warmup))
        for v in sub.values():
            v['value'] = ranks.world * v['value'] * (v['seconds'] / ranks.max(v['seconds']))
            v['ratio_vs_value'] = v['value'] / value
        line['batched'] = sub
    if not args.no_serving and args.workload == 'c2_64cube_re1000' and ranks.world == 1:
        line['serving'] = serving_sample(args.serving_requests, 50.0, args.serving_t_end)
    if ranks.rank == 0 and ranks.world == 1 and not args.no_cpu_baseline:
        rate, n, dt = cpu_oracle_rate(args.workload)
        line['cpu_baseline'] = {'value': rate, 'unit': 'cell-updates/s', 'cores': os.cpu_count(), 'kind': 'port',
                                'sample': f'{n} steps of {args.workload} from its seeded initial state, {dt:.1f} s'}
    return line


def replica_rate(world, cells, steps, max_ms):
    """Whole-job cell-updates/s of `world` replicas that each advanced `cells` cells by `steps` steps, timed
    by the slowest rank."""
    return world * cells * steps / (max_ms / 1e3)


def passes_in_timed(passes, args, cav):
    # passes counted over warm-up, timed steps and the kernel-timing steps after them; scale to the timed steps
    total = 2 * args.steps + args.warmup
    return int(round(passes * args.steps / total)) if total else 0


def run_ensemble(args, ranks):
    """The batched ensemble (C4): every rank advances its own copy of the ensemble; wall-clock over all streams."""
    from les_impulse3d_64_b200 import workloads
    from les_impulse3d_64_b200.ensemble import Ensemble
    cases = workloads.ensemble_cases(count=args.count)
    if args.precision:
        for c in cases:
            c['precision'] = args.precision
    ens = Ensemble(cases)
    try:
        ranks.barrier()
        with ClockSampler(ranks.local) as clocks:
            dt, _ = ens.timed(args.steps, warmup=args.warmup, chunk=args.chunk)
        cells = sum(ens.cells)
        device_bytes = ens.device_bytes()
    finally:
        ens.close()
    dt = ranks.max(dt)
    value = ranks.world * cells * args.steps / dt
    return {
        'metric': 'cell-updates/s per RK3 step', 'value': value, 'unit': 'cell-updates/s', 'n_gpus': ranks.world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': dt / args.steps * 1e3, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32' if (args.precision or 'mixed') == 'mixed' else 'f64',
        'data': 'synthetic (seeded Gaussian initial noise, numpy default_rng)',
        'config': {'workload': 'c4_ensemble', 'cavities': args.count, 'cells': cells, 'device_bytes': device_bytes,
                   'steps_queued_per_wait': args.chunk, 'timing': 'wall clock over all cavity streams',
                   'parallelism': f'replicas x{ranks.world}'},
        'clocks': clocks.summary(),
    }


def run_serving(args, ranks):
    """C5: a seeded Poisson stream of cavity requests served in real time by the batched mixed-form server,
    then by the plain FP64 form one request at a time; p50 / p99 time to solution of each."""
    from les_impulse3d_64_b200.serve import Server, serving_requests, summary
    reqs = serving_requests(args.requests, args.rate, seed=0, t_end=args.t_end, with_fields=True)
    ranks.barrier()
    with ClockSampler(ranks.local) as clocks:
        ours = summary(Server(budget_bytes=120e9, precision=args.precision or 'mixed', chunk=args.chunk).run(reqs))
    plain = summary(Server(budget_bytes=120e9, precision='fp64', chunk=args.chunk, batched=False,
                           max_running=1).run(reqs))
    ours['p50_ratio_vs_plain'] = plain['p50_s'] / ours['p50_s']
    ours['throughput_ratio_vs_plain'] = ours['cell_updates_per_s'] / plain['cell_updates_per_s']
    p99 = ranks.max(ours['p99_s'])
    return {
        'metric': 'p99 time-to-solution', 'value': p99, 'unit': 's', 'n_gpus': ranks.world, 'steps': None,
        'warmup': 0, 'ms_per_step': None, 'higher_is_better': False, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32' if (args.precision or 'mixed') == 'mixed' else 'f64',
        'data': 'synthetic (seeded Poisson request stream, numpy default_rng)',
        'config': {'workload': 'c5_serving', 'requests': args.requests, 'rate_per_s': args.rate,
                   't_end': args.t_end, 'sizes': '32^3, 64^3, 64x64x128, 96^3, 128^3', 'budget_bytes': 120e9,
                   'chunk': args.chunk, 'parallelism': f'replicas x{ranks.world}'},
        'serving': ours, 'plain_fp64_one_at_a_time': plain,
        'clocks': clocks.summary(),
    }


def run_reference(args, ranks):
    if ranks.rank != 0:
        return None
    from les_impulse3d_64_b200 import workloads
    w = workloads.WORKLOADS[args.workload]
    rate, n, dt = cpu_oracle_rate(args.workload, steps_budget_s=max(10.0, 2.0 * args.steps), max_steps=args.steps,
                                  warmup=args.warmup)
    line = {
        'metric': 'cell-updates/s per RK3 step', 'value': rate, 'unit': 'cell-updates/s', 'n_gpus': ranks.world,
        'steps': n, 'warmup': max(1, args.warmup), 'ms_per_step': dt / n * 1e3, 'higher_is_better': True,
        'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic (seeded Gaussian initial noise, numpy default_rng)',
        'config': workload_config(args, w, args.precision or w.get('precision', 'fp64'), ranks.world),
        'impl': 'reference',
        'cpu_baseline': {'value': rate, 'unit': 'cell-updates/s', 'cores': os.cpu_count(), 'kind': 'port',
                         'sample': f'{n} steps of {args.workload}, {dt:.1f} s (the reference ships no CPU path; '
                                   'this is its FP64 OpenMP restatement)'},
        'e2e': {'value': rate, 'unit': 'cell-updates/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    try:
        ref = reference_gpu_rate(args.workload, args.steps, args.warmup)
        if ref:
            line['reference_binary_gpu'] = ref
    except Exception as exc:          # the GPU reference build is an extra point, not the arm itself
        line['reference_binary_gpu'] = {'unavailable': f'{type(exc).__name__}: {exc}'}
    return line


def main():
    args = parse_args()
    ranks = Ranks()
    try:
        if args.impl == 'reference':
            line = run_reference(args, ranks)
        elif args.workload == 'c4_ensemble':
            line = run_ensemble(args, ranks)
        elif args.workload == 'c5_serving':
            line = run_serving(args, ranks)
        else:
            line = run_ours(args, ranks)
        if line is not None and ranks.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        ranks.close()


if __name__ == '__main__':
    main()
