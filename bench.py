#!/usr/bin/env python
"""Benchmark of the grid hot path: multigrid Poisson solves per second.

Workload (one "step"): a batch of B independent Poisson solves on a 128^3
zero-boundary grid (N_c = 128, 127^3 unknowns, h = 0.2 Angstrom), each
density a sum of 8 normalised Gaussians (widths U[0.5, 1.5] A, charges +-1,
re-centred to neutral; seeded synthetic data), solved with the reference's
method -- PoissonSolver(nn=3, relax='J'), the V-cycle schedule of
gpaw/poisson.py -- from a zero start to relative residual
||A phi - rho|| / ||rho|| <= 1e-10, i.e. the reference's own stopping test
sum(r^2) dv <= eps with eps = 1e-20 sum(rho^2) dv.

  value  solves/s over all ranks, inputs resident in HBM (device tensors)
  e2e    the same through the public API (PoissonSolver.solve_stream)
         from pinned host buffers: every step's densities copied in and
         potentials copied out inside the timed region, the copies
         overlapped with the neighbouring steps' solves
  roofline  the level-0 kernel with the largest time per outer iteration,
         timed live with CUDA events on the engine's stream: algorithmic
         bytes (each compulsory read and write once) / launch time
  cpu_baseline  the reference's own C (oracle/_ref) driven by the restated
         solver, one solve per host core in parallel, rank 0 only

  single_solve  latency of the drop-in PoissonSolver.solve(phi, rho) on one
         grid with NumPy arrays (GPAW's once-per-SCF-step call)

Every timed solve runs solve()'s charge integral and branch (background shift
or Gaussian compensation) on the device before its V-cycles.

--impl reference times that CPU implementation alone, as its own arm.
Multi-GPU (one process per GPU; --gpus N without a launcher relaunches under
torchrun): every rank solves its own batch (weak scaling) with no exchange in
the timed region; after it, the per-solve results (V-cycles, final error,
E_H) are all-gathered to rank 0 and the timings reduced by max.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 128
N_GRID_PTS = (N_GRID - 1) ** 3   # unknowns of one zero-boundary grid
H_ANG = 0.2
N_GAUSS = 8
REL_TOL = 1e-10
METRIC = 'poisson_solves_per_s_128^3_rel1e-10'


def densities(B, seed0):
    from gpawdft_b200.workloads import gaussian_density
    rhos = []
    L = None
    for i in range(B):
        rho, L = gaussian_density(N_GRID, H_ANG, N_GAUSS, seed0 + i)
        rhos.append(rho)
    return np.array(rhos), L


def eps_for(rho, dv):
    return REL_TOL ** 2 * float(np.dot(rho.ravel(), rho.ravel())) * dv


def _plain(o):
    """JSON fallback for ctypes / NumPy scalars."""
    if hasattr(o, 'value'):
        return o.value
    if isinstance(o, np.generic):
        return o.item()
    raise TypeError(type(o).__name__)


# ------------------------------------------------------------------ sharding
# The path shards by independent solves: each rank solves its own batch of
# densities (seeds disjoint across ranks, up to 1000 solves per rank) with no
# data exchange; the only collective is the max over ranks of the timings.
def shard_seed0(rank):
    return 1 + 1000 * rank


def reduce_max(x, dist, device):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


RESULT_COLUMNS = ('seed', 'vcycles', 'error', 'E_H')


def gather_results(table, dist, device):
    """All-gather each rank's per-solve table (rows: seed, V-cycles, final
    error sum(r^2) dv, Hartree energy) into the whole job's table, ordered by
    rank.  Every rank has the same number of rows."""
    table = np.ascontiguousarray(table, np.float64)
    if dist is None:
        return table
    import torch
    t = torch.from_numpy(table).to(device)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    return torch.cat(parts).cpu().numpy()


def results_summary(table, rho_norms):
    """Whole-job summary of the gathered per-solve table."""
    rel = np.sqrt(table[:, 2] / rho_norms) if rho_norms is not None else None
    return {'solves': int(len(table)),
            'columns': list(RESULT_COLUMNS),
            'vcycles_min': int(table[:, 1].min()),
            'vcycles_max': int(table[:, 1].max()),
            'max_rel_residual': (float(rel.max()) if rel is not None
                                 else None),
            'E_H_sum_Ha': float(table[:, 3].sum()),
            'seeds_distinct': bool(len(np.unique(table[:, 0])) ==
                                   len(table))}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples (100 ms period).

    Started before the warm-up so that the sampler is running when the
    timed region begins; ``window(t0, t1)`` keeps the samples whose host
    timestamps fall inside the timed region.
    """

    Q = ('timestamp,index,clocks.sm,clocks.max.sm,power.draw,'
         'clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')
    NAMES = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
             'sw_power_cap']

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.reader = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.Q,
                 '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        time.sleep(1.0)  # nvidia-smi start-up

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line))

    def stop(self, t0=None, t1=None):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None,
                    'reasons': ['unsampled']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.reader is not None:
            self.reader.join(timeout=5)
        rows = []
        for ts, line in self.lines:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                rows.append((ts, float(f[2]), float(f[3]),
                             [n for n, v in zip(self.NAMES, f[5:9])
                              if v.lower() == 'active']))
            except ValueError:
                continue
        # a sample line is printed when it is taken: keep those stamped in
        # the timed window (plus one period of slack on each side)
        sel = [r for r in rows if t0 is None or t0 - 0.1 <= r[0] <= t1 + 0.1]
        scope = 'timed region'
        if not sel:
            sel, scope = rows, 'whole run (timed region shorter than a sample)'
        if not sel:
            return {'sm_mhz': None, 'sm_max_mhz': None,
                    'reasons': ['unsampled']}
        reasons = sorted({n for r in sel for n in r[3]})
        return {'sm_mhz': float(np.median([r[1] for r in sel])),
                'sm_max_mhz': max(r[2] for r in sel), 'reasons': reasons,
                'samples': len(sel), 'scope': scope}


# ------------------------------------------------------------------ CPU side
def _cpu_solve(args):
    """One reference-C solve (process-pool worker)."""
    seed, backend = args
    from gpawdft_b200.workloads import gaussian_density
    from oracle import layer
    from oracle.geometry import GridDescriptor
    rho, L = gaussian_density(N_GRID, H_ANG, N_GAUSS, seed)
    gd = GridDescriptor((N_GRID,) * 3, (L,) * 3, 0)
    ps = layer.PoissonSolver(nn=3, relax='J', eps=eps_for(rho, gd.dv),
                             maxiter=1000, backend=backend)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    phi = gd.zeros()
    t = time.perf_counter()
    n = ps.solve(phi, rho)
    return n, time.perf_counter() - t


def cpu_arm(rounds, warmup, seed0=10_000):
    """Rounds of one solve per host core; returns per-round solves/s."""
    import multiprocessing as mp
    from oracle import ref
    backend = 'ref' if ref.available() else 'numpy'
    kind = 'reference' if backend == 'ref' else 'port'
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    ctx = mp.get_context('spawn')
    rates, niters = [], []
    with ctx.Pool(cores) as pool:
        for r in range(warmup + rounds):
            args = [(seed0 + r * cores + i, backend) for i in range(cores)]
            t = time.perf_counter()
            res = pool.map(_cpu_solve, args)
            dt = time.perf_counter() - t
            if r >= warmup:
                rates.append(cores / dt)
                niters.extend(n for n, _ in res)
    return {'rates': rates, 'cores': cores, 'kind': kind,
            'sample': '%d rounds x %d concurrent %d^3 solves (one per core), '
                      'reference C via the restated solver, %s' %
                      (rounds, cores, N_GRID - 1,
                       'oracle/_ref' if kind == 'reference' else 'NumPy port'),
            'vcycles_mean': float(np.mean(niters)) if niters else None}


def run_reference(args, rank, world):
    if rank != 0:
        return
    # one round (a solve per host core) takes ~10 s on a 16-core host: the
    # sample is capped at 6 timed rounds and 1 warm-up round so that the
    # reference arm ends within a couple of minutes whatever K and W are
    # (a step here is one such round; the line reports the rounds it timed)
    rounds, warm = max(1, min(args.steps, 6)), min(args.warmup, 1)
    r = cpu_arm(rounds, warm)
    v = float(np.mean(r['rates']))
    line = {'metric': METRIC, 'value': v, 'unit': 'solves/s', 'n_gpus': world,
            'steps': rounds, 'warmup': warm,
            'steps_requested': args.steps, 'warmup_requested': args.warmup,
            'step': 'one round: a solve per host core, run concurrently',
            'ms_per_step': 1000.0 * r['cores'] / v,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f64', 'data': 'synthetic', 'impl': 'reference',
            'config': config_dict(args, world, r['cores'], 'fp64'),
            'cpu_baseline': {'value': v, 'unit': 'solves/s',
                             'cores': r['cores'], 'kind': r['kind'],
                             'sample': r['sample']},
            'e2e': {'value': v, 'unit': 'solves/s', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0},
            'vcycles_mean': r['vcycles_mean'],
            'rounds_timed': rounds, 'rounds_warmup': warm}
    print(json.dumps(line), flush=True)


def config_dict(args, world, batch, precision=None):
    return {'workload': 'Poisson FD multigrid, N_c=%d zero boundary (%d^3 '
                        'unknowns), h=%.2f A, nn=3 Jacobi, %d Gaussians, '
                        'relative residual %g' % (N_GRID, N_GRID - 1, H_ANG,
                                                  N_GAUSS, REL_TOL),
            'batch_per_gpu': batch, 'grid': [N_GRID - 1] * 3,
            'precision': precision or args.precision,
            'parallelism': 'dp%d' % world,
            'l2': 'inputs larger than L2 (%d grids x %.1f MB per array)' %
                  (batch, (N_GRID - 1) ** 3 * 8 / 1e6)}


# ------------------------------------------------------------------ GPU arm
def run_ours(args, rank, world, dist):
    import torch
    from gpawdft_b200 import _lib
    from gpawdft_b200.fd_operators import Laplace
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver

    dev = torch.device('cuda', int(os.environ.get('LOCAL_RANK', 0)))
    torch.cuda.set_device(dev)
    B = args.batch
    rho_h, L = densities(B, shard_seed0(rank))
    gd = GridDescriptor((N_GRID,) * 3, (L,) * 3, 0)
    eps = [eps_for(r, gd.dv) for r in rho_h]
    ps = PoissonSolver(nn=3, relax='J', maxiter=1000, precision=args.precision,
                       batch=B)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    if args.host_loop:
        ps.set_device_loop(False)
    lib = _lib.load()
    rho_d = torch.from_numpy(rho_h).to(dev)
    phi_d = torch.zeros_like(rho_d)
    rho_pin = torch.from_numpy(rho_h).pin_memory()
    phi_pin = torch.empty_like(rho_pin).pin_memory()
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, dist, dev)

    def stats():
        import ctypes
        k = ctypes.c_int64()
        g = ctypes.c_int64()
        lib.gpw_poisson_last_stats(ps._engine[0], ctypes.byref(k),
                                   ctypes.byref(g))
        return k.value, g.value

    # ---- device-resident throughput
    niters = None
    clk = ClockSampler(dev.index)
    clk.start()
    for _ in range(args.warmup):
        phi_d.zero_()
        niters = ps.solve_batch(phi_d, rho_d, eps=eps)
    barrier()
    launches = 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record(stream)
    for _ in range(args.steps):
        phi_d.zero_()
        niters = ps.solve_batch(phi_d, rho_d, eps=eps)
        # the engine's launches plus the charge branch's: sum, shift and
        # (zero boundary) the Gaussian finish
        launches += stats()[0] + 3
    e1.record(stream)
    barrier()
    clocks = clk.stop(w0, time.time())
    t_dev = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
    value = world * B * args.steps / t_dev

    # ---- per-solve results of the last timed step, gathered from every rank
    # (the path's one data collective, after the timed region)
    from gpawdft_b200 import blas
    seeds = shard_seed0(rank) + np.arange(B)
    e_h = 0.5 * gd.dv * blas.vector_dots(phi_d, rho_d, B)
    table = np.stack([seeds, np.asarray(niters, float),
                      np.asarray(ps.last_errors, float), e_h], axis=1)
    rho_sq = np.array([float(np.dot(r.ravel(), r.ravel())) * gd.dv
                       for r in rho_h])
    all_table = gather_results(table, dist, dev)
    all_rho_sq = gather_results(rho_sq[:, None], dist, dev)[:, 0]
    results = results_summary(all_table, all_rho_sq)

    # ---- end to end through the public API from pinned host memory: every
    # step's densities go host -> device and its potentials device -> host;
    # solve_stream overlaps those copies with the neighbouring steps' solves
    phi_pins = [phi_pin, torch.empty_like(rho_pin).pin_memory()]
    rho_steps = [rho_pin] * args.steps
    out_steps = [phi_pins[k % 2] for k in range(args.steps)]
    ps.solve_stream(rho_steps[:2], eps=eps, out=out_steps[:2])   # warm-up
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    _, e2e_niters = ps.solve_stream(rho_steps, eps=eps, out=out_steps)
    f1.record(stream)
    barrier()
    t_e2e = max_over_ranks(f0.elapsed_time(f1) / 1000.0)
    e2e = world * B * args.steps / t_e2e
    io_bytes = rho_h.nbytes   # per step: densities in, potentials out
    assert all(np.array_equal(n, niters) for n in e2e_niters)

    # ---- dominant kernels, timed live on the engine's stream and buffers:
    # float64 form: the level-0 Jacobi sweep; float32 form: the fused
    # level-0 float32 sweep that adds its result into float64 phi
    import ctypes
    kernels = {}
    names = {0: 'star_tma_kernel<double,3,JACOBI> level-0 sweep',
             1: 'star_tma_kernel<double,3,RESIDUAL> level-0 residual+norm',
             2: 'star_tma_kernel<float,3,JACOBI> level-0 sweep',
             3: 'star_tma_kernel<float,3,JACOBI_ADD64> level-0 sweep + phi64 update',
             4: 'star_tma_kernel<double,3,RESID_DC> level-0 fp64 defect',
             5: 'star_tma_kernel<float,3,RESIDUAL> level-0 residual',
             6: 'star_tma_kernel<float,3,RESID_RESTRICT> level-0 residual '
                '+ restriction into level 1',
             7: 'star_tma_kernel<float,3,JACOBI_SCALED_IN> level-0 sweep '
                'reading the defect alone'}
    # launches of each per outer iteration: float64 method 3 sweeps + 2
    # residuals; float32 form (2 + 2 Chebyshev sweeps on level 0) 2 plain
    # sweeps, 1 residual, 1 defect, 1 update
    # (the float32 form's level-0 residual is restricted in the same launch
    # where the grid allows it: which 6, else the plain residual, which 5;
    # its second pre-sweep reads the defect alone where the plan allows it:
    # which 7 and one plain sweep, else two plain sweeps)
    per_iter = ({0: 3, 1: 2} if args.precision == 'fp64' else
                {2: 1, 7: 1, 6: 1, 4: 1, 3: 1})
    for which in list(per_iter):
        ms, nbytes = ctypes.c_double(), ctypes.c_double()
        rc = lib.gpw_poisson_time_level0(
            ps._engine[0], B, which, 20, ctypes.byref(ms), ctypes.byref(nbytes),
            stream.cuda_stream)
        if rc == _lib.GPW_ENOTSUP and which == 7:
            del per_iter[7]
            per_iter[2] = 2
            continue
        if rc == _lib.GPW_ENOTSUP and which == 6:
            del per_iter[6]
            per_iter[5] = 1
            which = 5
            rc = lib.gpw_poisson_time_level0(
                ps._engine[0], B, which, 20, ctypes.byref(ms),
                ctypes.byref(nbytes), stream.cuda_stream)
        _lib.check(rc)
        kernels[which] = (ms.value / 1e3, nbytes.value)
    # the dominant kernel: the largest time per outer iteration
    dom = max(per_iter, key=lambda w: kernels[w][0] * per_iter[w])
    # DRAM bytes (read + write) per grid point of the level-0 kernels, from
    # single-launch ncu captures of these kernels at 8 x 127^3 points
    # ((dram__bytes_read.sum + dram__bytes_write.sum) / points); traffic
    # grows with the points, so a launch's traffic is this times its points
    ncu_bytes_per_point = {2: (139.83e6 + 40.00e6) / 16387064,
                           4: (292.3e6 + 103.9e6) / 16387064,
                           3: (268.9e6 + 90.9e6) / 16387064}
    if 7 in per_iter:  # the defect without the stored first iterate
        ncu_bytes_per_point[4] = (284.82e6 + 49.36e6) / 16387064
    t_sweep, sweep_bytes = kernels[dom]
    achieved = sweep_bytes / t_sweep / 1e9
    peak, peak_src = measured_peak()
    kernel_table = {names[w]: {'ms': t * 1e3, 'GB/s': b / t / 1e9,
                               'frac': b / t / 1e9 / peak,
                               'launches_per_iteration': per_iter[w]}
                    for w, (t, b) in kernels.items()}

    # ---- the plain float64 method on the same batch, for the ratio
    fp64_plain = None
    if args.precision == 'fp32':
        ps64 = PoissonSolver(nn=3, relax='J', maxiter=1000, precision='fp64',
                             batch=B)
        ps64.set_grid_descriptor(gd)
        ps64.initialize()
        for _ in range(2):
            phi_d.zero_()
            ps64.solve_batch(phi_d, rho_d, eps=eps)
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.steps):
            phi_d.zero_()
            n64 = ps64.solve_batch(phi_d, rho_d, eps=eps)
        g1.record(stream)
        torch.cuda.synchronize()
        t64 = max_over_ranks(g0.elapsed_time(g1) / 1000.0)
        fp64_plain = {'value': world * B * args.steps / t64,
                      'unit': 'solves/s', 'vcycles_mean': float(np.mean(n64))}
        del ps64

    # ---- one grid per call through the drop-in PoissonSolver.solve(phi, rho)
    # with NumPy host arrays (GPAW's once-per-SCF-step call): host wall-clock
    # latency per call, the copies in and out included
    single = single_solve(args, gd, rho_h[0], eps[0])

    # ---- live per-launch breakdown of one outer iteration (eager launches)
    breakdown = [{'launch': n, 'ms': t}
                 for n, t in ps.profile_iteration(B, reps=5)]

    # ---- secondary: config (a) Laplace apply, 32 x 48^3 float64, zero BC
    stencil = stencil_config_a(dev, stream)

    out = {'metric': METRIC, 'value': value, 'unit': 'solves/s',
           'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
           'ms_per_step': 1000.0 * t_dev / args.steps,
           'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
           'dtype': 'f64' if args.precision == 'fp64' else 'f32+f64',
           'data': 'synthetic (seeded Gaussian-sum densities)',
           'config': config_dict(args, world, B),
           'e2e': {'value': e2e, 'unit': 'solves/s',
                   'h2d_bytes_per_step': io_bytes,
                   'd2h_bytes_per_step': io_bytes},
           'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak,
                        'unit': 'GB/s', 'frac': achieved / peak,
                        'traffic': (ncu_bytes_per_point[dom] * B * N_GRID_PTS
                                    if dom in ncu_bytes_per_point else None),
                        'traffic_source': 'ncu capture at batch 8, scaled to '
                                          'the launch\'s grid points',
                        'kernel': names[dom] + ' (batch %d)' % B,
                        'algorithmic_bytes_per_launch': sweep_bytes,
                        'launch_ms': t_sweep * 1e3,
                        'peak_source': peak_src,
                        'level0_kernels': kernel_table},
           'fp64_plain': fp64_plain,
           'gpu_launches': int(launches),
           'clocks': clocks,
           'vcycles': [int(x) for x in niters],
           'results': results,
           'single_solve': single,
           'iteration_breakdown': breakdown,
           'stencil_config_a': stencil}
    if rank == 0 and world == 1 and not args.no_secondary:
        # the other configurations' key numbers, measured after the timed
        # region on the same GPU (each also runs alone: --workload bands96 /
        # general / mixed192 / uneven512)
        import copy
        sa = copy.copy(args)
        sa.steps = min(args.steps, 10)
        del ps, rho_d, phi_d
        torch.cuda.empty_cache()
        sec = {}
        for key, fn in (('bands96', bands_line), ('general', general_line),
                        ('mixed192', mixed192_line), ('uneven512', uneven_line)):
            w0 = time.time()
            line = fn(sa)
            line['wall_s'] = time.time() - w0
            sec[key] = line
            torch.cuda.empty_cache()
        out['secondary'] = sec
    if rank == 0 and world == 1 and not args.no_cpu:
        r = cpu_arm(1, 0)
        out['cpu_baseline'] = {'value': float(np.mean(r['rates'])),
                               'unit': 'solves/s', 'cores': r['cores'],
                               'kind': r['kind'], 'sample': r['sample']}
    if rank == 0:
        print(json.dumps(out, default=_plain), flush=True)


def single_solve(args, gd, rho, eps, calls=10):
    """Latency of PoissonSolver.solve(phi, rho) on one 127^3 grid with NumPy
    arrays: each call copies rho in, runs the charge integral, the branch and
    the device-side V-cycle loop, and copies phi back."""
    from gpawdft_b200.poisson import PoissonSolver
    ps1 = PoissonSolver(nn=3, relax='J', maxiter=1000,
                        precision=args.precision, batch=1)
    ps1.set_grid_descriptor(gd)
    ps1.initialize()
    phi = np.zeros_like(rho)
    for _ in range(3):
        phi[:] = 0.0
        ps1.solve(phi, rho, eps=eps)
    ts = []
    n = None
    for _ in range(calls):
        phi[:] = 0.0
        t = time.perf_counter()
        n = ps1.solve(phi, rho, eps=eps)
        ts.append(time.perf_counter() - t)
    ts = np.array(ts) * 1e3
    return {'call': 'PoissonSolver.solve(phi, rho), NumPy float64 arrays, '
                    'one %d^3 grid, zero start' % (N_GRID - 1),
            'precision': args.precision, 'vcycles': int(n),
            'latency_ms_p50': float(np.median(ts)),
            'latency_ms_max': float(ts.max()),
            'solves_per_s': float(1e3 / ts.mean()),
            'timer': 'host wall clock around each call (%d calls)' % calls,
            'h2d_bytes': int(rho.nbytes), 'd2h_bytes': int(rho.nbytes)}


def measured_peak():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(p) as f:
            return float(json.load(f)['hbm_gbs']), 'MEASURED_PEAKS.json hbm_gbs (measured)'
    except Exception:
        return 6650.0, 'fallback 6.65 TB/s'


def stencil_config_a(dev, stream):
    """Laplace nn=3 apply on 32 x 48^3 float64 (and a 16x batch): GB/s."""
    import torch
    from gpawdft_b200.fd_operators import Laplace
    from gpawdft_b200.grid_descriptor import GridDescriptor
    h = 0.2 / 0.52917721
    gd = GridDescriptor((49,) * 3, (49 * h,) * 3, 0)
    op = Laplace(gd, 1.0, 3)
    res = {}
    peak, _ = measured_peak()
    for nb in (32, 512):
        g = torch.Generator(device=dev).manual_seed(0)
        a = torch.randn((nb, 48, 48, 48), dtype=torch.float64, device=dev,
                        generator=g)
        o = torch.empty_like(a)
        for _ in range(3):
            op.apply(a, o)
        torch.cuda.synchronize()
        reps = 20 if nb == 32 else 5
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            op.apply(a, o)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1000.0 / reps
        gbs = 2 * a.numel() * 8 / t / 1e9
        res['batch%d' % nb] = {'ms': t * 1e3, 'GB/s': gbs, 'frac': gbs / peak,
                               'l2_resident': nb == 32}
        del a, o
    return res


# ------------------------------------------------------------------ other configs
def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_mixed192(args):
    print(json.dumps(mixed192_line(args)), flush=True)


def mixed192_line(args):
    """Mixed precision: one 191^3 solve (N_c=192, h=0.15 A, 64 Gaussians with
    log-uniform widths 0.3-2.0 A and N(0,1) charges re-centred to neutral,
    seed 4) to relative residual 1e-10: float32 V-cycles inside float64
    defect correction -- the tuned Chebyshev schedule on the full hierarchy,
    and the configuration as written (4 levels, 2 pre- and 2 post-smoothing
    weighted-Jacobi sweeps) -- against the plain float64 method; E_H error of
    each against the float64 result.  (tests/test_gpu_mixed192.py checks all
    three against the reference's own C at this size.)"""
    import torch
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    from gpawdft_b200.workloads import gaussian_density
    N = 192
    rho, L = gaussian_density(N, 0.15, 64, 4, sigma_range=(0.3, 2.0),
                              log_sigma=True, charges='normal')
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    eps = eps_for(rho, gd.dv)
    rho_d = torch.from_numpy(rho).cuda()
    res = {}
    plans = {'fp64': ('fp64', 'reference', None),
             'fp32': ('fp32', 'chebyshev', None),
             'fp32_4levels_jacobi22': ('fp32', 'jacobi22', 4)}
    for key, (prec, inner, levels) in plans.items():
        ps = PoissonSolver(nn=3, relax='J', maxiter=1000, precision=prec,
                           inner=inner, max_levels=levels)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = torch.zeros_like(rho_d)
        for _ in range(max(1, args.warmup)):
            phi.zero_()
            ps.solve_batch(phi.unsqueeze(0), rho_d.unsqueeze(0), eps=eps)
        ts = []
        for _ in range(args.steps):
            phi.zero_()
            e0, e1 = _events()
            e0.record()
            n = ps.solve_batch(phi.unsqueeze(0), rho_d.unsqueeze(0), eps=eps)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        ph = phi.cpu().numpy()
        res[key] = {'time_s': float(np.median(ts)), 'vcycles': int(n[0]),
                    'levels': ps.levels + 1, 'inner': inner,
                    'E_H': 0.5 * gd.dv * float(np.dot(ph.ravel(), rho.ravel())),
                    'final_error': float(ps.last_errors[0])}
    line = {'metric': 'poisson_time_to_solution_191^3_rel1e-10',
            'value': res['fp32']['time_s'], 'unit': 's',
            'higher_is_better': False, 'n_gpus': 1, 'steps': args.steps,
            'warmup': args.warmup, 'dtype': 'f32+f64', 'data': 'synthetic',
            'config': {'workload': 'mixed-precision Poisson, N_c=192 zero '
                                   'boundary (191^3), h=0.15 A, 64 Gaussians'},
            'fp64_plain': res['fp64'], 'fp32_dc': res['fp32'],
            'E_H_error_Ha': abs(res['fp32']['E_H'] - res['fp64']['E_H']),
            'speedup_vs_fp64': res['fp64']['time_s'] / res['fp32']['time_s'],
            'as_written': dict(res['fp32_4levels_jacobi22'], E_H_error_Ha=abs(
                res['fp32_4levels_jacobi22']['E_H'] - res['fp64']['E_H']),
                speedup_vs_fp64=res['fp64']['time_s'] /
                res['fp32_4levels_jacobi22']['time_s'])}
    return line


def run_general(args):
    print(json.dumps(general_line(args)), flush=True)


def general_line(args):
    """General-offset stencils (gpaw/fd_operators.py:158-251): the GUC
    Laplacian of a face-centred-cubic cell (6 directions, nn=3: 37 points)
    on complex128 Bloch bands of a 96^3 periodic grid, and the Mehrstellen
    pair (LaplaceA, 19 points; LaplaceB, 7 points) on float64 127^3
    zero-boundary grids (the Poisson solver's nn='M').  GB/s of algorithmic
    bytes (input read once, output written once)."""
    import torch
    from gpawdft_b200.fd_operators import LaplaceA, LaplaceB, Laplace
    from gpawdft_b200.grid_descriptor import GridDescriptor
    peak, _ = measured_peak()
    res = {}

    def timeit(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    a0 = 96 * 0.18 / 0.52917721
    cell = [(0, a0 / 2, a0 / 2), (a0 / 2, 0, a0 / 2), (a0 / 2, a0 / 2, 0)]
    gd = GridDescriptor((96,) * 3, cell, 1)
    ph = np.exp(2j * np.pi * gd.sdisp_cd *
                np.array([0.1, -0.2, 0.3])[:, None])
    NB = 64
    g = torch.Generator(device='cuda').manual_seed(3)
    a = torch.randn((NB, 96, 96, 96), dtype=torch.complex128, device='cuda',
                    generator=g)
    o = torch.empty_like(a)
    op = Laplace(gd, -0.5, 3, complex)
    t = timeit(lambda: op.apply(a, o, ph), args.steps)
    gbs = 2 * a.numel() * 16 / t / 1e9
    res['guc_fcc_nn3_c128'] = {'ms': t * 1e3, 'GB/s': gbs, 'frac': gbs / peak,
                               'points': int(op.npoints), 'bands': NB}
    del a, o
    torch.cuda.empty_cache()
    gdz = GridDescriptor((128,) * 3, (128 * 0.2 / 0.52917721,) * 3, 0)
    b = torch.randn((16, 127, 127, 127), dtype=torch.float64, device='cuda',
                    generator=g)
    ob = torch.empty_like(b)
    for nm, opz in (('mehrstellen_A_f64', LaplaceA(gdz, 0.25 / np.pi)),
                    ('mehrstellen_B_f64', LaplaceB(gdz))):
        t = timeit(lambda: opz.apply(b, ob), args.steps)
        gbs = 2 * b.numel() * 8 / t / 1e9
        res[nm] = {'ms': t * 1e3, 'GB/s': gbs, 'frac': gbs / peak,
                   'points': int(opz.npoints), 'grids': 16}
    del b, ob
    # the same on 127 x 127 x 128 grids: 16-byte rows, as the multigrid
    # engine pads its levels, so the planes are staged by TMA
    gdp = GridDescriptor((128, 128, 129), (128 * 0.2 / 0.52917721,) * 3, 0)
    b = torch.randn((16, 127, 127, 128), dtype=torch.float64, device='cuda',
                    generator=g)
    ob = torch.empty_like(b)
    opz = LaplaceA(gdp, 0.25 / np.pi)
    t = timeit(lambda: opz.apply(b, ob), args.steps)
    gbs = 2 * b.numel() * 8 / t / 1e9
    res['mehrstellen_A_f64_16B_rows'] = {'ms': t * 1e3, 'GB/s': gbs,
                                         'frac': gbs / peak, 'points': 19,
                                         'grids': 16, 'shape': [127, 127, 128]}
    line = {'metric': 'general_stencil_GBps', 'value':
            res['guc_fcc_nn3_c128']['GB/s'], 'unit': 'GB/s',
            'higher_is_better': True, 'n_gpus': 1, 'steps': args.steps,
            'dtype': 'c128', 'data': 'synthetic', 'peak_GBps': peak,
            'config': {'workload': 'GUC nn=3 fcc 64 x 96^3 complex128; '
                                   'Mehrstellen 16 x 127^3 float64 (and '
                                   '16 x 127^2 x 128)'},
            'ops': res}
    return line


def run_uneven(args):
    print(json.dumps(uneven_line(args)), flush=True)


def uneven_line(args):
    """512 independent solves, cubic N_c log-uniform in [32, 128] rounded to
    multiples of 8 (seed 5), each density 4-32 neutral Gaussians (h = 0.2 A),
    relative residual 1e-10, float32 inner / float64 outer.  Solves of one
    size form one batched engine (its stencil variants autotuned); all the
    engines' convergence loops run on the device in ONE graph launch
    (gpw_poisson_solve_many), as concurrent branches.  Reports solves/s and
    the p50/p99 per-solve latency (device time from the launch to the end of
    the iteration in which the solve converged)."""
    import torch
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver, solve_many
    from gpawdft_b200.workloads import gaussian_density
    rng = np.random.default_rng(5)
    NS = 512
    Ns = np.exp(rng.uniform(np.log(32), np.log(128), NS))
    Ns = (np.round(Ns / 8) * 8).astype(int)
    ngs = rng.integers(4, 33, NS)
    groups = {}
    for i, (N, ng) in enumerate(zip(Ns, ngs)):
        groups.setdefault(int(N), []).append((i, int(ng)))
    solvers, phis, rhos, epss, sizes = [], [], [], [], []
    for N, members in sorted(groups.items()):
        rl, L = [], None
        for i, ng in members:
            r, L = gaussian_density(N, 0.2, ng, 5000 + i)
            rl.append(r)
        gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
        ps = PoissonSolver(nn=3, relax='J', maxiter=1000,
                           precision=args.precision, batch=len(rl))
        ps.set_grid_descriptor(gd)
        ps.initialize()
        solvers.append(ps)
        rhos.append(torch.from_numpy(np.array(rl)).cuda())
        phis.append(torch.zeros_like(rhos[-1]))
        epss.append([eps_for(r, gd.dv) for r in rl])
        sizes.append((N, len(rl)))

    def step():
        for p in phis:
            p.zero_()
        return solve_many(solvers, phis, rhos, epss)

    for _ in range(max(3, args.warmup)):
        nits = step()
    torch.cuda.synchronize()
    e0, e1 = _events()
    ts, lats = [], []
    e0.record()
    for _ in range(args.steps):
        s0, s1 = _events()
        s0.record()
        nits = step()
        s1.record()
        torch.cuda.synchronize()
        ts.append(s0.elapsed_time(s1) / 1e3)
        for ps, (N, nb) in zip(solvers, sizes):
            lats.extend(ps.last_latency(nb) / 1e3)
    e1.record()
    torch.cuda.synchronize()
    T = e0.elapsed_time(e1) / 1e3 / args.steps
    line = {'metric': 'batched_uneven_poisson_solves_per_s', 'value': NS / T,
            'unit': 'solves/s', 'higher_is_better': True, 'n_gpus': 1,
            'steps': args.steps, 'warmup': args.warmup,
            'dtype': 'f32+f64' if args.precision == 'fp32' else 'f64',
            'data': 'synthetic',
            'config': {'workload': '512 solves, N_c log-uniform 32-128 (x8), '
                                   '4-32 Gaussians, rel 1e-10, %s, one graph '
                                   'launch' % args.precision,
                       'sizes': {str(N): nb for N, nb in sizes}},
            'p50_latency_s': float(np.percentile(lats, 50)),
            'p99_latency_s': float(np.percentile(lats, 99)),
            'ms_per_step': 1e3 * T,
            'step_ms_min': 1e3 * min(ts),
            'vcycles_mean': float(np.mean(np.concatenate(nits)))}
    del solvers, phis, rhos
    return line


def run_learned(args):
    """Learned warm start at N_c = 128 (127^3, h = 0.2 A): the U-Net is
    trained on `--pairs` (default 20000) fresh (density, potential) pairs --
    densities of 8-64 neutral Gaussians with widths log-uniform in 0.3-2.0 A
    generated on the device, potentials from the float32 multigrid to
    relative residual 1e-6 -- then, on held-out densities (batch of 16):
    learned + float32 solves/s to relative residual 1e-10 (network
    inference, judged first iteration and the rest of the multigrid solve
    inside the timed region) vs the plain float64 method and the float32
    form from a zero start; V-cycles saved; held-out potential error."""
    import torch
    from gpawdft_b200 import blas, learned
    B = 16
    net = learned.PoissonUNet(seed=0)
    t0 = time.time()
    hist = learned.train(net, pairs=args.pairs, batch=4, N_c=128, lr=1e-3,
                         seed=6, log_every=500, logger=None)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    if args.save_weights:
        net.save(args.save_weights)
    sampler = learned.DensitySampler(N_c=128, seed=7)   # held out
    rho = sampler.sample(B)
    ps32 = learned.make_solver(128, batch=B, precision='fp32')
    ps64 = learned.make_solver(128, batch=B, precision='fp64')
    eps = learned.rel_eps(rho, ps32.gd.dv, 1e-10)
    ref = torch.zeros_like(rho)
    ps64.solve_batch(ref, rho, eps=eps)   # reference potentials
    phi = torch.zeros_like(rho)

    def timed(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        out = None
        for _ in range(reps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps, out

    def plain64():
        phi.zero_()
        return ps64.solve_batch(phi, rho, eps=eps)

    def zero32():
        phi.zero_()
        return ps32.solve_batch(phi, rho, eps=eps)

    def learned32():
        phi0, used, k = learned.warm_start(net, ps32, rho)
        n = ps32.solve_batch(phi0, rho, eps=eps) + k
        phi.copy_(phi0)
        return n, used

    t64, n64 = timed(plain64, args.steps)
    t32, n32 = timed(zero32, args.steps)
    tl, (nl, used) = timed(learned32, args.steps)
    d = phi - ref
    final_err = np.sqrt(blas.vector_dots(d, d, B) /
                        blas.vector_dots(ref, ref, B))
    pred = net.predict(rho)
    d = pred - ref
    pred_err = np.sqrt(blas.vector_dots(d, d, B) /
                       blas.vector_dots(ref, ref, B))
    # inference alone (pack + forward + unpack)
    t_inf, _ = timed(lambda: net.predict(rho), args.steps)
    line = {'metric': 'poisson_solves_per_s_128^3_rel1e-10_learned_fp32',
            'value': B / tl, 'unit': 'solves/s', 'higher_is_better': True,
            'n_gpus': 1, 'steps': args.steps, 'warmup': 2,
            'dtype': 'bf16 net + f32/f64 multigrid', 'data': 'synthetic',
            'config': {'workload': 'learned warm start, N_c=128 (127^3), '
                                   'U-Net 16/32/64/64, %d training pairs, '
                                   'held-out batch %d' % (args.pairs, B)},
            'plain_fp64': {'value': B / t64, 'vcycles_mean':
                           float(np.mean(n64))},
            'fp32_zero_start': {'value': B / t32, 'vcycles_mean':
                                float(np.mean(n32))},
            'learned_fp32': {'value': B / tl, 'vcycles_mean':
                             float(np.mean(nl)), 'guess_kept':
                             int(np.sum(used))},
            'speedup_vs_plain_fp64': t64 / tl,
            'vcycles_saved_vs_fp32_zero_start': float(np.mean(n32) -
                                                      np.mean(nl)),
            'heldout_prediction_rel_error': [float(x) for x in pred_err],
            'final_potential_rel_error_vs_fp64': float(final_err.max()),
            'inference_ms_batch': 1e3 * t_inf,
            'train_s': t_train, 'train_loss_history': hist[-5:]}
    print(json.dumps(line), flush=True)


def run_bands(args):
    print(json.dumps(bands_line(args)), flush=True)


def bands_line(args):
    """256 complex Bloch bands on a 96^3 periodic grid (h = 0.18 A, random k,
    phase-wrapped halos): Laplace nn=3 (scale -1/2), the same kinetic
    operator fused with a local potential, Gradient x/y/z n=3,
    restriction / interpolation nn=3 96^3 <-> 48^3, complex128 and complex64.
    GB/s of algorithmic bytes (input read once + output written once)."""
    import torch
    from gpawdft_b200.fd_operators import Gradient, Laplace
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.transformers import Transformer
    h = 0.18 / 0.52917721
    gd = GridDescriptor((96,) * 3, (96 * h,) * 3, 1)
    gc = gd.coarsen()
    k = np.random.default_rng(2).uniform(-0.5, 0.5, 3)
    ph = np.exp(2j * np.pi * gd.sdisp_cd * k[:, None])
    peak, _ = measured_peak()
    NB = args.batch if args.batch != 16 else 256
    res = {}

    def timeit(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    for dt, tdt in ((complex, torch.complex128), (np.complex64, torch.complex64)):
        g = torch.Generator(device='cuda').manual_seed(3)
        a = torch.randn((NB, 96, 96, 96), dtype=tdt, device='cuda', generator=g)
        o = torch.empty_like(a)
        es = a.element_size()
        name = 'c128' if tdt == torch.complex128 else 'c64'
        ops = [('laplace', Laplace(gd, -0.5, 3, dt))] + \
            [('grad%s' % 'xyz'[v], Gradient(gd, v, 1.0, 3, dt)) for v in range(3)]
        for nm, op in ops:
            t = timeit(lambda: op.apply(a, o, ph), args.steps)
            gbs = 2 * a.numel() * es / t / 1e9
            res['%s_%s' % (name, nm)] = {'ms': t * 1e3, 'GB/s': gbs,
                                         'frac': gbs / peak}
        # kinetic + local potential in one pass (gpaw/wavefunctions/fd.py:
        # 77-80): every band read once and written once, the potential
        # (one grid) read once
        vt = torch.randn((96, 96, 96), device='cuda', generator=g,
                         dtype=torch.float64 if name == 'c128'
                         else torch.float32)
        kin = ops[0][1]
        t = timeit(lambda: kin.apply_potential(a, o, vt, ph), args.steps)
        gbs = (2 * a.numel() * es + vt.numel() * vt.element_size()) / t / 1e9
        res['%s_kinetic_potential' % name] = {
            'ms': t * 1e3, 'GB/s': gbs, 'frac': gbs / peak,
            'vs_laplace_alone': t * 1e3 / res['%s_laplace' % name]['ms']}
        del o, vt
        R = Transformer(gd, gc, 3, dt)
        Ip = Transformer(gc, gd, 3, dt)
        c = R.apply(a, None, ph)
        for nm, fn in (('restrict', lambda: R.apply(a, c, ph)),
                       ('interpolate', lambda: Ip.apply(c, a, ph))):
            t = timeit(fn, args.steps)
            gbs = (a.numel() + c.numel()) * es / t / 1e9
            res['%s_%s' % (name, nm)] = {'ms': t * 1e3, 'GB/s': gbs,
                                         'frac': gbs / peak}
        del a, c
        torch.cuda.empty_cache()
    # eigensolver preconditioner (gpaw/preconditioner.py:34-60): a block of
    # 32 complex128 residuals, the caller's nn=3 kinetic operator, the same
    # Bloch phases; its three grids and nine launches per band are timed
    # whole, so the line reports time, not a roofline fraction
    from gpawdft_b200.preconditioner import Preconditioner
    nbp = min(NB, 32)
    g = torch.Generator(device='cuda').manual_seed(4)
    r = torch.randn((nbp, 96, 96, 96), dtype=torch.complex128, device='cuda', generator=g)
    P = Preconditioner(gd, Laplace(gd, -0.5, 3, complex), complex, block=nbp)
    t = timeit(lambda: P(r, ph), args.steps)
    res['c128_preconditioner'] = {'ms': t * 1e3, 'bands_per_s': nbp / t, 'block': nbp}
    del r, P
    torch.cuda.empty_cache()
    line = {'metric': 'band_stencil_GBps_256x96^3_bloch', 'value':
            res['c128_laplace']['GB/s'], 'unit': 'GB/s',
            'higher_is_better': True, 'n_gpus': 1, 'steps': args.steps,
            'dtype': 'c128', 'data': 'synthetic', 'peak_GBps': peak,
            'config': {'workload': '%d complex Bloch bands, 96^3 periodic' % NB},
            'ops': res}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--batch', type=int, default=16)
    ap.add_argument('--precision', default='fp32', choices=['fp64', 'fp32'])
    ap.add_argument('--workload', default='poisson128',
                    choices=['poisson128', 'mixed192', 'uneven512', 'bands96',
                             'learned128', 'general'])
    ap.add_argument('--pairs', type=int, default=20000,
                    help='learned128: training pairs')
    ap.add_argument('--save-weights', default=None,
                    help='learned128: save the trained network (.npz)')
    ap.add_argument('--host-loop', action='store_true',
                    help='replay the iteration graph from the host instead of '
                         'the device-side loop (for per-kernel profiling)')
    ap.add_argument('--no-cpu', action='store_true',
                    help='skip the cpu_baseline sample')
    ap.add_argument('--no-secondary', action='store_true',
                    help='poisson128: skip the secondary configurations '
                         '(band stencils, general stencils, 191^3 mixed '
                         'precision) measured after the headline')
    args = ap.parse_args()
    if args.workload != 'poisson128':
        {'mixed192': run_mixed192, 'uneven512': run_uneven,
         'bands96': run_bands, 'learned128': run_learned,
         'general': run_general}[args.workload](args)
        return
    args.warmup = max(args.warmup, 3) if args.impl == 'ours' else args.warmup
    if 'WORLD_SIZE' not in os.environ and args.gpus > 1:
        # one process per GPU: relaunch this command under torchrun
        import socket
        so = socket.socket()
        so.bind(('127.0.0.1', 0))
        port = so.getsockname()[1]
        so.close()
        cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1',
               '--nproc-per-node', str(args.gpus), '--master-addr',
               '127.0.0.1', '--master-port', str(port),
               os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    if world != args.gpus:
        print('bench.py: --gpus %d but WORLD_SIZE=%d; launch one process per '
              'GPU with --nproc-per-node %d' % (args.gpus, world, args.gpus),
              file=sys.stderr)
        sys.exit(2)
    rank = int(os.environ.get('RANK', '0'))
    dist = None
    if world > 1 and args.impl == 'ours':
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
        tdist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
        dist = tdist
    if args.impl == 'reference':
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
