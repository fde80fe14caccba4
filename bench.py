#!/usr/bin/env python
"""FDTD throughput benchmark of the B200 engine (one JSON line on rank 0).

Workload (opensol_b200/workloads.py, roofline_2d): the 8192 x 8192 E_z grid incl. 20 CPML cells per side, dx = 20 nm,
2000 seeded dielectric cylinders, a 1550 nm Gaussian line source and four 16-frequency flux lines.  One bench step
is one whole simulation of 10,000 Yee steps (fields, psi and spectra reset first), so

    value = cell-updates per second = 8192^2 x 10,000 x steps x ranks / device time      [Gcell-updates/s]

measured with CUDA events on the stream the engine launches on, max over ranks.  The fields (3 x 268 MB) exceed the
126 MB L2, so no flush is needed between steps.  e2e = the same metric through the public API from host inputs:
Simulation built and painted on the host beforehand, then per step the upload of the materials (pinned host memory),
the 10,000 steps and the read-back of all four flux spectra.

--impl reference times the CPU restatement of open_sol's step (the oracle, C + OpenMP on every host core) on a
bounded sample of the same grid.  With torchrun (N > 1) each rank runs an independent replica (the path does not
shard; no collective touches the data).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL_UPDATE = 28          # 3 float32 fields read + written, one float32 material word read
HZ2_BYTES_PER_CELL_UPDATE = 16      # H_z two steps per launch: 5 float32 arrays read, 3 written, per two steps
SIM_STEPS = 10_000
CPU_SAMPLE_STEPS = 24


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=5)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    p.add_argument('--sim-steps', type=int, default=SIM_STEPS)
    p.add_argument('--grid', type=int, default=8192, help='total cells per side (8192 = the benchmark workload; '
                   'smaller grids are profiling cases of the same kernels)')
    p.add_argument('--grid3d', type=int, default=512, help='em3d: total cells per side (512 = the benchmark '
                   'workload; smaller grids scale the sphere count with the volume, for profiling)')
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--no-e2e', action='store_true')
    p.add_argument('--no-replay', action='store_true', help='skip the reference-kernel replay leg')
    p.add_argument('--no-secondary', action='store_true',
                   help='skip the H_z, 3D, serving and adjoint figures that follow the headline')
    p.add_argument('--variant', type=int, default=1, help='1: temporally blocked kernels (default), 0: per step')
    p.add_argument('--steps-per-launch', type=int, default=3)
    p.add_argument('--tile-rows', type=int, default=0, help='rows per interior tile (0: autotune)')
    p.add_argument('--workload', default='roofline_2d',
                   choices=['roofline_2d', 'hz2d', 'em3d', 'serving', 'adjoint'],
                   help='roofline_2d: the headline 8192^2 2D run; hz2d: the same grid in the H_z polarisation; '
                        'em3d: the 512^3 3D run; serving: the batched job stream against one-at-a-time runs; '
                        'adjoint: gradient cost against one forward run')
    p.add_argument('--jobs', type=int, default=64, help='serving: jobs of the request stream')
    p.add_argument('--form3d', type=int, default=3, choices=[0, 1, 2, 3],
                   help='em3d: step form (0 two in-place kernels, 1 fused on two field sets, 2 fused with staged '
                        'planes, 3 lean staged fused pass); results are the same bits')
    p.add_argument('--x-chunk', type=int, default=0, help='em3d: x planes per block (0: the engine\'s choice)')
    p.add_argument('--hz-steps', type=int, default=2, choices=[1, 2], help='hz2d: Yee steps per interior launch')
    p.add_argument('--fused-config', type=int, default=-1,
                   help="em3d: launch shape of the fused forms (0..4; -1: the form's default)")
    return p.parse_args()


def dist_env():
    from opensol_b200.replicas import replica_env
    return replica_env()


def measured_peak_hbm():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix='.csv')

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.QUERY}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=open(self.path, 'w'), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(',')]
                    if len(parts) >= 9:
                        rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled']}
        sm = [float(r[1]) for r in rows if r[1].replace('.', '').isdigit()]
        sm_max = [float(r[2]) for r in rows if r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({name for r in rows for name, v in zip(names, r[5:9]) if v.lower() == 'active'})
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': max(sm_max) if sm_max else None,
                'reasons': reasons, 'samples': len(rows)}


def build_sim(device, grid=8192, amplitude=1.0, pinned=False):
    import opensol_b200 as ob
    from opensol_b200 import workloads
    sim = ob.Simulation(**workloads.roofline_2d_sim_args(total_cells=grid), verbose=False, device=device,
                        pinned_host=pinned)
    monitors = workloads.apply(sim, workloads.roofline_2d_ops(total_cells=grid, amplitude=amplitude))
    return sim, monitors


def cpu_baseline(sample_steps=CPU_SAMPLE_STEPS):
    """The oracle (CPU restatement of open_sol's step, C + OpenMP) on the same 8192^2 workload: a bounded sample of
    sample_steps Yee steps after a 2-step warm-up."""
    from oracle.fdtd2d import OracleEz2D
    from opensol_b200 import workloads
    subprocess.run(['make', '-s', '-C', os.path.join(ROOT, 'oracle')], check=True)
    o = OracleEz2D(**workloads.roofline_2d_sim_args())
    workloads.apply(o, workloads.roofline_2d_ops())
    o.finalize()
    o.run(n_steps=2)
    t0 = time.perf_counter()
    o.run(n_steps=sample_steps)
    wall = time.perf_counter() - t0
    cells = o.domain.nx * o.domain.ny
    return {'value': cells * sample_steps / wall / 1e9, 'unit': 'Gcell-updates/s',
            'cores': os.cpu_count(), 'kind': 'port',
            'sample': f'{sample_steps} Yee steps of the 8192x8192 roofline grid after 2 warm-up steps, '
                      f'C restatement with OpenMP on {os.cpu_count()} threads',
            'wall_s': wall}


def gpu_reference_replay(args, device, value, warmup_steps=50, timed_steps=2000):
    """open_sol's own GPU step on the same workload: the reference-kernel replay (its update_h / update_e RawKernels
    compiled unchanged for sm_100a, the CPML, source and DFT launches of its step sequence, H and E blocks replayed
    as CUDA graphs), timed with CUDA events over timed_steps steps after warmup_steps; ratio = this engine's value
    over the replay's."""
    from oracle import replay_ez2d
    ok, why = replay_ez2d.available()
    if not ok:
        return {'unavailable': why}
    from oracle.fdtd2d import OracleEz2D
    from opensol_b200 import workloads
    o = OracleEz2D(**workloads.roofline_2d_sim_args(total_cells=args.grid))
    workloads.apply(o, workloads.roofline_2d_ops(total_cells=args.grid))
    o.finalize()
    replay = replay_ez2d.ReferenceReplayEz2D(o, device)
    try:
        replay.run(warmup_steps)
        replay.reset()
        ms = replay.run(timed_steps)
    finally:
        replay.close()
    rate = o.domain.nx * o.domain.ny * timed_steps / (ms / 1e3) / 1e9
    return {'value': rate, 'unit': 'Gcell-updates/s', 'steps': timed_steps, 'ms': ms, 'ratio': value / rate,
            'kind': 'reference-kernel replay',
            'what': "open_sol's update_h_kernel / update_e_kernel (fdtd_ez_2d_kernels.py:23-122) compiled unchanged "
                    'for sm_100a with (32, 8, 1) blocks, its CPML psi / source / DFT elementwise launches restated, '
                    'the H and E blocks replayed as CUDA graphs per step as its _fixed_block does'}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle.fdtd2d import OracleEz2D
    from opensol_b200 import workloads
    subprocess.run(['make', '-s', '-C', os.path.join(ROOT, 'oracle')], check=True)
    o = OracleEz2D(**workloads.roofline_2d_sim_args())
    workloads.apply(o, workloads.roofline_2d_ops())
    o.finalize()
    cells = o.domain.nx * o.domain.ny
    sample = 10
    for _ in range(args.warmup):
        o.run(n_steps=sample)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.run(n_steps=sample)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = cells * sample * args.steps / total / 1e9
    line = {
        'impl': 'reference', 'metric': 'FDTD Gcell-updates/s', 'value': value, 'unit': 'Gcell-updates/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total / args.steps * 1e3,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': config_block(args, 'replicas' if world > 1 else 'single'),
        'cpu_baseline': {'value': value, 'unit': 'Gcell-updates/s', 'cores': os.cpu_count(), 'kind': 'port',
                         'sample': f'{sample} Yee steps of the 8192x8192 roofline grid per bench step (oracle: C '
                                   f'restatement of open_sol\'s CPU step, OpenMP on {os.cpu_count()} threads)'},
        'e2e': {'value': value, 'unit': 'Gcell-updates/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def config_block(args, parallelism):
    g = getattr(args, 'grid', 8192)
    return {'workload': f'roofline_2d: 2D E_z FDTD, {g}x{g} total grid incl. 20 CPML cells/side, dx 20 nm, 2000 '
                        'seeded cylinders eps_r U(2,12), 1550 nm Gaussian line source, 4 x 16-frequency flux lines, '
                        f'{args.sim_steps} Yee steps per bench step',
            'grid': [g, g], 'sim_steps': args.sim_steps, 'parallelism': parallelism,
            'l2': 'inputs larger than L2 (fields 3 x 268 MB), no flush'}


def run_b200(args):
    import torch
    from opensol_b200.replicas import ReplicaGroup
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    # independent replicas: the group only brackets the timed region and takes the max over ranks
    group = ReplicaGroup('nccl', timeout_s=300)
    barrier, reduce_max = group.barrier, group.reduce_max

    sim, monitors = build_sim(local, args.grid)
    sim.em.engine.configure(args.variant, args.steps_per_launch, args.tile_rows or 128)
    sim.em.finalize()
    engine = sim.em.engine
    autotuned = None
    if args.variant == 1 and not args.tile_rows:
        autotuned = engine.autotune()
        args.tile_rows = engine.tile_rows
    # a stream of its own (torch's default stream is handle 0, which os_fdtd*_set_stream reads as "the engine's own
    # stream"): the engine launches on it and the timing events are recorded on it
    stream = torch.cuda.Stream()
    engine.set_stream(stream.cuda_stream)
    cells = engine.nx * engine.ny
    engine.reset()
    tables = engine.chunk_tables(args.sim_steps)
    for _ in range(args.warmup):
        engine.reset()
        engine.advance(args.sim_steps, tables)
    torch.cuda.synchronize()

    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            engine.reset()
            engine.advance(args.sim_steps, tables)
            launches += engine.launch_count()
        stop.record(stream)
        torch.cuda.synchronize()
    barrier()
    device_ms = reduce_max(start.elapsed_time(stop))
    value = group.whole_job_rate(cells * args.sim_steps * args.steps, device_ms / 1e3) / 1e9
    flux = [m.flux() for m in monitors]
    if args.sim_steps >= 2000:   # the pulse reaches the first flux line after ~250 steps
        assert any(float(abs(f).max()) > 0 for f in flux), 'every flux is zero: the run did no work'

    # Dominant kernel: one more run with every launch bracketed by CUDA events on the engine's stream (the frame
    # launches then run ahead of the interior launch instead of beside it, so each pair times one kernel alone and
    # the shares compare with ncu's serialised launch list).
    engine.set_profiling(True)
    engine.reset()
    engine.advance(args.sim_steps, tables)
    times = engine.kernel_times()
    engine.set_profiling(False)
    peak, peak_kind = measured_peak_hbm()
    T = engine.steps_per_launch
    interior_cells, interior_tiles, general_tiles = engine.plan_info(T)
    if engine.variant == 1 and interior_cells:
        name = engine.KERNEL_KINDS[0]
        total_ms, n_launch = times[name]
        units = interior_cells * T                       # cell-updates one full-T launch performs
        launch_ms = reduce_max(total_ms / n_launch)
    else:
        name = engine.KERNEL_KINDS[3] if engine.variant == 0 else engine.KERNEL_KINDS[1]
        total_ms, n_launch = times[name]
        units = cells * (1 if engine.variant == 0 else T)
        launch_ms = reduce_max(total_ms / n_launch)
    # algorithmic bytes of a launch of T steps: the three fields and cb read once and the fields written once per cell
    # (28 B), i.e. 28 / T per cell-update; the one-step figure (28 B per cell-update) is kept beside it
    steps_in_launch = 1 if engine.variant == 0 else T
    bpc = BYTES_PER_CELL_UPDATE / steps_in_launch
    achieved = bpc * units / (launch_ms / 1e3) / 1e9
    roofline = {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                'traffic': None, 'peak_source': f'{peak_kind} hbm_gbs (copy bandwidth)', 'kernel': name,
                'bytes_per_cell_update': bpc, 'cell_updates_per_launch': units,
                'one_step_equivalent_gbs': BYTES_PER_CELL_UPDATE * units / (launch_ms / 1e3) / 1e9,
                'launch_ms': launch_ms, 'launch_timing': 'CUDA events per launch, each kernel alone',
                'steps_per_launch': T,
                'kernel_share': {k: v[0] / sum(t[0] for t in times.values()) for k, v in times.items()}}
    traffic_path = os.path.join(ROOT, 'profiles', 'traffic.json')
    if os.path.exists(traffic_path):
        with open(traffic_path) as f:
            t = json.load(f).get(name)
        if t and t.get('steps_per_launch') == T:
            roofline['traffic'] = t['dram_bytes_per_cell_update'] * units
            roofline['traffic_note'] = t['note']

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, local, world, barrier, reduce_max)

    line = {
        'metric': 'FDTD Gcell-updates/s', 'value': value, 'unit': 'Gcell-updates/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': device_ms / args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': {**config_block(args, 'replicas' if world > 1 else 'single'),
                   'kernel': {'variant': engine.variant, 'steps_per_launch': engine.steps_per_launch,
                              'tile_rows': engine.tile_rows, 'autotuned_ms_per_launch':
                                  None if autotuned is None else autotuned[1]}},
        'roofline': roofline,
        'gpu_launches': launches,
        'clocks': clocks.summary(),
    }
    if e2e is not None:
        line['e2e'] = e2e
    sim.clear()
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.grid == 8192:
        line['cpu_baseline'] = cpu_baseline()
    if rank == 0 and world == 1 and not args.no_replay:
        line['gpu_reference_replay'] = gpu_reference_replay(args, local, value)
    if rank == 0 and world == 1 and not args.no_secondary and args.grid == 8192:
        line['secondary'] = secondary_workloads(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    group.close()


def run_e2e(args, device, world, barrier, reduce_max):
    """Public-API runs from host inputs: per step the pinned host materials are uploaded, the 10,000 steps run and
    the four monitors' spectra come back (flux())."""
    import torch
    n = max(1, min(args.steps, 3))
    sims = [build_sim(device, args.grid, pinned=True) for _ in range(n + 1)]
    for sim, _ in sims:
        sim.em.engine.configure(args.variant, args.steps_per_launch, args.tile_rows)
    h2d = d2h = 0
    sim, mons = sims[0]
    sim.run(n_steps=args.sim_steps, verbose=False, print_every=0)   # warm-up run
    [m.flux() for m in mons]
    sim.clear()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for sim, mons in sims[1:]:
        sim.run(n_steps=args.sim_steps, verbose=False, print_every=0)
        [m.flux() for m in mons]
        h2d = sim.em.engine.h2d_bytes
        d2h = sum(m.n_freqs * m.n_cells * 2 * 16 for m in mons)
        sim.clear()
    torch.cuda.synchronize()
    wall = reduce_max(time.perf_counter() - t0)
    barrier()
    cells = args.grid * args.grid
    return {'value': world * cells * args.sim_steps * n / wall / 1e9, 'unit': 'Gcell-updates/s',
            'h2d_bytes_per_step': int(h2d), 'd2h_bytes_per_step': int(d2h), 'steps': n,
            'timing': 'host wall clock around Simulation.run + flux(), synchronized, max over ranks'}


def run_hz2d(args):
    """The roofline_2d geometry in the H_z polarisation (H_z, E_x, E_y; the same 2000 cylinders, line source and
    four flux lines): cell-updates/s over the total grid, one bench step = one whole simulation of args.sim_steps Yee
    steps from rest, device time with CUDA events on the engine's stream.  Roofline: the 28 algorithmic bytes per
    cell-update (3 fields read + written, one eps word) over the fused step kernel's mean launch time."""
    import torch
    import opensol_b200 as ob
    from opensol_b200 import workloads
    torch.cuda.set_device(0)
    sim = ob.Simulation(**workloads.roofline_2d_sim_args(total_cells=args.grid), polarization='hz', verbose=False)
    monitors = workloads.apply(sim, workloads.roofline_2d_ops(total_cells=args.grid))
    variant = args.variant if args.variant in (0, 1) else 1
    sim.em.engine.configure(variant=variant, steps_per_launch=args.hz_steps, tile_rows=args.tile_rows)
    sim.em.finalize()
    engine = sim.em.engine
    # a stream of its own (torch's default stream is handle 0, which os_fdtd*_set_stream reads as "the engine's own
    # stream"): the engine launches on it and the timing events are recorded on it
    stream = torch.cuda.Stream()
    engine.set_stream(stream.cuda_stream)
    tables = engine.chunk_tables(args.sim_steps)
    for _ in range(args.warmup):
        engine.reset()
        engine.advance(args.sim_steps, tables)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    with ClockSampler(0) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            engine.reset()
            engine.advance(args.sim_steps, tables)
            launches += engine.launch_count()
        stop.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    cells = engine.nx * engine.ny
    value = cells * args.sim_steps * args.steps / (ms / 1e3) / 1e9
    flux = [m.flux() for m in monitors]
    if args.sim_steps >= 2000:
        assert any(float(abs(f).max()) > 0 for f in flux), 'every flux is zero: the run did no work'
    engine.set_profiling(True)
    engine.reset()
    engine.advance(args.sim_steps, tables)
    times = engine.kernel_times()
    engine.set_profiling(False)
    peak, peak_kind = measured_peak_hbm()
    interior_cells, border_cells = engine.hz_plan()
    if engine.variant == 1 and interior_cells:
        name = engine.KERNEL_KINDS[0]
        units = interior_cells * engine.steps_per_launch   # cell-updates of one interior launch
    else:
        name = engine.KERNEL_KINDS[3 if engine.variant == 0 else 1]
        units = cells
    total_ms, n_launch = times[name]
    launch_ms = total_ms / n_launch
    two_step = engine.variant == 1 and interior_cells and engine.steps_per_launch == 2
    # algorithmic bytes per cell-update of the timed kernel: one step reads and writes the three fields and reads one
    # eps word (28 B); the two-step pass reads H_z, E_x, E_y and the stored faces cb_x, cb_y and writes the three
    # fields once per two steps (32 B per cell, 16 B per cell-update)
    bpc = HZ2_BYTES_PER_CELL_UPDATE if two_step else BYTES_PER_CELL_UPDATE
    achieved = bpc * units / (launch_ms / 1e3) / 1e9
    roofline = {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                'traffic': None, 'peak_source': f'{peak_kind} hbm_gbs (copy bandwidth)', 'kernel': name,
                'bytes_per_cell_update': bpc, 'cell_updates_per_launch': units,
                'border_cells': border_cells, 'launch_ms': launch_ms, 'lossless_form': engine.lossless_form(),
                'kernel_share': {k: v[0] / sum(t[0] for t in times.values()) for k, v in times.items()}}
    traffic_path = os.path.join(ROOT, 'profiles', 'traffic.json')
    if two_step:
        roofline['kernel'] = 'hz2d_interior2_kernel (two steps per launch)'
        roofline['one_step_equivalent_gbs'] = BYTES_PER_CELL_UPDATE * units / (launch_ms / 1e3) / 1e9
    if os.path.exists(traffic_path):
        with open(traffic_path) as f:
            t = json.load(f).get('hz2d_interior2_kernel' if two_step else 'hz2d_interior_kernel')
        if t:
            roofline['traffic'] = t['dram_bytes_per_cell_update'] * units
            roofline['traffic_note'] = t['note']
    line = {'metric': 'FDTD Gcell-updates/s (2D H_z)', 'value': value, 'unit': 'Gcell-updates/s', 'n_gpus': 1,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': f'hz2d: 2D H_z FDTD, {args.grid}x{args.grid} total grid incl. 20 CPML cells/side, '
                                   'dx 20 nm, 2000 seeded cylinders eps_r U(2,12), 1550 nm E_y sheet source, '
                                   f'4 x 16-frequency flux lines, {args.sim_steps} Yee steps per bench step',
                       'grid': [args.grid, args.grid], 'sim_steps': args.sim_steps,
                       'kernel': {'variant': engine.variant, 'rows_per_cta': engine.tile_rows,
                                  'steps_per_launch': engine.steps_per_launch},
                       'l2': 'inputs larger than L2 (fields 3 x 268 MB), no flush'},
            'roofline': roofline, 'gpu_launches': launches, 'clocks': clocks.summary()}
    sim.clear()
    if not args.no_cpu_baseline and args.grid == 8192:
        line['cpu_baseline'] = cpu_baseline_hz()
    return line


def cpu_baseline_hz(sample_steps=CPU_SAMPLE_STEPS):
    """The H_z oracle (C + OpenMP restatement of open_sol's H_z step) on the same 8192^2 grid: a bounded sample of
    sample_steps Yee steps after a 2-step warm-up."""
    from oracle.hz2d import OracleHz2D
    from opensol_b200 import workloads
    subprocess.run(['make', '-s', '-C', os.path.join(ROOT, 'oracle')], check=True)
    o = OracleHz2D(**workloads.roofline_2d_sim_args())
    workloads.apply(o, workloads.roofline_2d_ops())
    o.finalize()
    o.run(n_steps=2)
    t0 = time.perf_counter()
    o.run(n_steps=sample_steps)
    wall = time.perf_counter() - t0
    cells = o.domain.nx * o.domain.ny
    return {'value': cells * sample_steps / wall / 1e9, 'unit': 'Gcell-updates/s', 'cores': os.cpu_count(),
            'kind': 'port', 'sample': f'{sample_steps} H_z Yee steps of the 8192x8192 grid after 2 warm-up steps, '
                                      f'C restatement with OpenMP on {os.cpu_count()} threads', 'wall_s': wall}


def run_em3d(args):
    """The 512^3 3D workload (opensol_b200/workloads.py roofline_3d_physics): cell-updates/s over the total grid, one
    bench step = args.sim_steps Yee steps from rest (2000 when left at the 2D default)."""
    import torch
    from opensol_b200 import workloads
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    steps = args.sim_steps if args.sim_steps != SIM_STEPS else workloads.ROOFLINE_3D['steps']
    physics, box = workloads.roofline_3d_physics(total_cells=args.grid3d,
                                                 n_spheres=max(1, int(round(500 * (args.grid3d / 512) ** 3))),
                                                 device=local)
    physics.finalize()
    engine = physics.engine
    engine.set_variant(args.form3d)
    engine.set_fused_config(args.fused_config)
    if args.x_chunk > 0:
        engine.set_x_chunk(args.x_chunk)
    # a stream of its own (torch's default stream is handle 0, which os_fdtd*_set_stream reads as "the engine's own
    # stream"): the engine launches on it and the timing events are recorded on it
    stream = torch.cuda.Stream()
    engine.set_stream(stream.cuda_stream)
    tables = engine.chunk_tables(steps)
    for _ in range(args.warmup):
        engine.reset()
        engine.advance(steps, tables)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            engine.reset()
            engine.advance(steps, tables)
            launches += engine.launch_count()
        stop.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    cells = engine.nx * engine.ny * engine.nz
    value = cells * steps * args.steps / (ms / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    achieved = 52.0 * value
    line = {'metric': 'FDTD Gcell-updates/s (3D)', 'value': value, 'unit': 'Gcell-updates/s', 'n_gpus': 1,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': f'em3d: {engine.nx}^3 total grid incl. 12 CPML cells/face, dx 20 nm, 500 seeded '
                                   'spheres eps_r U(2,12), z dipole 1310 nm at the centre, 8-frequency flux box, '
                                   f'{steps} Yee steps per bench step', 'l2': 'fields 6 x 537 MB, no flush',
                       'step_form': args.form3d, 'fused_config': args.fused_config, 'x_chunk': args.x_chunk},
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s', 'frac': achieved / peak,
                         'traffic': None, 'peak_source': f'{peak_kind} hbm_gbs', 'bytes_per_cell_update': 52,
                         'kernel': 'em3d_lean_kernel + x / y face kernels (whole step)' if engine.interior()[1]
                         and args.form3d == 3 else 'em3d_h_kernel + em3d_e_kernel (whole step)'},
            'gpu_launches': launches, 'clocks': clocks.summary(),
            'flux_box_first': float(box.flux()[0])}
    traffic_path = os.path.join(ROOT, 'profiles', 'traffic.json')
    if os.path.exists(traffic_path):
        with open(traffic_path) as f:
            t = json.load(f).get('em3d_lean_step' if engine.interior()[1] and args.form3d == 3 else 'em3d_step')
        if t:
            line['roofline']['traffic'] = t['dram_bytes_per_cell_update'] * cells   # per step
            line['roofline']['traffic_note'] = t['note']
    return line


def run_serving(args):
    """The serving stream (opensol_b200/serving.py make_job_specs): sims/s of the batched loop with every job queued
    at once, against one-at-a-time runs of the same jobs; p50 / p99 latency with Poisson arrivals at 20 jobs/s."""
    import numpy as np
    import torch
    from opensol_b200 import serving
    torch.cuda.set_device(0)
    specs = serving.make_job_specs(n_jobs=args.jobs, rate=20.0, seed=7)
    work = sum(s.cells() * s.steps for s in specs)
    # warm-up: one untimed pass of the same stream, as a serving process that has run for a while: the kernels are
    # loaded and the engines' device-memory pool holds blocks of every size the stream needs (both arms take their
    # arrays from it)
    loop = serving.ServingLoop(max_active=48, chunk_steps=512)
    loop.run(specs, realtime=False)
    loop.close(trim=False)
    loop = serving.ServingLoop(max_active=48, chunk_steps=512)
    t0 = time.perf_counter()
    batched = {r.job_id: r for r in loop.run(specs, realtime=False)}
    t_batch = time.perf_counter() - t0
    loop.close(trim=False)
    t0 = time.perf_counter()
    alone = {s.job_id: serving.run_alone(s)[0] for s in specs}
    t_alone = time.perf_counter() - t0
    same = all(np.array_equal(a, b) for j, r in batched.items() for a, b in zip(r.fluxes, alone[j]))
    loop = serving.ServingLoop(max_active=48, chunk_steps=512)
    t0 = time.perf_counter()
    realtime = loop.run(specs, realtime=True)
    t_rt = time.perf_counter() - t0
    loop.close()
    p50, p99 = serving.latency_percentiles(realtime)
    line = {'metric': 'batched sims/s', 'value': len(specs) / t_batch, 'unit': 'sims/s', 'n_gpus': 1,
            'steps': 1, 'warmup': 1, 'ms_per_step': t_batch * 1e3, 'higher_is_better': True, 'scaling': 'strong',
            'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': f'serving: {len(specs)} jobs, square windows U{{256..2048}} + 15 CPML cells/side, '
                                   '1-40 rectangles eps_r U(1,12), line source U(1000,1600) nm, U(2000,20000) steps, '
                                   'two 4-frequency flux lines; Poisson 20 jobs/s for the latency run',
                       'max_active': 48, 'chunk_steps': 512, 'memory_budget_gb': 120,
                       'steps_per_launch': {'batched': 3, 'one_at_a_time': 3},
                       'admission': 'all jobs queued at once: largest (cells x steps) first, at most 16 set up per '
                                    'tick; latency run: arrival order',
                       'warm_up': 'one untimed pass of the same stream (kernels loaded, device-memory pool warm for '
                                  'both arms)',
                       'tile_rows': 'chosen per call from the active jobs (batched) / per grid (one at a time)'},
            'one_at_a_time_sims_per_s': len(specs) / t_alone, 'speedup_vs_one_at_a_time': t_alone / t_batch,
            'cell_updates_per_s_batched': work / t_batch, 'fluxes_equal_alone_and_batched': bool(same),
            'latency_p50_s': p50, 'latency_p99_s': p99, 'realtime_makespan_s': t_rt,
            'timing': 'host wall clock (synchronised), one process, one B200'}
    return line


def run_adjoint(args):
    """The adjoint workload (opensol_b200/workloads.py adjoint_2d_problem): the cost of one gradient (forward with
    checkpoints + backward) over the cost of one plain forward of the same problem through the public API
    (Simulation.run of all its steps from rest + flux()).  Both are host wall clock around synchronized calls; the
    device time of each (CUDA events on the engine's stream) is reported beside it."""
    import numpy as np
    import torch
    from opensol_b200 import workloads
    from opensol_b200.adjoint import FluxAdjoint2D
    torch.cuda.set_device(0)
    spec = workloads.ADJOINT_2D
    sim, monitor, box, eps = workloads.adjoint_2d_problem()
    engine = sim.em.engine
    stream = torch.cuda.Stream()
    engine.set_stream(stream.cuda_stream)
    adj = FluxAdjoint2D(sim, monitor, 0, box, spec['steps'], checkpoint_every=spec['checkpoint_every'])
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def plain_forward():
        engine.reset()
        sim.run(n_steps=spec['steps'], verbose=False, print_every=0)
        return float(monitor.flux()[0])

    def gradient():
        J = adj.forward()
        return J, adj.backward()

    plain_forward()
    gradient()
    torch.cuda.synchronize()
    plain, plain_dev, grad_wall, grad_dev, fw_wall = [], [], [], [], []
    with ClockSampler(0) as clocks:
        for _ in range(max(3, args.steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            start.record(stream)
            J_plain = plain_forward()
            stop.record(stream)
            torch.cuda.synchronize()
            plain.append(time.perf_counter() - t0)
            plain_dev.append(start.elapsed_time(stop) / 1e3)
            t0 = time.perf_counter()
            start.record(stream)
            J = adj.forward()
            engine.synchronize()
            t1 = time.perf_counter()
            grad = adj.backward()
            stop.record(stream)
            torch.cuda.synchronize()
            grad_wall.append(time.perf_counter() - t0)
            fw_wall.append(t1 - t0)
            grad_dev.append(start.elapsed_time(stop) / 1e3)
    assert J == J_plain, 'the checkpointed forward differs from the plain run'
    p, g = statistics.median(plain), statistics.median(grad_wall)
    cells = engine.nx * engine.ny
    line = {'metric': 'adjoint gradient cost / plain forward cost', 'value': g / p, 'unit': 'x',
            'n_gpus': 1, 'steps': len(plain), 'warmup': 1, 'ms_per_step': g * 1e3, 'higher_is_better': False,
            'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': f'adjoint: {engine.nx}^2 total grid incl. 20 CPML cells/side, dx 20 nm, '
                                   f'{box[1] - box[0]}x{box[3] - box[2]} design box eps_r U(1,12.1), 1550 nm line '
                                   f'source, flux objective at 1550 nm after {spec["steps"]} steps, checkpoints '
                                   f'every {spec["checkpoint_every"]}'},
            'plain_forward_s': p, 'gradient_s': g, 'checkpointed_forward_s': statistics.median(fw_wall),
            'plain_forward_device_s': statistics.median(plain_dev), 'gradient_device_s': statistics.median(grad_dev),
            'device_ratio': statistics.median(grad_dev) / statistics.median(plain_dev),
            'plain_forward_gcell_updates_per_s': cells * spec['steps'] / p / 1e9,
            'objective': J, 'grad_abs_max': float(np.abs(grad).max()), 'clocks': clocks.summary(),
            'timing': 'host wall clock around synchronized calls (median of the repeats); device time by CUDA events '
                      'on the engine stream'}
    return line


def secondary_workloads(args):
    """The other benchmark configurations, each run once in this process after the headline and reported inside its
    JSON line with its own clock record: the same grid in the H_z polarisation, the 512^3 3D run, the serving stream
    against one-at-a-time runs, and the adjoint gradient against a plain forward."""
    import copy
    import torch
    out = {}
    # tile_rows 0: each engine picks its own (the headline run stored the E_z autotuner's choice in args)
    plans = [('hz2d', run_hz2d, {'steps': 2, 'warmup': 1, 'sim_steps': SIM_STEPS, 'no_cpu_baseline': True,
                                 'tile_rows': 0}),
             ('em3d', run_em3d, {'steps': 1, 'warmup': 1, 'sim_steps': SIM_STEPS}),
             ('adjoint', run_adjoint, {'steps': 3, 'warmup': 1}),
             ('serving', run_serving, {'jobs': 32})]
    for name, fn, overrides in plans:
        a = copy.copy(args)
        for key, value in overrides.items():
            setattr(a, key, value)
        try:
            line = fn(a)
            out[name] = {k: v for k, v in line.items() if k not in ('n_gpus', 'data', 'vs_baseline')}
        except Exception as error:   # a failing secondary figure is reported, the headline stands
            out[name] = {'error': f'{type(error).__name__}: {error}'}
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return out


def main():
    args = parse_args()
    if args.impl == 'reference':
        run_reference(args)
        return
    if args.workload == 'roofline_2d':
        run_b200(args)
        return
    fn = {'em3d': run_em3d, 'hz2d': run_hz2d, 'serving': run_serving, 'adjoint': run_adjoint}[args.workload]
    print(json.dumps(fn(args)), flush=True)


if __name__ == '__main__':
    main()
