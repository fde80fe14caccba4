"""Continuous-batching serving loop for 2D FDTD jobs on one B200.

Jobs (ordinary Simulation objects of the public API) are admitted as they arrive, while the device-memory budget and
the slot count allow; their fields, coefficients and monitor sums stay resident on the device until they finish.  All
active jobs advance together: each tick is one call of os_fdtd2d_batch_advance, in which every T steps one border
launch and one interior launch cover the tiles of every active job and one launch folds all their DFT samples.  A job
that finishes is read back (its fluxes), released, and its slot goes to the next arrival; new jobs are built on the
host while the device runs the tick already queued.  Each job's arithmetic is exactly that of a run alone, so its
results are bit-identical alone and in the mix.

The request stream of the serving benchmark (make_job_specs): square windows of side U{256..2048} cells at dx = 20 nm
with 15 CPML cells per side, 1-40 axis-aligned rectangles of eps_r U(1, 12), one Gaussian line source at U(1000,
1600) nm, U(2000, 20000) steps, two 4-frequency flux lines, Poisson arrivals.
"""
from __future__ import annotations

import ctypes
import math
import time
import weakref
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _native
from .constants import DTYPE


class BatchAdvancer:
    """os_fdtd2d_batch_advance over a list of FDTDEngine2D_Ez engines (all on this batch's stream)."""

    def __init__(self, device=0):
        self.device = int(device)
        out = ctypes.c_void_p()
        _native.check(_native.load().os_fdtd2d_batch_create(self.device, ctypes.byref(out)))
        self._handle = out
        stream = ctypes.c_void_p()
        _native.check(_native.load().os_fdtd2d_batch_stream(self._handle, ctypes.byref(stream)))
        self.stream = stream.value
        self._adopted = []   # weak references to the engines on the batch stream

    def adopt(self, engine):
        """Put an engine on the batch stream (the batch launches on it); close() hands it back to its own stream."""
        engine.set_stream(self.stream)
        self._adopted.append(weakref.ref(engine))

    def advance(self, engines, n_steps, tables=None):
        """Enqueue n_steps steps of every engine (asynchronous).  tables: the engines' chunk_tables(n_steps) made
        beforehand for their present clocks (None, or a None entry: made here)."""
        n_steps = int(n_steps)
        n = len(engines)
        if n == 0 or n_steps <= 0:
            return
        if tables is None:
            tables = [None] * n
        tables = [t if t is not None else e.chunk_tables(n_steps) for e, t in zip(engines, tables)]
        handles = (ctypes.c_void_p * n)(*[e.handle.value for e in engines])
        fp = ctypes.POINTER(ctypes.c_float)
        values = (fp * n)(*[_native.fptr(t[0]) if t[0].size else None for t in tables])
        firsts = (ctypes.c_int64 * n)(*[t[1] for t in tables])
        counts = (ctypes.c_int64 * n)(*[t[2] for t in tables])
        phases = (fp * n)(*[_native.fptr(t[3]) if t[3].size else None for t in tables])
        _native.check(_native.load().os_fdtd2d_batch_advance(self._handle, handles, n, n_steps, values, firsts,
                                                             counts, phases))
        for e, t in zip(engines, tables):
            e.h2d_bytes += t[0].nbytes + t[3].nbytes
            e.n_step += n_steps
            e.time = t[4]

    def last_ms(self):
        ms, launches = ctypes.c_float(), ctypes.c_int64()
        _native.check(_native.load().os_fdtd2d_batch_last_ms(self._handle, ctypes.byref(ms), ctypes.byref(launches)))
        return float(ms.value), int(launches.value)

    def close(self):
        if self._handle is not None:
            # engines still open go back to their own streams before the batch stream is destroyed
            for ref in self._adopted:
                engine = ref()
                if engine is not None and engine._handle is not None:
                    engine.set_stream(None)
            self._adopted = []
            _native.load().os_fdtd2d_batch_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class JobSpec:
    """One request: window side (cells), rectangles (x0, y0, x1, y1 as fractions of the window, eps_r), source
    wavelength, steps, arrival time [s]."""
    job_id: int
    side: int
    rectangles: list
    wavelength: float
    steps: int
    arrival: float = 0.0
    dx: float = 20e-9
    npml: int = 15
    n_freqs: int = 4

    def cells(self):
        n = self.side + 2 * self.npml
        return n * n

    def device_bytes(self):
        """Device memory of the job: two field sets (6 floats), cb, psi slabs, spectra and staging, per cell 28 B."""
        n = self.side + 2 * self.npml
        return 28 * n * n + 32 * 4 * self.npml * n + 2 * 2 * 16 * self.n_freqs * n + (1 << 20)


def make_job_specs(n_jobs=256, rate=20.0, seed=7, side_range=(256, 2048), steps_range=(2000, 20000)):
    """The seeded request stream: Poisson arrivals at `rate` per second and the job mix described above."""
    rng = np.random.default_rng(seed)
    t = 0.0
    specs = []
    for job_id in range(n_jobs):
        t += float(rng.exponential(1.0 / rate)) if rate else 0.0
        side = int(rng.integers(side_range[0], side_range[1] + 1))
        rects = []
        for _ in range(int(rng.integers(1, 41))):
            x0, x1 = sorted(rng.uniform(0.2, 0.8, 2))
            y0, y1 = sorted(rng.uniform(0.0, 1.0, 2))
            rects.append((float(x0), float(y0), float(x1), float(y1), float(rng.uniform(1.0, 12.0))))
        specs.append(JobSpec(job_id, side, rects, float(rng.uniform(1000e-9, 1600e-9)),
                             int(rng.integers(steps_range[0], steps_range[1] + 1)), arrival=t))
    return specs


def build_job(spec, device=0, steps_per_launch=3, tile_rows=0):
    """(Simulation, flux monitors) of a request, finalized and on the device."""
    from .simulation import Simulation
    window = spec.side * spec.dx
    sim = Simulation(window, window, spec.dx, npml=spec.npml, boundaries='pml', verbose=False, device=device)
    for x0, y0, x1, y1, eps in spec.rectangles:
        sim.add_dielectric_rectangle(x0 * window, y0 * window, x1 * window, y1 * window, eps_r=eps)
    sim.add_line_source('y', 0.1 * window, wavelength=spec.wavelength, bandwidth=0.5)
    freqs = np.linspace(0.8, 1.2, spec.n_freqs) * (2.99792458e8 / spec.wavelength)
    monitors = [sim.add_flux_monitor('y', frac * window, (0.0, window), frequencies=freqs.tolist())
                for frac in (0.05, 0.9)]
    sim.em.engine.configure(variant=1, steps_per_launch=steps_per_launch, tile_rows=tile_rows)
    sim.em.finalize()
    return sim, monitors


@dataclass
class JobResult:
    job_id: int
    fluxes: list
    arrival: float
    admitted: float
    finished: float
    steps: int
    cells: int

    @property
    def latency(self):
        return self.finished - self.arrival


@dataclass
class _Active:
    spec: JobSpec
    sim: object
    monitors: list
    remaining: int
    admitted: float
    bytes: int = 0
    extra: dict = field(default_factory=dict)


class ServingLoop:
    """Admission by memory budget and slots, all active jobs stepped together in batched launches (three steps per
    blocked launch, as for one job alone).

    A tick advances every active job by chunk_steps, or by what it has left when that is less: the jobs with a full
    chunk left go together in one batched call, and the few that finish inside the tick in one call per remaining
    step count, so a job near its end never shortens everyone's tick.  Order of admission: arrival order when
    arrivals are honoured in real time; with every job queued at once, the largest (cells x steps) first, so that the
    small jobs fill the slots at the end instead of one large job running alone."""

    def __init__(self, device=0, memory_budget=120e9, max_active=48, chunk_steps=512, steps_per_launch=3,
                 tile_rows=0, admit_per_tick=16):
        self.device = int(device)
        self.memory_budget = float(memory_budget)
        self.max_active = int(max_active)
        self.admit_per_tick = max(1, int(admit_per_tick))
        self.chunk_steps = int(chunk_steps)
        self.steps_per_launch = int(steps_per_launch)
        self.tile_rows = int(tile_rows)
        self.advancer = BatchAdvancer(self.device)
        self.ticks = 0
        self.device_ms = 0.0
        self.launches = 0
        self.peak_active = 0
        self.peak_bytes = 0
        self.tick_log = []   # with time_ticks: (jobs, cell-updates, device ms) per tick

    def run(self, specs, realtime=True, time_ticks=False):
        """Serve `specs` (arrival times honoured on the wall clock when realtime, else all queued at once); returns
        the JobResults in completion order.  time_ticks: wait for every tick and add up its device time (device_ms,
        launches), at the price of a host wait per tick.

        Each tick is enqueued first; the jobs it finishes go back to their own streams behind it, and their fluxes
        are read after the next tick is enqueued (so the device never waits for that read); while the device runs the
        tick the host also admits arrivals (they join the next tick) and makes the next tick's source and phase
        tables.  At most admit_per_tick jobs are set up per tick, so a burst of
        arrivals starts on the device while the rest of it is still being set up on the host."""
        if realtime:
            pending = deque(sorted(specs, key=lambda s: (s.arrival, s.job_id)))
        else:
            pending = deque(sorted(specs, key=lambda s: (-s.cells() * s.steps, s.job_id)))
        active, results = [], []
        used = 0
        t0 = time.perf_counter()

        def admit(into, held):
            now = time.perf_counter() - t0
            budget = self.admit_per_tick
            while (pending and budget > 0 and (not realtime or pending[0].arrival <= now)
                   and len(into) < self.max_active and held + pending[0].device_bytes() <= self.memory_budget):
                budget -= 1
                spec = pending.popleft()
                sim, monitors = build_job(spec, self.device, self.steps_per_launch, self.tile_rows)
                self.advancer.adopt(sim.em.engine)
                into.append(_Active(spec, sim, monitors, spec.steps, time.perf_counter() - t0, spec.device_bytes()))
                held += spec.device_bytes()
            return held

        def calls(jobs):
            # (steps, jobs) of one tick: the jobs with a full chunk left together, the finishing ones by steps left
            groups = {}
            for a in jobs:
                groups.setdefault(min(self.chunk_steps, a.remaining), []).append(a)
            return sorted(groups.items(), key=lambda kv: -kv[0])

        def finish(jobs):
            # the jobs left the batch stream when their last tick was enqueued: their own streams wait for that tick
            # only, so reading them does not wait for the tick queued after it
            nonlocal used
            for a in jobs:
                fluxes = [m.flux() for m in a.monitors]
                finished = time.perf_counter() - t0
                arrival = a.spec.arrival if realtime else 0.0
                results.append(JobResult(a.spec.job_id, fluxes, arrival, a.admitted, finished, a.spec.steps,
                                         a.spec.cells()))
                a.sim.em.engine.close()
                used -= a.bytes

        tables = {}      # id(job) -> its chunk tables for the next tick, made while the device runs the current one
        unread = []      # jobs whose last tick is queued; read after the next tick is queued
        while pending or active or unread:
            if not active:
                used = admit(active, used)
                tables = {}
                if not active:
                    finish(unread)
                    unread = []
                    if pending:
                        time.sleep(max(0.0, min(0.005, pending[0].arrival - (time.perf_counter() - t0))))
                    continue
            self.peak_active = max(self.peak_active, len(active))
            self.peak_bytes = max(self.peak_bytes, used)
            for n, group in calls(active):
                self.advancer.advance([a.sim.em.engine for a in group], n, [tables.get(id(a)) for a in group])
                for a in group:
                    a.remaining -= n
                if time_ticks:
                    ms, launches = self.advancer.last_ms()
                    self.device_ms += ms
                    self.launches += launches
                    self.tick_log.append((len(group), sum(a.spec.cells() for a in group) * n, ms))
            self.ticks += 1
            done = [a for a in active if a.remaining == 0]
            survivors = [a for a in active if a.remaining > 0]
            for a in done:
                a.sim.em.engine.set_stream(None)   # back to its own stream, behind this tick's work
            # the jobs of the previous tick, now that this one keeps the device busy
            finish(unread)
            unread = done
            # while the device runs the tick: arrivals join the next one, whose tables are made now
            used = admit(survivors, used)
            tables = {id(a): a.sim.em.engine.chunk_tables(min(self.chunk_steps, a.remaining)) for a in survivors}
            active = survivors
        return results

    def close(self, trim=True):
        """Release the batch and (trim) the device memory the finished jobs left in the engines' pool; trim=False
        keeps it for the next loop, whose jobs then take their arrays from the pool instead of cudaMalloc."""
        self.advancer.close()
        if trim:
            _native.check(_native.load().os_fdtd_pool_trim())


def run_alone(spec, device=0, steps_per_launch=3, tile_rows=0):
    """One job on its own (the plain one-at-a-time run): (fluxes, wall seconds); tile_rows 0 = the engine's choice
    from the grid, None = autotuned."""
    t0 = time.perf_counter()
    sim, monitors = build_job(spec, device, steps_per_launch, tile_rows or 0)
    if tile_rows is None:
        sim.em.engine.autotune()
    sim.em.engine.advance(spec.steps)
    fluxes = [m.flux() for m in monitors]
    wall = time.perf_counter() - t0
    sim.em.engine.close()
    return fluxes, wall


def latency_percentiles(results):
    lat = np.array([r.latency for r in results])
    return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
