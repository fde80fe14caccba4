"""Simulation and MultiphysicsRunner of the B200 engine: open_sol's scripting entry (open_sol/simulation.py:18-326) and
tick loop (open_sol/coupling/runner.py:8-229) for the FDTD path.

``Simulation(size_x, size_y, dx, npml, courant, boundaries, polarization)`` builds the padded uniform domain and one
EMPhysics; unknown attributes fall through to that physics, so ``sim.add_line_source(...)`` and
``sim.add_flux_monitor(...)`` read as in the reference.  ``run(duration | n_steps)`` finalizes, prepares the runner and
advances in print_every chunks; with a single stride-1 solver the runner hands each chunk to the solver's
``advance_ticks``, i.e. to one device chunk.
"""
from __future__ import annotations

import math
import sys
import time as _time
import warnings
from types import MappingProxyType

from .boundaries import resolve_boundary
from .domain import Domain
from .physics import EMPhysics


class MultiphysicsRunner:
    """Steps named solvers in whole ticks of dt_sync = min(dt_limit) (coupling/runner.py:8-229, without couplings)."""

    def __init__(self):
        self.physics = {}
        self.strides = {}
        self.couplings = []
        self.t = 0.0
        self.tick = 0
        self._prepared = False
        self._dt_sync = math.inf
        self._schedule = ()
        self._hand_off = None
        self.prepare_warnings = []

    def add(self, name, solver, every: int = 1):
        if name in self.physics:
            raise ValueError(f"physics '{name}' is already attached")
        if int(every) < 1:
            raise ValueError(f"physics '{name}': every must be >= 1, got {every}")
        solver.name = name
        self.physics[name] = solver
        self.strides[name] = int(every)
        self._prepared = False

    def prepare(self):
        limits = {name: float(solver.dt_limit()) for name, solver in self.physics.items()}
        dt_sync = min(limits.values(), default=math.inf)
        if not dt_sync > 0:
            raise ValueError(f"dt_limit must be positive; got {limits}")
        for name, limit in limits.items():
            span = self.strides[name] * dt_sync
            if limit < span * (1.0 - 1e-9):
                raise ValueError(f"physics '{name}' advances at most {limit:.4e} s per step, but every="
                                 f"{self.strides[name]} makes it cover {span:.4e} s per step; use every=1 "
                                 f"for it (sync dt = {dt_sync:.4e} s)")
        self._dt_sync = dt_sync
        self._schedule = tuple((solver, self.strides[name], self.strides[name] * dt_sync)
                               for name, solver in self.physics.items())
        solver, stride, _ = self._schedule[0] if len(self._schedule) == 1 else (None, 0, 0)
        self._hand_off = (solver if stride == 1 and not self.couplings
                          and callable(getattr(solver, 'advance_ticks', None)) else None)
        self._prepared = True
        self.prepare_warnings = []
        return self.prepare_warnings

    @property
    def dt_sync(self):
        if self._prepared:
            return self._dt_sync
        return min((float(s.dt_limit()) for s in self.physics.values()), default=math.inf)

    def advance(self, n_ticks: int, t_end: float = None) -> int:
        """Run up to n_ticks ticks, stopping once t >= t_end - dt_sync/2 (runner.py:174-204)."""
        if not self._prepared:
            self.prepare()
        dt_sync = self._dt_sync
        if not math.isfinite(dt_sync):
            raise ValueError("nothing steps in time (every physics has an infinite dt_limit); use a stationary study")
        stop_time = math.inf if t_end is None else t_end - 0.5 * dt_sync
        if self._hand_off is not None:
            n_done, self.t = self._hand_off.advance_ticks(int(n_ticks), self.t, dt_sync, stop_time)
            self.tick += n_done
            return n_done
        n_done = 0
        while n_done < n_ticks and self.t < stop_time:
            tick, t = self.tick, self.t
            for solver, stride, span in self._schedule:
                if tick % stride == 0:
                    solver.step(t, span)
            self.t = t + dt_sync
            self.tick = tick + 1
            n_done += 1
        return n_done

    def flush(self):
        for solver in self.physics.values():
            sync = getattr(getattr(solver, 'engine', None), 'synchronize', None)
            if sync is not None:
                sync()

    def clear(self):
        self.physics.clear()
        self.strides.clear()
        self._schedule = ()
        self._hand_off = None
        self._prepared = False
        self._dt_sync = math.inf


class Simulation:
    """Domain + named physics driven by one MultiphysicsRunner; single-physics attributes fall through."""

    def __init__(self, size_x: float = None, size_y: float = None, dx: float = None, npml: int = 15,
                 courant: float = None, boundaries=None, *, polarization: str = 'ez', device: int = 0,
                 verbose: bool = True, pinned_host: bool = False):
        if size_x is None or size_y is None or dx is None:
            raise ValueError("Simulation() needs (size_x, size_y, dx, ...) for the single-physics EM-FDTD convenience "
                             "path; use Simulation.multiphysics(domain) for the multi-physics path.")
        bc = resolve_boundary(boundaries, npml)
        domain = Domain.uniform(size_x, size_y, dx, npml=npml, courant=courant, boundary_config=bc, verbose=verbose,
                                pinned_host=pinned_host)
        self._init_common(domain)
        self.add_physics('em', EMPhysics(domain, polarization=polarization, boundary_config=bc, device=device))

    @classmethod
    def multiphysics(cls, domains):
        sim = cls.__new__(cls)
        sim._init_common(domains)
        return sim

    def _init_common(self, domains):
        self.domains = list(domains) if isinstance(domains, (list, tuple)) else [domains]
        if not self.domains:
            raise ValueError('Simulation needs at least one Domain')
        self.domain = self.domains[0]
        self._physics_domains = {}
        self.runner = MultiphysicsRunner()
        self.callbacks = []
        self._physics_by_name = {}
        self._finalized_names = set()

    @property
    def grid(self):
        return self.domain.grid

    @property
    def materials(self):
        return self.domain.materials

    @property
    def physics(self):
        return MappingProxyType(self._physics_by_name)

    def add_physics(self, name: str, solver, every: int = 1, domain=None):
        domain = domain if domain is not None else getattr(solver, 'domain', self.domain)
        self.runner.add(name, solver, every=every)
        self._physics_by_name[name] = solver
        self._physics_domains[name] = domain
        return solver

    def finalize(self, names=None) -> dict:
        if names is None:
            names = [name for name in self._physics_by_name if name not in self._finalized_names]
        out = {}
        for name in names:
            solver = self._physics_by_name[name]
            solver.finalize()
            self._finalized_names.add(name)
            out[name] = list(getattr(solver, 'finalize_warnings', ()))
        return out

    def clear(self):
        for solver in self._physics_by_name.values():
            close = getattr(getattr(solver, 'engine', None), 'close', None)
            if close is not None:
                close()
        self.runner.clear()
        self._physics_by_name.clear()
        self._physics_domains.clear()
        self._finalized_names.clear()
        self.domain = None
        self.domains = []

    def __getattr__(self, name):
        if name.startswith('__'):
            raise AttributeError(name)
        by_name = self.__dict__.get('_physics_by_name')
        if by_name:
            if name in by_name:
                return by_name[name]
            if len(by_name) == 1:
                sole_name, sole = next(iter(by_name.items()))
                try:
                    return getattr(sole, name)
                except AttributeError:
                    raise AttributeError(f"'Simulation' has no attribute '{name}' and neither has its only physics "
                                         f"'{sole_name}'.") from None
            attached = list(by_name)
            raise AttributeError(f"'Simulation' has no attribute '{name}'. Multiple physics attached ({attached}); "
                                 f"call sim.<name>.{name}(...) explicitly (e.g. sim.{attached[0]}.{name}).")
        raise AttributeError(f"'Simulation' has no attribute '{name}' and no physics are attached.")

    def run(self, duration: float = None, n_steps: int = None, print_every: int = 500, flush: bool = True,
            verbose: bool = True):
        """finalize() new physics, prepare the runner, advance by `duration` [s] or `n_steps` ticks in print_every
        chunks, then flush (simulation.py:272-326)."""
        if (duration is None) == (n_steps is None):
            raise ValueError("Simulation.run needs exactly one of duration [s] or n_steps")
        if n_steps is not None and int(n_steps) < 0:
            raise ValueError(f"n_steps must be >= 0, got {n_steps}")
        if duration is not None and not float(duration) >= 0:
            raise ValueError(f"duration must be >= 0, got {duration}")
        runner = self.runner
        if not math.isfinite(runner.dt_sync):
            raise ValueError(f"Simulation.run: nothing steps in time (every physics in {list(self._physics_by_name)} "
                             f"is quasi-static, dt_limit inf)")
        for name, messages in self.finalize().items():
            for message in messages:
                warnings.warn(f"physics '{name}': {message}", stacklevel=2)
        runner.prepare()
        t_end = None if duration is None else runner.t + float(duration)
        tick_budget = sys.maxsize if n_steps is None else int(n_steps)
        span = f"n_steps={tick_budget}" if n_steps is not None else f"duration={float(duration):.4e} s"
        if verbose:
            print(f"\nOpen_sol: physics={list(self._physics_by_name)}, couplings=0, dt_sync={runner.dt_sync:.4e} s, "
                  f"{span}")
        callbacks = list(self.callbacks)
        wall_start = _time.perf_counter()
        ticks_done = 0
        while ticks_done < tick_budget:
            if callbacks:
                chunk = 1
            elif print_every > 0:
                chunk = print_every - ticks_done % print_every
            else:
                chunk = tick_budget - ticks_done
            n_advanced = runner.advance(min(chunk, tick_budget - ticks_done), t_end)
            if n_advanced == 0:
                break
            ticks_done += n_advanced
            for callback in callbacks:
                callback(runner)
            if verbose and print_every > 0 and ticks_done % print_every == 0:
                print(f"  tick {runner.tick}, t = {runner.t:.4e} s")
        if flush:
            runner.flush()
        wall = _time.perf_counter() - wall_start
        if verbose:
            print(f"Done: {ticks_done} ticks in {wall:.2f} s (t = {runner.t:.4e} s)")
        return ticks_done
