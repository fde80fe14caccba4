"""EMPhysics3D on the B200 engine: open_sol's em_fdtd_3d physics (open_sol/physics/em3d/physics3d.py:133-497) with the
same constructor, PhysicsSolver contract, dipoles and flux planes / boxes, stepping FDTDEngine3D on the device.

finalize follows the reference (physics3d.py:192-217, 261-282): material index, dipole calibration from the live
face cb, DFT sample interval.  ``advance_ticks`` lets MultiphysicsRunner hand whole chunks to the device.
"""
from __future__ import annotations

import numpy as np

from .constants import DTYPE
from .domain3d import AXES, BoundaryConfig3D
from .engine3d import FDTDEngine3D
from .monitors import dft_sample_interval, resolve_frequencies
from .monitors3d import FluxBox3D, PlaneFlux3D
from .sources import make_temporal, resolve_frequency

DIPOLE_ORIENTATIONS = ('x', 'y', 'z')
MATERIAL_ARRAYS = ('eps_r', 'eps_xx', 'eps_yy', 'sigma_e', 'mu_r', 'sigma_m')


def nearest_face(edges, coordinate, window):
    """Index f of the E face (hi face of cell f) nearest `coordinate`, f in [window.start, window.stop - 2]
    (sources3d.py:31-38)."""
    first, last = window.start, window.stop - 2
    if last < first:
        raise ValueError('a dipole along an axis needs at least 2 window cells on that axis')
    return min(range(first, last + 1), key=lambda face: abs(float(edges[face + 1]) - coordinate))


class DipoleSource3D:
    """E_component += weight * s(t) on cell `cell`; weight = cb (I l) / V of the face (sources3d.py:41-75)."""

    def __init__(self, component, cell, temporal, moment, volume):
        if component not in ('ex', 'ey', 'ez'):
            raise ValueError(f"dipole component must be 'ex', 'ey' or 'ez', got {component!r}")
        self.component = component
        self.axis = 'xyz'.index(component[1])
        self.cell = tuple(int(i) for i in cell)
        self.temporal = temporal
        self.moment = float(moment)
        self.volume = float(volume)
        self.weight = None

    def calibrate(self, engine):
        """weight = live face cb x FP32(moment / volume) (sources3d.py:56-61)."""
        cb = engine.face_cb(self.axis, self.cell)
        self.weight = DTYPE(cb * DTYPE(self.moment / self.volume / 1.0))
        engine.set_dipole_weight(self)


class EMPhysics3D:
    """3D FDTD on a Domain3D on one B200."""

    name = 'em'
    type_label = 'em_fdtd_3d'

    def __init__(self, domain, precision='single', device=0):
        if getattr(domain, 'dimensions', 2) != 3:
            raise ValueError('EMPhysics3D needs a Domain3D (a model with domain size_z)')
        config = domain.boundary_config
        if not isinstance(config, BoundaryConfig3D):
            raise ValueError(f'em_fdtd_3d needs a Domain3D built with a BoundaryConfig3D, got {type(config).__name__}')
        config.validate()
        if config.npml_sides != domain.npml_sides:
            raise ValueError(f'BoundaryConfig3D PML cells {config.npml_sides} do not match the domain padding '
                             f'{domain.npml_sides}')
        self.domain = domain
        self.boundary_config = config
        self.engine = FDTDEngine3D(domain, config, precision, device)
        self.sources = []
        self.monitors = []
        self._materials_dirty = True
        self._finalized = False
        self.finalize_warnings = []
        self.runtime_warnings = []

    # ---- PhysicsSolver contract
    def prepare(self, domain):
        return

    def dt_limit(self) -> float:
        return float(self.engine.dt)

    def step(self, t=None, dt=None):
        self._before_steps()
        self.engine.advance(1)

    def advance_ticks(self, n_ticks: int, t: float, dt: float, stop_time: float):
        """Whole chunk of the runner's tick loop: ticks while t < stop_time, t += dt after each, at most n_ticks."""
        n_done = 0
        while n_done < n_ticks and t < stop_time:
            t = t + dt
            n_done += 1
        if n_done:
            self._before_steps()
            self.engine.advance(n_done)
        return n_done, t

    def run(self, n_steps):
        """n_steps Yee steps (a script's loop of step())."""
        self._before_steps()
        self.engine.advance(int(n_steps))

    def _before_steps(self):
        if not self._finalized:
            self.finalize()
        elif self._materials_dirty:
            self._refresh_materials()

    def state(self):
        return {**self.engine.state(), 'eps_r': self.domain.materials.array('eps_r'), 'q_accum': None}

    def materials_changed(self, names):
        if not set(MATERIAL_ARRAYS).isdisjoint(names):
            self._materials_dirty = True

    def finalize(self):
        """Material index, dipole calibration, DFT sample interval (before the first step only)."""
        self._refresh_materials()
        if self.engine.n_step == 0:
            interval = dft_sample_interval(self.engine.dt, self.sources,
                                           [monitor.frequencies for monitor in self.monitors])
            for monitor in self.monitors:
                monitor.sample_interval = interval
            self.engine.set_sample_interval(interval)
        self._finalized = True

    def _refresh_materials(self):
        self.engine.rebuild_materials()
        for source in self.sources:
            source.calibrate(self.engine)
        self._materials_dirty = False

    # ---- materials
    def add_dielectric_sphere(self, cx, cy, cz, radius, eps_r, sigma_e=0.0):
        """eps_r (and sigma_e) on the cells whose centre lies within radius of (cx, cy, cz) (later writes win)."""
        mask = self.domain.sphere_mask(cx, cy, cz, radius)
        self.domain.materials.set_mask(mask, eps_r=eps_r, sigma_e=sigma_e)
        self.materials_changed(('eps_r', 'sigma_e'))

    # ---- sources
    def add_dipole(self, x, y, z, orientation='z', dipole_moment=1e-12, wavelength=None, frequency=None,
                   bandwidth=0.5, waveform='gaussian'):
        """Electric point dipole of moment I l [A m] on the E face nearest (x, y, z) (physics3d.py:403-423)."""
        if orientation not in DIPOLE_ORIENTATIONS:
            raise ValueError(f"dipole orientation must be one of {DIPOLE_ORIENTATIONS}, got {orientation!r}")
        domain = self.domain
        domain.validate_physical_pos(x, y, z, 'Dipole')
        temporal = make_temporal(waveform, resolve_frequency(wavelength, frequency), bandwidth)
        axis = AXES.index(orientation)
        cell = list(domain.pos_to_cell(x, y, z))
        cell[axis] = nearest_face(domain.cell_edges()[axis], (x, y, z)[axis], domain.physical_window()[axis])
        source = DipoleSource3D('e' + orientation, cell, temporal, dipole_moment,
                                self.engine.face_dual_volume(axis, cell))
        self.sources.append(source)
        self.engine.attach_dipole(source)
        self._materials_dirty = True
        return source

    # ---- monitors
    def _window_edges(self):
        return tuple((cells.start, cells.stop) for cells in self.domain.physical_window())

    def _nearest_edge(self, axis, coordinate):
        first, last = self._window_edges()[axis]
        edges = self.domain.cell_edges()[axis]
        return first + int(np.argmin(np.abs(edges[first:last + 1] - float(coordinate))))

    def add_flux_plane(self, normal, position, wavelengths=None, frequencies=None):
        """Flux through the cell-edge plane nearest `position` along `normal` across the whole physical window."""
        axis = AXES.index(normal)
        bounds = list(self._window_edges())
        bounds[axis] = (self._nearest_edge(axis, position),) * 2
        monitor = PlaneFlux3D(axis, bounds[axis][0], bounds, resolve_frequencies(wavelengths, frequencies),
                              self.engine.dt, self.engine.widths, self.engine.shape, self.engine.periodic)
        self.monitors.append(monitor)
        self.engine.attach_flux_monitor(monitor)
        return monitor

    def add_flux_box(self, lo, hi, wavelengths=None, frequencies=None):
        """Net outward flux through the box between the cell edges nearest the corners lo, hi."""
        bounds = []
        for axis in range(3):
            first = self._nearest_edge(axis, min(lo[axis], hi[axis]))
            last = self._nearest_edge(axis, max(lo[axis], hi[axis]))
            if last <= first:
                raise ValueError(f'flux box spans no cell along {AXES[axis]}: corners {lo[axis]:.4g} and '
                                 f'{hi[axis]:.4g} m snap to the same cell edge')
            bounds.append((first, last))
        monitor = FluxBox3D(bounds, resolve_frequencies(wavelengths, frequencies), self.engine.dt,
                            self.engine.widths, self.engine.shape, self.engine.periodic)
        self.monitors.append(monitor)
        self.engine.attach_flux_monitor(monitor)
        return monitor
