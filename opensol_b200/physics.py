"""EMPhysics on the B200 engine: open_sol's 2D FDTD physics (open_sol/physics/em/__init__.py:63) with the same
constructor, PhysicsSolver contract, material helpers, sources and monitors, stepping its engine on the device.

Both polarisations step float32 fields: 'ez' (E_z, H_x, H_y on FDTDEngine2D_Ez) and 'hz' (H_z, E_x, E_y on
FDTDEngine2D_Hz, face-averaged eps_xx / eps_yy); precision='double' raises.  Setup follows
the reference's finalize order (physics/em/__init__.py:181-203): coefficients, Courant check, source calibration,
DFT sample interval.  ``advance_ticks`` lets MultiphysicsRunner hand whole chunks to the device
(coupling/runner.py:97-101,183-186).
"""
from __future__ import annotations

import math

import numpy as np

from .boundaries import BoundaryConfig, inverse_spacings
from .constants import C0, DTYPE
from .engine2d import FDTDEngine2D_Ez, FDTDEngine2D_Hz
from .poles import DrudePole, LorentzPole, bounding_box
from .monitors import PROBE_COMPONENTS, DFTMonitor, FieldProbe, FluxMonitor, dft_sample_interval, resolve_frequencies
from .sources import (LineSource, TFSFSource, calibrate_line_source, calibrate_tangential_sheet, carrier_angular_frequency,
                      make_temporal, resolve_frequency)


class EMPhysics:
    """2D FDTD physics of a Domain, polarisation 'ez' (E_z, H_x, H_y) or 'hz' (H_z, E_x, E_y), on one B200."""

    name = 'em'
    coordinate_grids = ('cartesian',)

    def __init__(self, domain, polarization: str = 'ez', boundary_config=None, precision: str = 'single',
                 device: int = 0):
        if polarization not in ('ez', 'hz'):
            raise ValueError(f"polarization must be 'ez' (E_z, H_x, H_y) or 'hz' (H_z, E_x, E_y), got "
                             f"{polarization!r}")
        if precision not in ('single', 'double'):
            raise ValueError(f"EMPhysics precision must be 'single' (float32 fields) or 'double' (float64), got "
                             f"{precision!r}")
        if precision != 'single':
            raise NotImplementedError('the B200 engine steps float32 fields (stepper precision single)')
        self.domain = domain
        self.polarization = polarization
        self.precision = precision
        bc = boundary_config if boundary_config is not None else domain.boundary_config
        if bc is None:
            bc = BoundaryConfig.all_pml(domain.npml_sides['x_lo'])
        bc._validate()
        if bc.npml_sides != domain.npml_sides:
            raise ValueError(f"boundary_config PML cells {bc.npml_sides} do not match the domain padding "
                             f"{domain.npml_sides}; build the Domain with the same boundary_config")
        self.boundary_config = bc
        if polarization == 'hz':
            # eps_xx / eps_yy start from eps_r (register_em_arrays, physics/em/materials.py:27-35)
            materials = domain.materials
            for name in ('eps_xx', 'eps_yy'):
                if materials.get(name) is None:
                    np.copyto(materials.array(name), materials.array('eps_r'))
            self.engine = FDTDEngine2D_Hz(domain, bc, device=device)
        else:
            self.engine = FDTDEngine2D_Ez(domain, bc, device=device)
        self.sources = []
        self.monitors = []
        self.dispersive_regions = []   # (pole, box, cropped bool mask) in add order
        self._calibrations = []       # (source, omega, normal width)
        self._calibration_dirty = False
        self._finalized = False
        self.finalize_warnings = []
        self.runtime_warnings = []

    @property
    def permittivity_arrays(self):
        """MaterialGrid permittivity arrays the engine reads (physics/em/__init__.py:154-156)."""
        return ('eps_r',) if self.polarization == 'ez' else ('eps_xx', 'eps_yy')

    # --- PhysicsSolver contract ------------------------------------------------------------------------
    def prepare(self, domain):
        return

    def dt_limit(self) -> float:
        return float(self.engine.dt)

    def step(self, t: float = None, dt: float = None):
        """One Yee step (dt is advisory: the engine keeps its Courant dt)."""
        self._before_steps()
        self.engine.advance(1)

    def advance_ticks(self, n_ticks: int, t: float, dt: float, stop_time: float):
        """Whole chunk of the runner's tick loop (coupling/runner.py:183-203): ticks while t < stop_time, t += dt
        after each, at most n_ticks; returns (ticks run, new t)."""
        n_done = 0
        while n_done < n_ticks and t < stop_time:
            t = t + dt
            n_done += 1
        if n_done:
            self._before_steps()
            self.engine.advance(n_done)
        return n_done, t

    def _before_steps(self):
        if not self._finalized:
            self.finalize()
        if self._calibration_dirty:
            self._calibrate_sources()

    def state(self) -> dict:
        return self.engine.state()

    def finalize(self) -> None:
        """Coefficients from the final materials, Courant check, source calibration, DFT sample interval
        (physics/em/__init__.py:181-203), then the device engine brought up to date."""
        self.finalize_host()
        self.engine.sync_device()

    def finalize_host(self) -> None:
        """The host half of finalize: Courant check, calibrated source profiles, DFT sample interval."""
        self.finalize_warnings = []
        self._check_courant_stability()
        self._calibrate_sources()
        if self.engine.n_step == 0:
            dft_monitors = [mon for mon in self.monitors if hasattr(mon, 'frequencies')]   # not the probes
            m = dft_sample_interval(float(self.engine.dt), self.sources, [mon.frequencies for mon in dft_monitors])
            for monitor in dft_monitors:
                monitor.sample_interval = m
            self.engine.set_sample_interval(m)
        self._finalized = True

    def materials_changed(self, names) -> None:
        """Materials were rewritten: the device coefficients follow at the next step (the engine tracks the
        MaterialGrid version, bumped here for writes made in place on the arrays) and the sources recalibrate
        (physics/em/__init__.py:205-209)."""
        if frozenset(names) & {'eps_r', 'eps_xx', 'eps_yy', 'sigma_e', 'mu_r', 'sigma_m'}:
            self.domain.materials.version += 1
            self._calibration_dirty = True

    def renderer(self):
        raise NotImplementedError('rendering is outside the B200 FDTD engine')

    # --- checks / calibration --------------------------------------------------------------------------
    def _check_courant_stability(self):
        """ValueError when eps_r mu_r < (C0 dt)^2 (1/dx^2 + 1/dy^2) in some cell (physics/em/__init__.py:242-281,
        without poles)."""
        dt = float(self.engine.dt)
        dx_cells, dy_cells = self.domain.cell_widths()
        light = (C0 * dt) ** 2
        required_x = (light / dx_cells ** 2).astype(DTYPE)
        required_y = (light / dy_cells ** 2).astype(DTYPE)
        materials = self.domain.materials
        if self.polarization == 'ez':
            eps = materials.array('eps_r')
        else:
            eps = np.minimum(materials.array('eps_xx'), materials.array('eps_yy'))
        mu = materials.get('mu_r')
        # uniform grid: the light term is one value; the poles add mu_r x their step term on their cells
        requirement = required_x[0] + required_y[0]
        if self.dispersive_regions:
            pole_term = np.zeros(eps.shape, dtype=DTYPE)
            for pole, box, cropped in self.dispersive_regions:
                pole_term[box] += cropped.astype(DTYPE) * DTYPE(pole.step_term(dt))
            requirement = requirement + (pole_term if mu is None else mu * pole_term)
        product = eps if mu is None else eps * mu
        worst = float((product / requirement).min())
        if worst >= 1.0 - 1e-6:
            return
        ix, iy = np.unravel_index(int(np.argmin(product / requirement)), product.shape)
        x_centers, y_centers = self.domain.cell_centers()
        required = light * (1.0 / dx_cells[ix] ** 2 + 1.0 / dy_cells[iy] ** 2)
        stable = math.floor(float(self.domain.grid.courant) * math.sqrt(max(worst, 0.0)) * 1e3) / 1e3
        raise ValueError(f'eps_r * mu_r = {float(product[ix, iy]):.4g} at ({x_centers[ix]:.4g}, {y_centers[iy]:.4g}) '
                         f'm is below (C0 dt)^2 (1/dx^2 + 1/dy^2) = {required:.4g} there, so the time step is '
                         f'unstable; lower courant_factor to <= {stable:.3f}, or raise eps_r / mu_r')

    def _calibrate_sources(self):
        dt = float(self.domain.grid.dt)
        for source, omega, width in self._calibrations:
            if self.polarization == 'ez':
                source.profile = calibrate_line_source(source, self.domain.materials, omega, width, dt,
                                                       self.dispersive_regions)
            else:
                normal = 1 if source.axis == 'x' else 0
                source.profile = calibrate_tangential_sheet(
                    source, self.domain.materials, omega, width, dt,
                    self.engine.shares_y if normal == 1 else self.engine.shares_x,
                    self.domain.kernel_widths()[normal], self.dispersive_regions)
        self._calibration_dirty = False

    # --- dispersive poles ---------------------------------------------------------------------------
    def add_drude_rectangle(self, x0, y0, x1, y1, drude):
        """Drude medium on the cells of the rectangle, its eps_inf written as their eps_r
        (physics/em/__init__.py:329-340)."""
        self._add_pole(drude, self.domain.rect_mask(x0, y0, x1, y1), set_background=True)

    def add_drude_circle(self, cx, cy, radius, drude):
        self._add_pole(drude, self.domain.circle_mask(cx, cy, radius), set_background=True)

    def add_dispersive(self, pole, mask, weights=None):
        """Drude or Lorentz pole on a cell mask (a full-grid bool array or a domain mask), the permittivity arrays
        kept as the background (physics/em/__init__.py:342-361); cut-cell weights are not built."""
        if weights is not None:
            raise NotImplementedError('conformal pole weights are not built')
        if not isinstance(pole, (DrudePole, LorentzPole)):
            raise TypeError(f"add_dispersive needs a DrudePole or LorentzPole, got {type(pole).__name__}")
        self._add_pole(pole, mask, set_background=False)

    def _add_pole(self, pole, mask, set_background):
        """The pole on its mask's bounding box (the E_z engine steps it on the cells, the H_z engine on the face
        sets of E_x / E_y the mask reaches); set_background writes eps_inf into every permittivity array of the
        polarisation under the mask (FDTDEngine2D_Ez / _Hz.add_drude)."""
        grid = self.domain.grid
        full = mask.full((grid.nx, grid.ny)) if hasattr(mask, 'full') else np.asarray(mask, dtype=bool)
        if full.shape != (grid.nx, grid.ny):
            raise ValueError(f"Pole mask must have the grid shape {(grid.nx, grid.ny)}, got {full.shape}")
        box = bounding_box(full)
        if box is not None:
            self.engine.attach_pole(pole, box, full[box])
            self.dispersive_regions.append((pole, box, full[box]))
        if set_background:
            names = ('eps_r',) if self.polarization == 'ez' else ('eps_xx', 'eps_yy')
            for name in names:
                self.domain.materials.assign(name, full, pole.eps_inf)
            self.materials_changed(names)
        self._calibration_dirty = True

    # --- material helpers --------------------------------------------------------------------------------
    def add_dielectric_rectangle(self, x0, y0, x1, y1, eps_r, sigma_e=0.0):
        self._set_dielectric(self.domain.rect_mask(x0, y0, x1, y1), eps_r, sigma_e)

    def add_dielectric_circle(self, cx, cy, radius, eps_r, sigma_e=0.0):
        self._set_dielectric(self.domain.circle_mask(cx, cy, radius), eps_r, sigma_e)

    def _set_dielectric(self, mask, eps_r, sigma_e):
        """Isotropic eps_r into every permittivity array of this polarisation, plus sigma_e
        (physics/em/__init__.py:323-327)."""
        permittivity = {name: eps_r for name in self.permittivity_arrays}
        self.domain.materials.set_mask(mask, sigma_e=sigma_e, **permittivity)
        self.materials_changed(self.permittivity_arrays + ('sigma_e',))

    # --- sources ----------------------------------------------------------------------------------------
    def add_line_source(self, axis, position, wavelength=None, frequency=None, bandwidth=0.5, amplitude=1.0,
                        waveform='gaussian', span=None):
        """Sheet current radiating `amplitude` [V/m] to each side (physics/em/__init__.py:442-473); axis 'x' = line
        along x at y = position; span = (start, end) [m] or None (whole grid line)."""
        temporal = make_temporal(waveform, resolve_frequency(wavelength, frequency), bandwidth)
        d = self.domain
        if axis not in ('x', 'y'):
            raise ValueError(f"Line source axis must be 'x' or 'y', got {axis!r}")
        if axis == 'x':
            d.validate_physical_pos(0.0, position, "Line source (y)")
            line_cell, along_cell, n_along = d.pos_to_cell_y(position), d.pos_to_cell_x, d.grid.nx
        else:
            d.validate_physical_pos(position, 0.0, "Line source (x)")
            line_cell, along_cell, n_along = d.pos_to_cell_x(position), d.pos_to_cell_y, d.grid.ny
        along_axis = 0 if axis == 'x' else 1
        normal_width = float(d.cell_widths()[1 - along_axis][line_cell])
        if self.polarization == 'hz':
            # on the hi face of the line cell: w_perp = the dual spacing there (placement.py:254-265)
            periodic = self.boundary_config.periodic_y if axis == 'x' else self.boundary_config.periodic_x
            n_cells = d.grid.ny if axis == 'x' else d.grid.nx
            if line_cell == n_cells - 1 and not periodic:
                raise ValueError(f"Line source: the H_z sheet sits on the hi face of cell {line_cell}, the outer grid "
                                 f"wall; move the line at least one cell inside")
            _, inv_face = inverse_spacings(d.kernel_widths()[1 - along_axis])
            normal_width = 1.0 / float(inv_face[line_cell])
        if span is None:
            lo, hi = 0, n_along
        else:
            start, end = sorted((float(span[0]), float(span[1])))
            for coord in (start, end):
                if axis == 'x':
                    d.validate_physical_pos(coord, position, "Line source span")
                else:
                    d.validate_physical_pos(position, coord, "Line source span")
            lo, hi = along_cell(start), along_cell(end) + 1
            window = d.physical_window()[along_axis]
            bc = self.boundary_config
            if lo == window.start and getattr(bc, f'{axis}_lo').value == 'cpml':
                lo = 0
            if hi == window.stop and getattr(bc, f'{axis}_hi').value == 'cpml':
                hi = n_along
        source = LineSource(axis, line_cell, temporal, amplitude, span=(lo, hi),
                            profile=np.zeros(hi - lo, dtype=DTYPE))
        self.sources.append(source)
        self._calibrations.append((source, carrier_angular_frequency(temporal), normal_width))
        self._calibration_dirty = True
        self.engine.attach_line_source(source)
        return source

    def add_tfsf(self, x0, y0, x1, y1, wavelength=None, frequency=None, bandwidth=0.5, amplitude=1.0,
                 waveform='gaussian'):
        """+x plane wave of incident peak `amplitude` [V/m] (E_z; E_y on hz) inside the box (physics/em/__init__.py:475-490 with
        placement.tfsf_box_cells): the box's cells plus one scattered-field cell on every side lie in the physical
        window (this engine's boundary presets have no mirror face a box could open onto)."""
        d = self.domain
        temporal = make_temporal(waveform, resolve_frequency(wavelength, frequency), bandwidth)
        d.validate_physical_pos(x0, y0, "TFSF box corner 0")
        d.validate_physical_pos(x1, y1, "TFSF box corner 1")
        x_lo, x_hi = sorted((x0, x1))
        y_lo, y_hi = sorted((y0, y1))
        ix0, ix1 = d.pos_to_cell_x(x_lo), d.pos_to_cell_x(x_hi) + 1
        iy0, iy1 = d.pos_to_cell_y(y_lo), d.pos_to_cell_y(y_hi) + 1
        window_x, window_y = d.physical_window()
        if ix0 <= window_x.start or ix1 >= window_x.stop or iy0 <= window_y.start or iy1 >= window_y.stop:
            raise ValueError(f"TFSF box cells [{ix0}, {ix1}) x [{iy0}, {iy1}) need at least one scattered-field cell "
                             f"inside the physical window [{window_x.start}, {window_x.stop}) x "
                             f"[{window_y.start}, {window_y.stop}) on every side")
        grid = d.grid
        widths = (np.full(grid.nx, float(grid.dx)), np.full(grid.ny, float(grid.dy)))   # yee_grid.grid_cell_widths
        source = TFSFSource(ix0, ix1, iy0, iy1, temporal, float(grid.dt), amplitude, cell_widths=widths,
                            polarization=self.polarization)
        self.sources.append(source)
        self.engine.attach_tfsf(source)
        return source

    # --- monitors ---------------------------------------------------------------------------------------
    def add_field_probe(self, x, y, field_component=None):
        """Raw Yee samples of one field component at the cell containing (x, y) after every step; None = the
        out-of-plane field (physics/em/__init__.py:492-498, placement.probe_cell)."""
        components = PROBE_COMPONENTS[self.polarization]
        if field_component is None:
            field_component = components[0]
        if field_component not in components:
            raise ValueError(f"field probe component of an {self.polarization!r} physics must be one of "
                             f"{components}, got {field_component!r}")
        d = self.domain
        d.validate_physical_pos(x, y, "Field probe")
        probe = FieldProbe(d.pos_to_cell_x(x), d.pos_to_cell_y(y), field_component)
        self.monitors.append(probe)
        self.engine.attach_probe(probe)
        return probe

    def add_dft_monitor(self, x0, y0, x1, y1, wavelengths=None, frequencies=None, downsample=1):
        """Running DFT of E_z over the cell box of the physical box (x0, y0)-(x1, y1); downsample s > 1 records every
        s-th cell along x and y (physics/em/__init__.py:500-509, placement.box_cells)."""
        d = self.domain
        d.validate_physical_pos(x0, y0, "DFT monitor corner 0")
        d.validate_physical_pos(x1, y1, "DFT monitor corner 1")
        x_lo, x_hi = sorted((x0, x1))
        y_lo, y_hi = sorted((y0, y1))
        cells = (d.pos_to_cell_x(x_lo), d.pos_to_cell_x(x_hi) + 1, d.pos_to_cell_y(y_lo), d.pos_to_cell_y(y_hi) + 1)
        monitor = DFTMonitor(slice(cells[0], cells[1]), slice(cells[2], cells[3]),
                             resolve_frequencies(wavelengths, frequencies), float(d.grid.dt),
                             polarization=self.polarization, downsample=downsample)
        self.monitors.append(monitor)
        self.engine.attach_dft_monitor(monitor)
        return monitor

    def add_flux_monitor(self, axis, position, span, wavelengths=None, frequencies=None):
        """Poynting flux through a line (axis 'x' = along x at y = position, flux > 0 toward +y)
        (physics/em/__init__.py:511-518, placement.flux_line_cells)."""
        d = self.domain
        if span is None or len(span) != 2:
            raise ValueError(f"Flux monitor needs span = (start, end) along the line [m], got {span!r}")
        lo, hi = sorted((float(span[0]), float(span[1])))
        dx_cells, dy_cells = d.cell_widths()
        if axis == 'x':
            d.validate_physical_pos(lo, position, "Flux monitor start")
            d.validate_physical_pos(hi, position, "Flux monitor end")
            normal, line_cell, cells, widths = 'y', d.pos_to_cell_y(position), (d.pos_to_cell_x(lo),
                                                                               d.pos_to_cell_x(hi) + 1), dx_cells
        elif axis == 'y':
            d.validate_physical_pos(position, lo, "Flux monitor start")
            d.validate_physical_pos(position, hi, "Flux monitor end")
            normal, line_cell, cells, widths = 'x', d.pos_to_cell_x(position), (d.pos_to_cell_y(lo),
                                                                               d.pos_to_cell_y(hi) + 1), dy_cells
        else:
            raise ValueError(f"Flux monitor axis (along the line) must be 'x' or 'y', got {axis!r}")
        monitor = FluxMonitor(normal, line_cell, cells, resolve_frequencies(wavelengths, frequencies),
                              float(d.grid.dt), widths, polarization=self.polarization)
        self.monitors.append(monitor)
        self.engine.attach_flux_monitor(monitor)
        return monitor
