"""Uniform 2D domain with the PML padded outside the physical window, its float32 material arrays and cell masks.

Geometry follows open_sol exactly (open_sol/core/domain.py:14-282): cell edges (k - origin) * dx, centres halfway,
masks evaluated on the float32 centres with open_sol's own numpy expressions.  A mask is kept as its bounding box
plus the boolean block inside it (BoxMask): painting 2000 cylinders on an 8192 x 8192 grid touches only the cells
near each one, and the cells it sets are exactly those of the reference's full-grid mask.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .boundaries import resolve_boundary
from .constants import DTYPE, FACES
from .grid import Grid2D


def containing_cell(coord, edges, first, last):
    """Cell index i with edges[i] <= coord < edges[i+1] (1e-9-cell snap), clamped to [first, last]
    (core/domain.py:275-282)."""
    coord = float(coord)
    if not math.isfinite(coord):
        raise ValueError(f"non-finite coordinate {coord}")
    snap = 1e-9 * (edges[first + 1] - edges[first])
    index = int(np.searchsorted(edges, coord + snap, side='right')) - 1
    return min(max(index, first), last)


@dataclass(frozen=True)
class BoxMask:
    """Cells of a mask: the tuple of slices bounding it and the boolean block over those slices."""
    box: tuple
    block: np.ndarray

    def full(self, shape):
        mask = np.zeros(shape, dtype=bool)
        mask[self.box] = self.block
        return mask


def _window_slice(centres, lo, hi):
    """Slice of the cells whose float32 centre can lie in [lo, hi] (two cells of margin on each side)."""
    a = int(np.searchsorted(centres, lo, side='left')) - 2
    b = int(np.searchsorted(centres, hi, side='right')) + 2
    return slice(max(a, 0), min(max(b, 0), centres.size))


class MaterialGrid:
    """Host float32 (nx, ny[, nz]) material arrays eps_r, sigma_e, mu_r, sigma_m and the H_z polarisation's eps_xx,
    eps_yy (core/material_grid.py:7-91).  An array still at its default is not allocated (None): a lossless,
    non-magnetic E_z grid uploads eps_r alone."""

    DEFAULTS = {'eps_r': 1.0, 'sigma_e': 0.0, 'mu_r': 1.0, 'sigma_m': 0.0, 'eps_xx': 1.0, 'eps_yy': 1.0}

    def __init__(self, shape, pinned=False):
        self.shape = tuple(shape)
        self.pinned = bool(pinned)   # page-locked host arrays (fast uploads; needs the CUDA library)
        self._arrays = {'eps_r': self._new(1.0)}
        self.version = 0   # bumped on every write (engines re-upload when it changed)

    def _new(self, value):
        if self.pinned:
            from ._native import pinned_empty
            arr = pinned_empty(self.shape, DTYPE)
            arr.fill(DTYPE(value))
            return arr
        return np.full(self.shape, DTYPE(value), dtype=DTYPE)

    def property_names(self):
        return tuple(self.DEFAULTS)

    def add_properties(self, schema: dict):
        """Register properties with their fill values (core/material_grid.py:45-47): an array filled with a value
        other than its default is allocated now, the others stay implicit."""
        for name, value in schema.items():
            if name not in self.DEFAULTS:
                raise AttributeError(f"MaterialGrid has no property '{name}'; registered: {list(self.DEFAULTS)}")
            if DTYPE(value) != DTYPE(self.DEFAULTS[name]) or name in self._arrays:
                self.array(name).fill(DTYPE(value))

    def get(self, name):
        """The array of `name`, or None while it holds its default everywhere."""
        return self._arrays.get(name)

    def array(self, name):
        """The array of `name`, allocated at its default on first use."""
        if name not in self.DEFAULTS:
            raise AttributeError(f"MaterialGrid has no property '{name}'; registered: {list(self.DEFAULTS)}")
        if name not in self._arrays:
            self._arrays[name] = self._new(self.DEFAULTS[name])
        return self._arrays[name]

    def __getattr__(self, name):
        if name in MaterialGrid.DEFAULTS:
            return self.array(name)
        raise AttributeError(name)

    def assign(self, name, mask, value):
        """Write a scalar (or full-grid array) into `name` where `mask` is set (mask None = every cell)."""
        if name not in self._arrays and mask is not None and np.isscalar(value) \
                and DTYPE(value) == DTYPE(self.DEFAULTS[name]):
            return   # writing the default into an untouched array changes nothing
        arr = self.array(name)
        self.version += 1
        if mask is None:
            np.copyto(arr, np.asarray(value, dtype=DTYPE))
            return
        if isinstance(mask, BoxMask):
            src = value if np.isscalar(value) else np.asarray(value, dtype=DTYPE)[mask.box]
            np.copyto(arr[mask.box], DTYPE(src) if np.isscalar(src) else src, where=mask.block)
            return
        mask = np.asarray(mask, dtype=bool)
        if mask.shape != self.shape:
            raise ValueError(f'mask shape {mask.shape} differs from the grid {self.shape}')
        np.copyto(arr, DTYPE(value) if np.isscalar(value) else np.asarray(value, dtype=DTYPE), where=mask)

    def set_mask(self, mask, **props):
        for name, val in props.items():
            if val is not None:
                self.assign(name, mask, val)


class Domain:
    """Grid + MaterialGrid + per-side PML padding of a uniform grid; physical origin at the window's lower corner
    (core/domain.py:135-197)."""

    dimensions = 2

    def __init__(self, grid, boundary_config, size_x, size_y, dx, npml_sides, pinned_host=False):
        self.grid = grid
        self.boundary_config = boundary_config
        self.size_x = float(size_x)
        self.size_y = float(size_y)
        self.dx = float(dx)
        self.npml_sides = dict(npml_sides)
        self.ox, self.oy = npml_sides['x_lo'], npml_sides['y_lo']
        if grid.nx - npml_sides['x_lo'] - npml_sides['x_hi'] < 1 or \
                grid.ny - npml_sides['y_lo'] - npml_sides['y_hi'] < 1:
            raise ValueError(f"Domain has no physical cells: grid {grid.nx} x {grid.ny}, PML sides {npml_sides}")
        self.materials = MaterialGrid((grid.nx, grid.ny), pinned=pinned_host)
        shape = (grid.nx, grid.ny)
        self._widths = tuple(np.full(n, self.dx) for n in shape)
        self._edges = tuple((np.arange(n + 1) - origin) * self.dx for n, origin in zip(shape, (self.ox, self.oy)))
        self._centers = tuple(0.5 * (e[:-1] + e[1:]) for e in self._edges)
        self._centers_f32 = tuple(c.astype(DTYPE) for c in self._centers)

    @classmethod
    def uniform(cls, size_x, size_y, dx, npml=15, courant=None, boundary_config=None, verbose=True,
                pinned_host=False):
        """core/domain.py:179-196: the CPML cells are added outside the size_x x size_y window."""
        bc = boundary_config if boundary_config is not None else resolve_boundary(None, npml)
        sides = bc.npml_sides
        total_x = size_x + (sides['x_lo'] + sides['x_hi']) * dx
        total_y = size_y + (sides['y_lo'] + sides['y_hi']) * dx
        grid = Grid2D(total_x, total_y, dx, courant, verbose=verbose)
        return cls(grid, bc, size_x, size_y, dx, sides, pinned_host=pinned_host)

    def physical_window(self):
        return (slice(self.npml_sides['x_lo'], self.grid.nx - self.npml_sides['x_hi']),
                slice(self.npml_sides['y_lo'], self.grid.ny - self.npml_sides['y_hi']))

    def cell_widths(self):
        """float64 widths of all cells per axis (the requested dx, not the float32 grid.dx)."""
        return self._widths

    def cell_edges(self):
        return self._edges

    def cell_centers(self):
        return self._centers

    def kernel_widths(self):
        """Widths the Yee kernels use: the float32 grid.dx as float64 (physics/em/yee_grid.py:11-16)."""
        return tuple(np.full(n, float(self.grid.dx)) for n in (self.grid.nx, self.grid.ny))

    def _validate(self, x, y, label):
        edge_tolerance = 1e-9 * max(self.size_x, self.size_y)
        if not (-edge_tolerance <= x <= self.size_x + edge_tolerance and
                -edge_tolerance <= y <= self.size_y + edge_tolerance):
            raise ValueError(f"{label} position ({x*1e6:.10g}, {y*1e6:.10g}) µm outside physical domain "
                             f"({self.size_x*1e6:.10g} x {self.size_y*1e6:.10g}) µm")

    def validate_physical_pos(self, x, y, label=''):
        self._validate(x, y, label)

    def pos_to_cell_x(self, x):
        window = self.physical_window()[0]
        return containing_cell(x, self._edges[0], window.start, window.stop - 1)

    def pos_to_cell_y(self, y):
        window = self.physical_window()[1]
        return containing_cell(y, self._edges[1], window.start, window.stop - 1)

    def pos_to_cell(self, x, y):
        return self.pos_to_cell_x(x), self.pos_to_cell_y(y)

    def rect_mask(self, x0, y0, x1, y1):
        """Cells whose float32 centre lies in [x_min, x_max) x [y_min, y_max) (core/domain.py:255-260)."""
        X, Y = self._centers_f32
        x_min, x_max = min(x0, x1), max(x0, x1)
        y_min, y_max = min(y0, y1), max(y0, y1)
        sx, sy = _window_slice(X, x_min, x_max), _window_slice(Y, y_min, y_max)
        Xb, Yb = X[sx][:, None], Y[sy][None, :]
        return BoxMask((sx, sy), (Xb >= x_min) & (Xb < x_max) & (Yb >= y_min) & (Yb < y_max))

    def circle_mask(self, cx, cy, radius):
        """Cells whose float32 centre lies within radius of (cx, cy) (core/domain.py:262-267)."""
        if not radius >= 0:
            raise ValueError(f"circle radius must be >= 0, got {radius}")
        X, Y = self._centers_f32
        sx = _window_slice(X, cx - radius, cx + radius)
        sy = _window_slice(Y, cy - radius, cy + radius)
        Xb, Yb = X[sx][:, None], Y[sy][None, :]
        return BoxMask((sx, sy), (Xb - cx) ** 2 + (Yb - cy) ** 2 <= radius ** 2)
