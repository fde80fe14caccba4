"""Grid arithmetic shared by the 2D and 3D engines: how many cells cover a length, and the explicit time step.

Two rules are fixed by open_sol, because every cell index and every step of a run depends on them bit for bit:

* the time step is a Courant fraction (0.99 unless given, allowed range (0, 1]) of the Yee scheme's CFL limit on
  the finest spacing of each axis, dt = fraction / (c0 sqrt(sum over axes of 1 / d^2)), evaluated in float64 and
  rounded once to float32 (open_sol/core/grid.py:9-17 for two axes, core/grid3d.py:8-17 for three);
* a length L covered by cells of width d has ceil(L / d - 1e-9) cells: the slack absorbs quotients such as
  4e-6 / 20e-9 = 200.00000000000003 that would otherwise gain a cell (core/grid.py:20-22).
"""
from __future__ import annotations

import math

import numpy as np

from .constants import C0, DTYPE

DEFAULT_COURANT_FACTOR = 0.99
_CELL_COUNT_SLACK = 1e-9


def _courant_fraction(courant, n_axes: int) -> float:
    fraction = DEFAULT_COURANT_FACTOR if courant is None else float(courant)
    if 0.0 < fraction <= 1.0:
        return fraction
    raise ValueError(f"courant must be a fraction of the {n_axes}D CFL limit in (0, 1], got {courant} "
                     f"(it is not C0 dt / dx: 0.99 means dt = 0.99 dx / (C0 sqrt({n_axes})) on equal cells)")


def yee_time_step(*spacings: float, courant: float = None) -> np.float32:
    """float32 time step of a Yee grid whose finest spacing per axis is given (two or three axes)."""
    fraction = _courant_fraction(courant, len(spacings))
    inverse_square_sum = sum(1.0 / float(d) ** 2 for d in spacings)
    return DTYPE(fraction / (C0 * np.sqrt(inverse_square_sum)))


def courant_time_step(dx_min: float, dy_min: float, courant_factor: float = None, dz_min: float = None):
    """open_sol's helper signature (2D, or 3D with dz_min) over yee_time_step."""
    spacings = (dx_min, dy_min) if dz_min is None else (dx_min, dy_min, dz_min)
    return yee_time_step(*spacings, courant=courant_factor)


def uniform_cell_count(length: float, dx: float) -> int:
    """Cells of width dx that cover length."""
    return math.ceil(length / dx - _CELL_COUNT_SLACK)


class Grid2D:
    """An nx x ny grid of square cells of width dx (held as float32, as the engines use it) and its time step.

    Grid2D(size_x, size_y, dx, courant=None, verbose=True) takes the total extent incl. any CPML padding."""

    __slots__ = ('nx', 'ny', 'dx', 'dy', 'size_x', 'size_y', 'dt', 'courant')

    def __init__(self, size_x: float, size_y: float, dx: float, courant: float = None, verbose: bool = True):
        if not dx > 0:
            raise ValueError(f"Grid2D needs dx > 0, got {dx}")
        counts = [uniform_cell_count(extent, dx) for extent in (size_x, size_y)]
        if min(counts) < 1:
            raise ValueError(f"Grid2D has no cells: size {size_x} x {size_y} m, dx {dx} m")
        self.nx, self.ny = counts
        self.dx = self.dy = DTYPE(dx)
        self.size_x, self.size_y = (n * self.dx for n in counts)
        self.dt = yee_time_step(dx, dx, courant=courant)
        self.courant = DTYPE(_courant_fraction(courant, 2))
        if verbose:
            print(self.describe())

    @property
    def shape(self):
        return (self.nx, self.ny)

    def describe(self) -> str:
        return (f"Grid2D {self.nx}x{self.ny}: cell {float(self.dx) * 1e9:.1f} nm, step {float(self.dt) * 1e18:.3f} as, "
                f"extent {float(self.size_x) * 1e6:.2f} x {float(self.size_y) * 1e6:.2f} um")
