"""Flux planes and flux boxes of the 3D engine: the sample geometry and the host readout of open_sol's PlaneFlux3D /
FluxBox3D (physics/em3d/monitors3d.py:23-162).

A plane at cell edge `edge` along its normal holds two (E, H) pairs: (E_first, H_second) sampled on the faces of the
first tangential axis and the cells of the second, and (E_second, H_first) the other way round (first / second =
normal + 1 / + 2 mod 3).  E is the mean of the layers edge - 1 and edge, H lies on layer edge - 1; both are summed as
complex128 running DFTs on the device.  flux() = cos(omega dt / 2) sum sign Re(E conj(H e^{j pi f dt})) x area, the
face widths as trapezoid weights, computed on the host in float64 as the reference does.
"""
from __future__ import annotations

import numpy as np

from .monitors import check_frequencies


def face_samples(widths, first_edge, last_edge, wrap=False):
    """(face slice, trapezoid weights) of samples on the cell edges first_edge..last_edge (face f = edge f + 1; edge
    0 has no face); wrap: a periodic axis spanned whole, every face with its dual width (monitors3d.py:23-36)."""
    widths = np.asarray(widths, dtype=np.float64)
    if wrap:
        return slice(0, widths.size), 0.5 * (widths + np.roll(widths, -1))
    edges = np.arange(max(first_edge, 1), last_edge + 1)
    below = np.where(edges > first_edge, widths[np.maximum(edges - 1, 0)], 0.0)
    above = np.where(edges < last_edge, widths[np.minimum(edges, widths.size - 1)], 0.0)
    return slice(int(edges[0]) - 1, int(edges[-1])), 0.5 * (below + above)


class PlaneFlux3D:
    """Spectral Poynting flux through the cell-edge plane `edge` along normal_axis (0 / 1 / 2) over the edge ranges
    bounds[t] = (first, last) of the tangential axes; > 0 toward +normal."""

    def __init__(self, normal_axis, edge, bounds, frequencies, dt, widths, shape, periodic=(False, False, False)):
        n_normal = shape[normal_axis]
        if not 1 <= edge <= n_normal - 1:
            raise ValueError(f"flux plane at {'xyz'[normal_axis]} edge {edge} needs a cell on both sides (edges 1 to "
                             f'{n_normal - 1})')
        self.normal_axis = int(normal_axis)
        self.edge = int(edge)
        self.bounds = tuple(tuple(int(v) for v in b) for b in bounds)
        self.frequencies = check_frequencies(frequencies)
        self.dt = float(dt)
        self.sample_interval = 1
        first_axis, second_axis = (normal_axis + 1) % 3, (normal_axis + 2) % 3
        self.pairs = []
        for e_axis, h_axis, face_axis, cell_axis, sign in ((first_axis, second_axis, first_axis, second_axis, 1.0),
                                                           (second_axis, first_axis, second_axis, first_axis, -1.0)):
            wrap = bool(periodic[face_axis]) and tuple(self.bounds[face_axis]) == (0, shape[face_axis])
            face_slice, face_weights = face_samples(widths[face_axis], *self.bounds[face_axis], wrap=wrap)
            first, last = self.bounds[cell_axis]
            cell_weights = np.asarray(widths[cell_axis][first:last], dtype=np.float64)
            origin, extent = [0, 0, 0], [1, 1, 1]
            origin[face_axis], extent[face_axis] = face_slice.start, face_slice.stop - face_slice.start
            origin[cell_axis], extent[cell_axis] = first, last - first
            weights = {face_axis: face_weights, cell_axis: cell_weights}
            low_axis, high_axis = sorted((face_axis, cell_axis))
            self.pairs.append({'e_comp': e_axis, 'h_comp': h_axis, 'sign': sign, 'origin': tuple(origin),
                               'extent': tuple(extent), 'area': np.outer(weights[low_axis], weights[high_axis]),
                               'pair_id': None})
        self._reader = None   # pair index -> (E, H) complex128 (nf, n_low, n_high), set by the engine

    def spectra(self):
        """[(E, H) per pair] complex128 running DFTs phased at the E sample times (H not yet re-timed)."""
        out = []
        for index, pair in enumerate(self.pairs):
            if self._reader is None:
                zeros = np.zeros((self.frequencies.size,) + pair['area'].shape, np.complex128)
                out.append((zeros, zeros.copy()))
            else:
                out.append(self._reader(index))
        return out

    def flux(self):
        retime = np.exp(1j * np.pi * self.frequencies * self.dt)[:, None, None]
        total = np.zeros(self.frequencies.size)
        for pair, (e_spectrum, h_spectrum) in zip(self.pairs, self.spectra()):
            h_spectrum = h_spectrum * retime
            total += pair['sign'] * np.einsum('fij,ij->f', np.real(e_spectrum * np.conj(h_spectrum)), pair['area'])
        return np.cos(np.pi * self.frequencies * self.dt) * total


class FluxBox3D:
    """Net outward flux through the six cell-edge faces of a box (edge ranges per axis, inclusive)."""

    def __init__(self, edge_bounds, frequencies, dt, widths, shape, periodic=(False, False, False)):
        self.frequencies = check_frequencies(frequencies)
        self.edge_bounds = tuple(tuple(int(edge) for edge in bounds) for bounds in edge_bounds)
        self.faces = [(sign, PlaneFlux3D(axis, self.edge_bounds[axis][side], self.edge_bounds, self.frequencies, dt,
                                         widths, shape, periodic))
                      for axis in range(3) for side, sign in ((0, -1.0), (1, 1.0))]

    @property
    def sample_interval(self):
        return self.faces[0][1].sample_interval

    @sample_interval.setter
    def sample_interval(self, value):
        for _, plane in self.faces:
            plane.sample_interval = value

    def planes(self):
        return [plane for _, plane in self.faces]

    def flux(self):
        return sum(sign * plane.flux() for sign, plane in self.faces)
