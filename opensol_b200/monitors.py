"""Flux monitors, field-map DFT monitors and the DFT sampling rule of the B200 engines.

The running DFTs live on the device as float64 (complex128) sums, exactly like open_sol's line spectra
(open_sol/physics/em/monitors.py:84-96): each term is a float32 phase times a float32 field sample, which is exact in
float64, so the device sums equal the reference's.  Phases exp(-j omega t) m dt are computed on the host in float64
and rounded to complex64 (monitors.py:22-24) into a per-sample table the kernels read.
"""
from __future__ import annotations

import numpy as np


def check_frequencies(frequencies, label='frequencies'):
    """Non-empty 1D float64 copy of finite positive values (monitors.py:194-200)."""
    frequencies = np.atleast_1d(np.array(frequencies, dtype=np.float64))
    if frequencies.ndim != 1 or frequencies.size == 0 or not np.all(np.isfinite(frequencies) & (frequencies > 0)):
        raise ValueError(f"monitor {label} must be a non-empty 1D list of finite positive values, got {frequencies}")
    return frequencies


def resolve_frequencies(wavelengths, frequencies):
    """Monitor frequencies [Hz] from exactly one of wavelengths [m] / frequencies [Hz] (physics/em/__init__.py:571)."""
    from .constants import C0
    if (wavelengths is None) == (frequencies is None):
        raise ValueError("pass exactly one of wavelengths or frequencies")
    if frequencies is not None:
        return check_frequencies(frequencies)
    return C0 / check_frequencies(wavelengths, 'wavelengths')


def dft_sample_interval(dt, sources, monitor_frequencies, harmonic_order=1) -> int:
    """Largest m with 1/(m dt) >= max monitor frequency + harmonic_order x the sources' spectral limit
    (monitors.py:177-191); 1 for a source without a spectral limit or without monitors."""
    if not sources or not monitor_frequencies:
        return 1
    limits = []
    for source in sources:
        spectral_limit = getattr(getattr(source, 'temporal', None), 'spectral_limit', None)
        limit = spectral_limit() if spectral_limit is not None else None
        if limit is None:
            return 1
        limits.append(float(limit))
    sample_rate = float(harmonic_order) * max(limits) + max(float(np.max(f)) for f in monitor_frequencies)
    return max(1, int(np.floor(1.0 / (sample_rate * float(dt)))))


def dft_phase_table(omega, times, dt_m):
    """(n_samples, nf, 2) float32 table of complex64 exp(-j omega t) * dt_m per sample time (monitors.py:22-24)."""
    table = np.empty((len(times), omega.size, 2), dtype=np.float32)
    for q, t in enumerate(times):
        phase = -omega * float(t)
        table[q, :, 0] = (np.cos(phase) * float(dt_m)).astype(np.float32)
        table[q, :, 1] = (np.sin(phase) * float(dt_m)).astype(np.float32)
    return table


class FluxMonitor:
    """Spectral Poynting flux through the hi face of a line of cells (physics/em/monitors.py:325-379): axis = the
    monitor's normal ('x': a line of constant x-cell `position`; 'y': of constant y-cell), > 0 toward +axis.  E_z with
    H_y / H_x for polarisation 'ez'; E_y / E_x on the hi faces with H_z for 'hz'.  The spectra are read from the
    engine's device sums when flux() is called."""

    def __init__(self, axis, position, span, frequencies, dt, cell_widths, polarization='ez'):
        if polarization not in ('ez', 'hz'):
            raise ValueError(f"FluxMonitor polarization must be 'ez' or 'hz', got {polarization!r}")
        if axis not in ('x', 'y'):
            raise ValueError(f"FluxMonitor axis must be 'x' or 'y', got {axis!r}")
        span = (int(span[0]), int(span[1]))
        if not 0 <= span[0] < span[1]:
            raise ValueError(f"FluxMonitor span must be a half-open cell range lo < hi, got {span}")
        cell_widths = np.asarray(cell_widths, dtype=np.float64)
        if cell_widths.ndim != 1 or cell_widths.size < span[1]:
            raise ValueError(f"FluxMonitor cell_widths (shape {cell_widths.shape}) must cover span {span}")
        self.axis = axis
        self.position = int(position)
        self.span = span
        self.frequencies = check_frequencies(frequencies)
        self.dt = float(dt)
        self.n_freqs = len(self.frequencies)
        self.polarization = polarization
        # ez: S_x = -E_z H_y, S_y = +E_z H_x; hz: S_x = +E_y H_z, S_y = -E_x H_z (monitors.py:350-362)
        self._flux_sign = (-1.0 if axis == 'x' else 1.0) if polarization == 'ez' else (1.0 if axis == 'x' else -1.0)
        self._cell_widths = cell_widths[span[0]:span[1]].copy()
        self.sample_interval = 1
        self._reader = None   # () -> (e_spectra, h_spectra) complex128 (nf, n), set by the engine

    @property
    def n_cells(self):
        return self.span[1] - self.span[0]

    def spectra(self):
        """(E, H) complex128 (nf, n_cells) running DFTs, both phased at the E sample time (H not yet re-timed)."""
        if self._reader is None:
            return (np.zeros((self.n_freqs, self.n_cells), np.complex128),
                    np.zeros((self.n_freqs, self.n_cells), np.complex128))
        return self._reader()

    def flux(self):
        """(n_freqs,) float64 power per unit length: sign cos(omega dt/2) Re(E conj(H e^{j pi f dt})) summed over the
        line widths (monitors.py:371-379)."""
        e_spectra, h_spectra = self.spectra()
        h_spectra = h_spectra * np.exp(1j * np.pi * self.frequencies * self.dt)[:, None]
        e_time_average = np.cos(np.pi * self.frequencies * self.dt)
        integrand = self._flux_sign * e_time_average[:, None] * np.real(e_spectra * np.conj(h_spectra))
        return integrand @ self._cell_widths


def dft_sample_slice(start: int, stop: int, stride: int) -> slice:
    """Cells a DFTMonitor samples along one axis of the box [start, stop): every stride-th cell from the middle of the
    first stride-cell block (monitors.py:152-155)."""
    return slice(start + min(stride, stop - start) // 2, stop, stride)


class DFTMonitor:
    """Running DFT over the cell box (x_slice, y_slice) at each frequency (physics/em/monitors.py:248-322): E_z
    ('ez', ez_dft), or H_z plus E_x / E_y collocated to the cell centres ('hz', hz_dft / ex_dft / ey_dft; the partner
    face of cell 0 wraps on a periodic axis), += phase_f * sample at every DFT sample step, complex64 sums on the
    device; downsample s > 1 records every s-th cell along x and y (x_samples / y_samples)."""

    def __init__(self, x_slice, y_slice, frequencies, dt, polarization='ez', downsample=1):
        for label, cells in (('x_slice', x_slice), ('y_slice', y_slice)):
            if cells.step not in (None, 1) or cells.stop is None or not (cells.start or 0) < cells.stop:
                raise ValueError(f"DFTMonitor {label} must be a non-empty unit-step slice, got {cells}")
        if isinstance(downsample, bool) or int(downsample) != downsample or downsample < 1:
            raise ValueError(f"DFTMonitor downsample must be an int >= 1, got {downsample!r}")
        if polarization not in ('ez', 'hz'):
            raise ValueError(f"DFTMonitor polarization must be 'ez' or 'hz', got {polarization!r}")
        self.polarization = polarization
        self.x_slice = x_slice
        self.y_slice = y_slice
        self.downsample = int(downsample)
        self.x_samples = dft_sample_slice(x_slice.start or 0, x_slice.stop, self.downsample)
        self.y_samples = dft_sample_slice(y_slice.start or 0, y_slice.stop, self.downsample)
        self.frequencies = check_frequencies(frequencies)
        self.dt = float(dt)
        self.n_freqs = len(self.frequencies)
        self.mx = len(range(self.x_samples.start, self.x_samples.stop, self.downsample))
        self.my = len(range(self.y_samples.start, self.y_samples.stop, self.downsample))
        self.sample_interval = 1
        self._reader = None   # () -> complex64 (nf, mx, my), set by the engine

    def _maps(self):
        parts = 1 if self.polarization == 'ez' else 3
        if self._reader is None:
            maps = np.zeros((parts, self.n_freqs, self.mx, self.my), np.complex64)
            return maps[0] if parts == 1 else maps
        return self._reader()

    @property
    def ez_dft(self):
        """(n_freqs, mx, my) complex64 running DFT of E_z (read from the device)."""
        if self.polarization != 'ez':
            raise AttributeError("an 'hz' DFTMonitor has hz_dft, ex_dft and ey_dft")
        return self._maps()

    @property
    def hz_dft(self):
        if self.polarization != 'hz':
            raise AttributeError("an 'ez' DFTMonitor has ez_dft")
        return self._maps()[0]

    @property
    def ex_dft(self):
        if self.polarization != 'hz':
            raise AttributeError("an 'ez' DFTMonitor has ez_dft")
        return self._maps()[1]

    @property
    def ey_dft(self):
        if self.polarization != 'hz':
            raise AttributeError("an 'ez' DFTMonitor has ez_dft")
        return self._maps()[2]


PROBE_COMPONENTS = {'ez': ('ez', 'hx', 'hy'), 'hz': ('hz', 'ex', 'ey')}


class FieldProbe:
    """One field component at cell (ix, iy), recorded after every step (core/monitors.py:194-243): get_data() gives
    (times float64, values float32) since the probe was added or the engine was last reset; the values are recorded
    on the device and read in one transfer."""

    def __init__(self, ix, iy, field_component='ez'):
        self.ix = int(ix)
        self.iy = int(iy)
        self.field_component = field_component
        self._reader = None   # () -> (times, values), set by the engine

    def get_data(self):
        if self._reader is None:
            return np.empty(0, np.float64), np.empty(0, np.float32)
        return self._reader()
