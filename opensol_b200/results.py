"""Result dicts of the 2D monitors and the results.npz file open_sol's readers load.

The result dicts follow open_sol's monitor results (physics/em/results.py:109-151, core/monitors.py:284-288): a flux
line gives kind 'flux_spectrum' (frequency, wavelength, power, unit, mirror_factor and, when every source shares one
waveform, power_per_cw), a field map kind 'dft_fields' (centres, extent, shape, downsample, quantity, per-cw factor
and, at a frequency index, the float64 intensity), a probe kind 'timeseries'.  The normalising spectrum of the shared
waveform is its sampled DFT over the steps run on the monitor's sample grid (core/sources.py:103-139).

`save_results` writes a results directory in open_sol's layout (io/results_io.py:226-260): results.npz (metadata
'format' 'open_sol.results' version 1; result arrays under 'result/<key>/<name>', the other entries in the JSON
'metadata' member, io/results_io.py:399-436,517-535, io/model_io.py:564-589), log.txt and summary.json (its 'files'
lists what was written), so open_sol's load_results reads it.  All of this is host-side numpy on results the device
has already produced.
"""
import json
import math
import os
from pathlib import Path

import numpy as np

from .constants import C0
from .sources import ContinuousWave, RickerWavelet

__all__ = ['RESULTS_FORMAT', 'RESULTS_FORMAT_VERSION', 'WaveformSpectrumCache', 'dft_result', 'flux_result',
           'load_results', 'probe_result', 'probe_unit', 'results_arrays', 'sampled_waveform_spectrum',
           'save_results', 'simulation_results']

RESULTS_FORMAT = 'open_sol.results'
RESULTS_FORMAT_VERSION = 1
SUMMARY_FILE = 'summary.json'
LOG_FILE = 'log.txt'
ARRAYS_FILE = 'results.npz'

_DFT_QUANTITY = {'ez': 'abs(E_z)^2', 'hz': 'abs(E_x)^2 + abs(E_y)^2'}
_PROBE_UNITS = {'ez': 'V/m', 'ex': 'V/m', 'ey': 'V/m', 'hx': 'A/m', 'hy': 'A/m', 'hz': 'A/m'}
_VALID_SPECTRUM_FRACTION = 1e-6        # per-cw values are NaN where |S|^2 < this x |S(carrier)|^2
_SPECTRUM_CHUNK_ELEMENTS = 1 << 20     # complex128 phase-matrix elements summed per chunk
_NONFINITE_TEXT = {'nan': math.nan, 'inf': math.inf, '-inf': -math.inf}


# ---- normalising spectrum of the sources' waveform ----
def sampled_waveform_spectrum(temporal, dt, frequencies, first_step, last_step, sample_interval=1):
    """S(omega) = sum over the multiples n of m = sample_interval in [first_step, last_step] of s(n dt) e^{-j omega n dt}
    m dt, complex128 at `frequencies` [Hz] (core/sources.py:103-116; the same chunked sum, so the same rounding)."""
    m = int(sample_interval)
    first = -(-int(first_step) // m) * m
    times = np.arange(first, int(last_step) + 1, m, dtype=np.float64) * dt
    weighted = np.asarray(temporal(times), dtype=np.float64) * (dt * m)
    angular = -2.0 * np.pi * np.atleast_1d(np.asarray(frequencies, dtype=np.float64))
    spectrum = np.zeros(angular.size, dtype=np.complex128)
    chunk = max(1, _SPECTRUM_CHUNK_ELEMENTS // max(angular.size, 1))
    for start in range(0, times.size, chunk):
        spectrum += np.exp(1j * np.outer(angular, times[start:start + chunk])) @ weighted[start:start + chunk]
    return spectrum


class WaveformSpectrumCache:
    """sampled_waveform_spectrum over steps 1 .. n_step, kept per (waveform object, dt, frequencies, m): a later call
    adds only the steps run since, and starts over when n_step shrank or the waveform object changed
    (core/sources.py:119-139)."""

    def __init__(self):
        self._entries = {}

    def spectrum(self, temporal, dt, frequencies, n_step, sample_interval=1):
        frequencies = np.asarray(frequencies, dtype=np.float64)
        n_step, sample_interval = int(n_step), int(sample_interval)
        key = (id(temporal), float(dt), frequencies.tobytes(), sample_interval)
        owner, summed, spectrum = self._entries.get(key, (None, 0, None))
        if spectrum is None or owner is not temporal or n_step < summed:
            summed, spectrum = 0, np.zeros(frequencies.size, dtype=np.complex128)
        if n_step > summed:
            spectrum = spectrum + sampled_waveform_spectrum(temporal, dt, frequencies, summed + 1, n_step,
                                                            sample_interval)
        self._entries[key] = (temporal, n_step, spectrum)
        return spectrum.copy()


_SOURCE_SPECTRA = {}   # id(source) -> (source, WaveformSpectrumCache); the source is held so its id stays its own


def _waveform_spectrum(source, physics, frequencies, sample_interval):
    entry = _SOURCE_SPECTRA.get(id(source))
    if entry is None or entry[0] is not source:
        entry = _SOURCE_SPECTRA[id(source)] = (source, WaveformSpectrumCache())
    return entry[1].spectrum(source.temporal, float(physics.engine.dt), frequencies, physics.engine.n_step,
                             sample_interval)


def _carrier_angular_frequency(temporal):
    """2 pi f0 (f_peak of a Ricker wavelet) [rad/s] (physics/em/sources.py:395-398)."""
    frequency = temporal.f_peak if isinstance(temporal, RickerWavelet) else temporal.f0
    return 2.0 * np.pi * float(frequency)


def _normalizing_spectrum(source, physics, frequency, sample_interval):
    """(S(omega) of the source's waveform at `frequency`, valid mask): valid where |S|^2 >= 1e-6 |S(carrier)|^2 and,
    for a continuous wave, inside the main lobe |f - f0| < 1 / (n_step dt) (physics/em/results.py:66-78)."""
    spectrum = _waveform_spectrum(source, physics, frequency, sample_interval)
    carrier = _carrier_angular_frequency(source.temporal) / (2.0 * np.pi)
    carrier_power = float(np.abs(_waveform_spectrum(source, physics, [carrier], sample_interval)[0]) ** 2)
    valid = (np.abs(spectrum) ** 2 >= _VALID_SPECTRUM_FRACTION * carrier_power) & (carrier_power > 0.0)
    if isinstance(source.temporal, ContinuousWave):
        duration = physics.engine.n_step * float(physics.engine.dt)
        valid &= np.abs(frequency - source.temporal.f0) * duration < 1.0
    return spectrum, valid


def common_waveform(sources):
    """The waveform every source shares (same type and parameters), None without sources or when they differ."""
    sources = list(sources)
    if not sources:
        return None
    first = sources[0].temporal
    if any(type(source.temporal) is not type(first) or vars(source.temporal) != vars(first) for source in sources):
        return None
    return first


def _shared_waveform_spectrum(physics, frequency, sample_interval):
    sources = [] if physics is None else list(physics.sources)
    if common_waveform(sources) is None:
        return None
    return _normalizing_spectrum(sources[0], physics, frequency, sample_interval)


def _per_cw(values, spectrum, valid, factor=1.0):
    """values / (factor |S|^2) along the leading (frequency) axis, NaN where not valid."""
    scale = np.where(valid, 1.0 / (factor * np.where(valid, np.abs(spectrum) ** 2, 1.0)), np.nan)
    return np.asarray(values, dtype=np.float64) * scale.reshape(scale.shape + (1,) * (np.ndim(values) - 1))


# ---- result dicts ----
def _spectral_axes(monitor):
    frequency = np.array(monitor.frequencies, dtype=np.float64)
    return frequency, C0 / frequency


def flux_result(monitor, physics=None):
    """Flux spectrum of a FluxMonitor (power > 0 toward +x / +y, 'a.u.': dt-weighted spectra); with `physics` whose
    sources share one waveform also 'power_per_cw' [W/m] = power / (2 |S|^2).  'mirror_factor' is 1: the engines step
    no mirror faces, so no line has an image to count."""
    frequency, wavelength = _spectral_axes(monitor)
    result = {'kind': 'flux_spectrum', 'frequency': frequency, 'wavelength': wavelength,
              'power': 1.0 * monitor.flux(), 'unit': 'a.u.', 'mirror_factor': 1.0}
    shared = _shared_waveform_spectrum(physics, frequency, monitor.sample_interval)
    if shared is not None:
        result['power_per_cw'] = _per_cw(result['power'], *shared, factor=2.0)
    return result


def dft_result(monitor, domain, freq_index=None, physics=None):
    """Field-map result: sampled cell centres [m], box extent, shape, downsample, quantity; with `physics` whose sources
    share one waveform 'intensity_per_cw_factor' = 1 / |S|^2; an int freq_index adds float64 'intensity' = |E|^2 of
    that frequency (E_z, or |E_x|^2 + |E_y|^2 and 'hz_intensity' = |H_z|^2) and 'freq_index'."""
    frequency, wavelength = _spectral_axes(monitor)
    x_centers, y_centers = domain.cell_centers()
    x_edges, y_edges = domain.cell_edges()
    x_start, x_stop = monitor.x_slice.start or 0, monitor.x_slice.stop
    y_start, y_stop = monitor.y_slice.start or 0, monitor.y_slice.stop
    result = {'kind': 'dft_fields', 'frequency': frequency, 'wavelength': wavelength,
              'x_centers': np.array(x_centers[monitor.x_samples], dtype=np.float64),
              'y_centers': np.array(y_centers[monitor.y_samples], dtype=np.float64),
              'extent': (float(x_edges[x_start]), float(x_edges[x_stop]),
                         float(y_edges[y_start]), float(y_edges[y_stop])),
              'shape': (int(monitor.mx), int(monitor.my)), 'downsample': int(monitor.downsample),
              'quantity': _DFT_QUANTITY[monitor.polarization]}
    shared = _shared_waveform_spectrum(physics, frequency, monitor.sample_interval)
    if shared is not None:
        result['intensity_per_cw_factor'] = _per_cw(np.ones_like(frequency), *shared)
    if freq_index is not None:
        if isinstance(freq_index, bool) or not isinstance(freq_index, (int, np.integer)):
            raise TypeError(f"freq_index must be an int, got {freq_index!r}")
        if not 0 <= int(freq_index) < monitor.n_freqs:
            raise IndexError(f"freq_index {freq_index} out of range for {monitor.n_freqs} DFT frequencies")
        index = int(freq_index)
        result['freq_index'] = index

        def spectrum(name):
            return np.asarray(getattr(monitor, name)[index]).astype(np.complex128)
        if monitor.polarization == 'ez':
            result['intensity'] = np.abs(spectrum('ez_dft')) ** 2
        else:
            result['intensity'] = np.abs(spectrum('ex_dft')) ** 2 + np.abs(spectrum('ey_dft')) ** 2
            result['hz_intensity'] = np.abs(spectrum('hz_dft')) ** 2
    return result


def probe_unit(component):
    """'V/m' for an E component, 'A/m' for an H component."""
    return _PROBE_UNITS[component]


def probe_result(probe, unit=''):
    """Time series of a FieldProbe: 't' [s], float32 'values', component and unit."""
    times, values = probe.get_data()
    return {'kind': 'timeseries', 't': times, 'values': values, 'component': probe.field_component, 'unit': unit}


def simulation_results(sim, freq_index=0, physics_name='em'):
    """{'<physics>.flux<k>' / '.map<k>' / '.probe<k>': result dict} of every monitor of a Simulation's 2D physics, k
    counting each kind in the order the monitors were added; maps at `freq_index` (None: no intensity)."""
    from .monitors import DFTMonitor, FieldProbe, FluxMonitor
    physics = sim.em
    results, counts = {}, {'flux': 0, 'map': 0, 'probe': 0}

    def key(kind):
        name = f'{physics_name}.{kind}{counts[kind]}'
        counts[kind] += 1
        return name
    for monitor in physics.monitors:
        if isinstance(monitor, FluxMonitor):
            results[key('flux')] = flux_result(monitor, physics)
        elif isinstance(monitor, DFTMonitor):
            results[key('map')] = dft_result(monitor, physics.domain, freq_index=freq_index, physics=physics)
        elif isinstance(monitor, FieldProbe):
            results[key('probe')] = probe_result(monitor, probe_unit(monitor.field_component))
    return results


# ---- results directory ----
def _is_array(value):
    return isinstance(value, np.ndarray) and value.ndim >= 1 and value.dtype.kind in 'biufc'


def _name_part(key):
    text = str(key)
    if '/' in text:
        raise ValueError(f"result key {text!r} contains '/', which separates the levels of results.npz names")
    return text


def _json_safe(value):
    """Builtin JSON values: tuples as lists, non-finite floats as 'nan' / 'inf' / '-inf', numpy scalars as Python."""
    if value is None or isinstance(value, (bool, int, str)):
        return value
    if isinstance(value, np.generic):
        return _json_safe(value.item())
    if isinstance(value, float):
        if math.isfinite(value):
            return value
        return 'nan' if math.isnan(value) else ('inf' if value > 0 else '-inf')
    if isinstance(value, dict):
        return {str(k): _json_safe(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [_json_safe(v) for v in value]
    if isinstance(value, np.ndarray):
        return _json_safe(value.tolist())
    if isinstance(value, os.PathLike):
        return os.fspath(value)
    raise TypeError(f'{type(value).__name__} is not JSON serialisable')


def results_arrays(results):
    """(npz arrays, metadata) of {key: result dict}: >= 1-D numeric arrays under 'result/<key>/<name>' (one level of
    nested dict: 'result/<key>/<entry>/<name>'), every other entry in metadata['results'][key]."""
    arrays = {}
    metadata = {'format': RESULTS_FORMAT, 'version': RESULTS_FORMAT_VERSION, 'fields': {}, 'results': {},
                'sweep_results': [], 'sector_results': [], 'sector_combined_results': {}, 'snapshots': [],
                'sweep_snapshots': []}
    for key, result in results.items():
        prefix = f'result/{_name_part(key)}/'
        entries = {}
        for name, value in result.items():
            if _is_array(value):
                arrays[prefix + _name_part(name)] = value
            elif isinstance(value, dict) and any(_is_array(item) for item in value.values()):
                entries[name] = {k: v for k, v in value.items() if not _is_array(v)}
                for k, v in value.items():
                    if _is_array(v):
                        arrays[f'{prefix}{_name_part(name)}/{_name_part(k)}'] = v
            else:
                entries[name] = value
        metadata['results'][key] = entries
    return arrays, _json_safe(metadata)


def _write_npz(path, arrays, metadata):
    if 'metadata' in arrays:
        raise ValueError("array key 'metadata' clashes with the .npz metadata entry")
    entries = dict(arrays, metadata=np.array(json.dumps(metadata)))
    with open(path, 'wb') as handle:   # a file object: numpy appends no '.npz'
        np.savez(handle, **entries)


def save_results(directory, results, log_lines=(), summary=None):
    """Write results.npz, log.txt and, last, summary.json (summary plus 'files') into `directory` (created); an old
    summary.json is removed first, so a directory with a summary lists complete files only.  Returns the files dict."""
    directory = Path(directory)
    directory.mkdir(parents=True, exist_ok=True)
    (directory / SUMMARY_FILE).unlink(missing_ok=True)
    summary = dict(summary or {})
    files = {'summary': SUMMARY_FILE, 'log': LOG_FILE, 'arrays': ARRAYS_FILE, 'meshes': None, 'model': None,
             'figures': []}
    summary['files'] = files
    arrays, metadata = results_arrays(results)
    _write_npz(directory / ARRAYS_FILE, arrays, metadata)
    (directory / LOG_FILE).write_text(''.join(f'{line}\n' for line in log_lines), encoding='utf-8', newline='\n')
    partial = directory / (SUMMARY_FILE + '.partial')
    partial.write_text(json.dumps(_json_safe(summary), indent=1), encoding='utf-8')
    os.replace(partial, directory / SUMMARY_FILE)
    return files


def _restore_nonfinite(value):
    if isinstance(value, str) and value in _NONFINITE_TEXT:
        return _NONFINITE_TEXT[value]
    return value


def read_results_npz(path):
    """{key: result dict} of a results.npz (arrays joined back into their result dicts, nested names into their
    entry's dict, in archive order); ValueError for another format or version."""
    with np.load(path, allow_pickle=False) as npz:
        metadata = json.loads(str(npz['metadata']))
        if metadata.get('format') != RESULTS_FORMAT or metadata.get('version') != RESULTS_FORMAT_VERSION:
            raise ValueError(f"{path}: format {metadata.get('format')!r} version {metadata.get('version')!r} is not "
                             f"{RESULTS_FORMAT!r} version {RESULTS_FORMAT_VERSION}")
        results = {key: {name: _restore_nonfinite(value) for name, value in entries.items()}
                   for key, entries in metadata['results'].items()}
        for array_name in npz.files:
            levels = array_name.split('/')
            if levels[0] != 'result' or len(levels) < 3 or levels[1] not in results:
                continue
            if len(levels) == 3:
                results[levels[1]][levels[2]] = npz[array_name]
            else:
                results[levels[1]].setdefault(levels[2], {})['/'.join(levels[3:])] = npz[array_name]
    return results


def load_results(directory):
    """(summary, {key: result dict}, log lines) of a results directory; FileNotFoundError without summary.json."""
    directory = Path(directory)
    summary_path = directory / SUMMARY_FILE
    if not summary_path.is_file():
        raise FileNotFoundError(f'{summary_path} not found: {directory} is not an open_sol results directory')
    summary = json.loads(summary_path.read_text(encoding='utf-8'))
    files = summary.get('files') if isinstance(summary.get('files'), dict) else {}
    results = {}
    if files.get('arrays') and (directory / files['arrays']).is_file():
        results = read_results_npz(directory / files['arrays'])
    log_path = directory / LOG_FILE
    log_lines = log_path.read_text(encoding='utf-8').splitlines() if log_path.is_file() else []
    return summary, results, log_lines
