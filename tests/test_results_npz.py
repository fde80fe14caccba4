"""results.npz in open_sol's layout.  The fixtures tests/golden/results_<case>.npz were written by open_sol's own
results writer from its monitors' result dicts after a reference run (tests/golden/make_golden_results.py).

CPU: reading a fixture and writing it back gives the same archive members in the same order, the same dtypes and
values and the same metadata JSON, and a results directory round-trips.  GPU: the engine's monitors, run on the same
case, give result dicts equal to the fixture's bit for bit (spectra, intensities, per-cw normalisation, probe series)
and the archive save_results writes equals the fixture's."""
import json
import os

import numpy as np
import pytest

from cases_dft import case

from opensol_b200 import results as res

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
CASES = ('dft_pml', 'dft_hz_pml')


def _fixture(name):
    return os.path.join(GOLDEN, f'results_{name}.npz')


def _assert_same_archive(path, reference_path):
    with np.load(path, allow_pickle=False) as got, np.load(reference_path, allow_pickle=False) as want:
        assert got.files == want.files
        assert json.loads(str(got['metadata'])) == json.loads(str(want['metadata']))
        assert str(got['metadata']) == str(want['metadata'])
        for name in want.files:
            assert got[name].dtype == want[name].dtype, name
            np.testing.assert_array_equal(got[name], want[name], err_msg=name)


@pytest.mark.parametrize('name', CASES)
def test_fixture_round_trips_through_reader_and_writer(name, tmp_path):
    results = res.read_results_npz(_fixture(name))
    kinds = {key: r['kind'] for key, r in results.items()}
    assert kinds['em.flux0'] == 'flux_spectrum' and kinds['em.map0'] == 'dft_fields'
    assert kinds['em.probe0'] == 'timeseries'
    files = res.save_results(tmp_path / 'run', results, log_lines=['line one', 'line two'], summary={'n_step': 500})
    assert files['arrays'] == 'results.npz'
    _assert_same_archive(tmp_path / 'run' / 'results.npz', _fixture(name))
    summary, loaded, log_lines = res.load_results(tmp_path / 'run')
    assert summary['n_step'] == 500 and summary['files'] == files
    assert log_lines == ['line one', 'line two']
    for key, result in results.items():
        assert set(loaded[key]) == set(result)
        for entry, value in result.items():
            if isinstance(value, np.ndarray):
                np.testing.assert_array_equal(loaded[key][entry], value)
            else:
                assert loaded[key][entry] == value


def test_nonfinite_entries_and_nested_arrays_round_trip(tmp_path):
    results = {'em.x': {'kind': 'xy', 'series': {'a': np.arange(3.0), 'label': 'q'}, 'peak': float('nan'),
                        'edge': float('-inf'), 'shape': (2, 3)}}
    arrays, metadata = res.results_arrays(results)
    assert list(arrays) == ['result/em.x/series/a']
    assert metadata['results']['em.x'] == {'kind': 'xy', 'series': {'label': 'q'}, 'peak': 'nan', 'edge': '-inf',
                                           'shape': [2, 3]}
    res.save_results(tmp_path, results)
    _, loaded, _ = res.load_results(tmp_path)
    got = loaded['em.x']
    assert np.isnan(got['peak']) and got['edge'] == -np.inf and got['shape'] == [2, 3]
    np.testing.assert_array_equal(got['series']['a'], np.arange(3.0))
    assert got['series']['label'] == 'q'


def test_writer_refuses_bad_keys_and_reader_other_formats(tmp_path):
    with pytest.raises(ValueError, match="separates the levels"):
        res.results_arrays({'em/a': {'kind': 'x'}})
    np.savez(tmp_path / 'other.npz', metadata=np.array(json.dumps({'format': 'other', 'version': 1})))
    with pytest.raises(ValueError, match='is not'):
        res.read_results_npz(tmp_path / 'other.npz')
    with pytest.raises(FileNotFoundError):
        res.load_results(tmp_path / 'missing')


def test_sampled_waveform_spectrum_cache_adds_only_new_steps():
    """A cached spectrum extended over later steps is the sum of the two ranges; a shorter n_step starts over."""
    from opensol_b200.sources import GaussianPulse
    pulse = GaussianPulse(4.5e14, 0.5)
    freqs = np.array([4.0e14, 5.0e14])
    dt = 5e-17
    cache = res.WaveformSpectrumCache()
    first = cache.spectrum(pulse, dt, freqs, 300, 2)
    np.testing.assert_array_equal(first, res.sampled_waveform_spectrum(pulse, dt, freqs, 1, 300, 2))
    both = cache.spectrum(pulse, dt, freqs, 700, 2)
    np.testing.assert_array_equal(both, first + res.sampled_waveform_spectrum(pulse, dt, freqs, 301, 700, 2))
    np.testing.assert_array_equal(cache.spectrum(pulse, dt, freqs, 100, 2),
                                  res.sampled_waveform_spectrum(pulse, dt, freqs, 1, 100, 2))
    # the DFT sum itself: sum over multiples of m of s(n dt) e^{-j w n dt} m dt
    n = np.arange(2, 301, 2)
    direct = np.array([np.sum(pulse(n * dt) * np.exp(-2j * np.pi * f * n * dt)) * 2 * dt for f in freqs])
    np.testing.assert_allclose(first, direct, rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize('name', CASES)
def test_engine_results_equal_reference_results(name, tmp_path):
    from cases import apply_ops
    from cases_dft import apply_poles
    import opensol_b200 as ob
    spec = case(name)
    sim = ob.Simulation(**spec['sim'], verbose=False)
    apply_ops(sim, spec)
    apply_poles(sim.em, spec, ob.DrudePole, ob.LorentzPole, sim.em.domain.circle_mask)
    for x0, y0, x1, y1, f, ds in spec['dft']:
        sim.em.add_dft_monitor(x0, y0, x1, y1, frequencies=f, downsample=ds)
    for x, y, comp in spec['probes']:
        sim.em.add_field_probe(x, y, comp)
    sim.run(n_steps=spec['checkpoints'][-1], verbose=False, print_every=0)
    got = res.simulation_results(sim, freq_index=0)
    want = res.read_results_npz(_fixture(name))
    assert list(got) == list(want)
    for key, result in want.items():
        assert set(got[key]) == set(result), key
        for entry, value in result.items():
            if isinstance(value, np.ndarray):
                assert np.asarray(got[key][entry]).dtype == value.dtype, (key, entry)
                np.testing.assert_array_equal(got[key][entry], value, err_msg=f'{key} {entry}')
            else:
                assert res._json_safe(got[key][entry]) == value, (key, entry)
    res.save_results(tmp_path, got)
    _assert_same_archive(tmp_path / 'results.npz', _fixture(name))
    sim.em.engine.close()


class _FakeEngine:
    def __init__(self, dt, n_step):
        self.dt, self.n_step = dt, n_step


class _FakeSource:
    def __init__(self, temporal):
        self.temporal = temporal


class _FakePhysics:
    def __init__(self, sources, dt=5e-17, n_step=2000):
        self.sources, self.engine = sources, _FakeEngine(dt, n_step)


class _FakeFlux:
    def __init__(self, frequencies, power):
        self.frequencies, self._power, self.sample_interval = np.asarray(frequencies), np.asarray(power), 2

    def flux(self):
        return self._power


def test_flux_result_normalisation_branches():
    """power_per_cw = power / (2 |S|^2) of the shared waveform's sampled spectrum; NaN where |S|^2 is below 1e-6 of
    the carrier's; a continuous wave keeps only its main lobe; sources with different waveforms give no per-cw entry."""
    from opensol_b200.sources import ContinuousWave, GaussianPulse
    pulse = GaussianPulse(4.5e14, 0.3)
    freqs = [4.5e14, 4.6e14, 1.5e15]                  # the last far outside the pulse's band
    physics = _FakePhysics([_FakeSource(pulse), _FakeSource(GaussianPulse(4.5e14, 0.3))])
    mon = _FakeFlux(freqs, [2.0, 1.0, 0.5])
    result = res.flux_result(mon, physics)
    assert result['kind'] == 'flux_spectrum' and result['mirror_factor'] == 1.0
    s = res.sampled_waveform_spectrum(pulse, 5e-17, freqs, 1, 2000, 2)
    np.testing.assert_allclose(result['power_per_cw'][:2], np.array([2.0, 1.0]) / (2 * np.abs(s[:2]) ** 2),
                               rtol=1e-12)
    assert np.isnan(result['power_per_cw'][2])
    mixed = _FakePhysics([_FakeSource(pulse), _FakeSource(GaussianPulse(5e14, 0.3))])
    assert 'power_per_cw' not in res.flux_result(mon, mixed)
    cw = ContinuousWave(4.5e14)
    run = _FakePhysics([_FakeSource(cw)], n_step=2000)   # 100 fs: main lobe |f - f0| < 1e13 Hz
    out = res.flux_result(_FakeFlux([4.5e14, 4.7e14], [1.0, 1.0]), run)['power_per_cw']
    assert np.isfinite(out[0]) and np.isnan(out[1])
