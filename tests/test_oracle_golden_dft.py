"""Pin the oracle's field-map (running DFT) monitors and field probes to open_sol itself: the fixtures of
tests/golden/dft_*.npz (generated by running the reference's CPU backend, see tests/golden/make_golden_dft.py) must be
reproduced bit for bit -- the complex64 maps at every checkpoint, the sample boxes, the flux line spectra, the fields'
digests and the probes' times and values."""
import hashlib
import os

import numpy as np
import pytest

from cases import apply_ops
from cases_dft import CASES_DFT
from oracle.fdtd2d import OracleEz2D

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_oracle_dft(spec):
    """(oracle, {checkpoint: ([map spectra], [flux E spectra], {field: digest})}) of a case."""
    o = OracleEz2D(**spec['sim'])
    fluxes = apply_ops(o, spec)
    maps = [o.add_dft_monitor(x0, y0, x1, y1, frequencies=f, downsample=ds) for x0, y0, x1, y1, f, ds in spec['dft']]
    o.probe_records = [o.add_field_probe(x, y, comp) for x, y, comp in spec.get('probes', [])]
    snaps = {}
    done = 0
    for cp in spec['checkpoints']:
        o.run(n_steps=cp - done)
        done = cp
        snaps[cp] = ([m.ez_dft.copy() for m in maps], [m.e_acc.copy() for m in fluxes],
                     {n: _digest(getattr(o, n)) for n in ('ez', 'hx', 'hy')})
    return o, maps, snaps


@pytest.mark.parametrize('spec', CASES_DFT, ids=[c['name'] for c in CASES_DFT])
def test_oracle_maps_match_reference(spec):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    o, maps, snaps = run_oracle_dft(spec)
    assert int(g['sample_interval']) == o.sample_interval
    for k, mon in enumerate(maps):
        xs, ys = mon.x_samples, mon.y_samples
        assert [xs.start, xs.stop, mon.downsample, mon.ez_dft.shape[1], ys.start, ys.stop, mon.ez_dft.shape[2]] == \
            g[f'map{k}_box'].tolist()
    for cp, (spectra, flux_e, digests) in snaps.items():
        for name, d in digests.items():
            assert d == str(g[f'sha_{name}_{cp}']), f'{name} at step {cp}'
        for k, spec_k in enumerate(spectra):
            ref = g[f'map{k}_{cp}']
            assert ref.dtype == np.complex64 and spec_k.shape == ref.shape
            np.testing.assert_array_equal(spec_k, ref)
            assert np.abs(ref).max() > 0   # the map saw the pulse
        for k, e in enumerate(flux_e):
            np.testing.assert_array_equal(e, g[f'spec_e{k}_{cp}'])


@pytest.mark.parametrize('spec', CASES_DFT, ids=[c['name'] for c in CASES_DFT])
def test_oracle_probes_match_reference(spec):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    o, _, _ = run_oracle_dft(spec)
    for k, (ix, iy, _, times, values) in enumerate(o.probe_records):
        assert [ix, iy] == g[f'probe{k}_cell'].tolist()
        np.testing.assert_array_equal(np.array(times), g[f'probe{k}_t'])
        np.testing.assert_array_equal(np.array(values, dtype=np.float32), g[f'probe{k}_v'])
        assert np.abs(g[f'probe{k}_v']).max() > 0
