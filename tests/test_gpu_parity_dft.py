"""GPU parity of the field-map (running DFT) monitors and field probes of the 2D E_z and H_z engines, through the C
ABI, against open_sol's own outputs (tests/golden/dft_*.npz) and the oracle.  Bar: bit-identical complex64 maps and float32 probe
values (array_equal), for every kernel variant and for chunk boundaries that do and do not fall on sample steps."""
import hashlib
import os

import numpy as np
import pytest

from cases import apply_ops
from cases_dft import CASES_DFT, CASES_DFT_HZ, apply_poles
from test_oracle_golden_dft import field_names, map_keys, map_parts, run_oracle_dft

import opensol_b200 as ob
from opensol_b200 import serving

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
CONFIGS = [(1, 3, 0), (1, 2, 8), (1, 4, 16), (2, 3, 0), (0, 1, 0)]   # (variant, steps per launch, tile rows)
CONFIGS_HZ = [(1, 1, 0), (1, 1, 16), (0, 1, 0), (1, 2, 0)]
FIXTURE_RUNS = ([(spec, c) for spec in CASES_DFT for c in CONFIGS] + [(spec, c) for spec in CASES_DFT_HZ
                                                                      for c in CONFIGS_HZ])


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _build(spec, config):
    sim = ob.Simulation(**spec['sim'], verbose=False)
    fluxes = apply_ops(sim, spec)
    apply_poles(sim.em, spec, ob.DrudePole, ob.LorentzPole, sim.em.domain.circle_mask)
    maps = [sim.em.add_dft_monitor(x0, y0, x1, y1, frequencies=f, downsample=ds)
            for x0, y0, x1, y1, f, ds in spec['dft']]
    sim.probes = [sim.em.add_field_probe(x, y, comp) for x, y, comp in spec.get('probes', [])]
    sim.em.engine.configure(variant=config[0], steps_per_launch=config[1], tile_rows=config[2])
    return sim, fluxes, maps


@pytest.mark.parametrize('spec,config', FIXTURE_RUNS,
                         ids=[f"{sp['name']}-v{c[0]}_T{c[1]}_r{c[2]}" for sp, c in FIXTURE_RUNS])
def test_maps_bit_exact_against_reference(spec, config):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    sim, fluxes, maps = _build(spec, config)
    done = 0
    for cp in spec['checkpoints']:
        sim.run(n_steps=cp - done, verbose=False, print_every=0)
        done = cp
        for name in field_names(spec):
            assert _digest(sim.em.engine.read_field(name)) == str(g[f'sha_{name}_{cp}']), f'{name} at {cp}'
        for k, mon in enumerate(maps):
            for got, key in zip(map_parts(mon), map_keys(spec, k, cp)):
                assert got.dtype == np.complex64
                np.testing.assert_array_equal(got, g[key])
        for k, mon in enumerate(fluxes):
            np.testing.assert_array_equal(mon.spectra()[0], g[f'spec_e{k}_{cp}'])
    for k, probe in enumerate(sim.probes):
        times, values = probe.get_data()
        assert [probe.ix, probe.iy] == g[f'probe{k}_cell'].tolist()
        np.testing.assert_array_equal(times, g[f'probe{k}_t'])
        np.testing.assert_array_equal(values, g[f'probe{k}_v'])
    sim.em.engine.close()


def test_hz_probes_record_every_step():
    """H_z engine: the probes' values equal the fields read back after each single step."""
    from cases_hz import HZ_CASES
    spec = HZ_CASES[0]
    sim = ob.Simulation(**spec['sim'], verbose=False)
    apply_ops(sim, spec)
    eng = sim.em.engine
    cells = [(0.4e-6, 0.5e-6, 'hz'), (0.6e-6, 0.3e-6, 'ex'), (0.5e-6, 0.7e-6, 'ey')]
    probes = [sim.em.add_field_probe(x, y, c) for x, y, c in cells]
    sim.em.finalize()
    expected = [[] for _ in probes]
    for _ in range(40):
        eng.advance(1)
        for k, p in enumerate(probes):
            expected[k].append(eng.read_field(p.field_component)[p.ix, p.iy])
    eng.advance(25)   # and a longer chunk
    for k, p in enumerate(probes):
        times, values = p.get_data()
        assert values.shape == (65,) and times.shape == (65,)
        np.testing.assert_array_equal(values[:40], np.array(expected[k], dtype=np.float32))
        np.testing.assert_array_equal(times[-1], eng.time)
    final = [eng.read_field(p.field_component)[p.ix, p.iy] for p in probes]
    assert [p.get_data()[1][-1] for p in probes] == final
    eng.close()


def _ez_probe_run(config, n_probes, flux, chunks, late=None):
    """An E_z run on a 136 x 496 grid (CPML 8) whose probes sit in the interior box, in the CPML slabs and on the grid
    corners; `late` (a chunk index) adds one more probe, near the interior box's edge, after that chunk.  (probe data,
    launches per chunk, interior cells of the plan)."""
    from opensol_b200.monitors import FieldProbe
    spec = {'sim': {'size_x': 3.0e-6, 'size_y': 12.0e-6, 'dx': 25e-9, 'npml': 8, 'boundaries': 'pml'},
            'ops': [['add_dielectric_circle', [1.5e-6, 6.0e-6, 0.6e-6], {'eps_r': 4.0}],
                    ['add_line_source', ['y', 0.6e-6], {'wavelength': 700e-9, 'bandwidth': 0.6}]]}
    if flux:
        spec['ops'].append(['add_flux_monitor', ['y', 2.4e-6, [0.5e-6, 11.0e-6]],
                            {'wavelengths': [650e-9, 750e-9]}])
    sim = ob.Simulation(**spec['sim'], verbose=False)
    apply_ops(sim, spec)
    eng = sim.em.engine
    nx, ny = eng.nx, eng.ny
    cells = [(nx // 2, ny // 2, 'ez'), (nx // 2 + 1, 250, 'hx'), (40, 300, 'hy'), (3, 100, 'ez'),
             (nx // 2, 2, 'hy'), (0, 0, 'ez'), (nx - 1, ny - 1, 'hx')][:n_probes]
    probes = []
    for ix, iy, comp in cells:
        probes.append(FieldProbe(ix, iy, comp))
        eng.attach_probe(probes[-1])
    eng.configure(variant=config[0], steps_per_launch=config[1], tile_rows=config[2])
    sim.em.finalize()
    launches = []
    for k, n in enumerate(chunks):
        eng.advance(n)
        launches.append(eng.launch_count())
        if late is not None and k == late:
            probes.append(FieldProbe(11, 130, 'hy'))
            eng.attach_probe(probes[-1])
    out = [p.get_data() for p in probes]
    interior = eng.plan_info()[0]
    eng.close()
    return out, launches, interior


EZ_PROBE_CONFIGS = [(1, 3, 0), (1, 4, 16), (1, 2, 8), (2, 3, 0)]


@pytest.mark.parametrize('config', EZ_PROBE_CONFIGS, ids=[f'v{c[0]}_T{c[1]}_r{c[2]}' for c in EZ_PROBE_CONFIGS])
@pytest.mark.parametrize('n_probes,flux', [(7, False), (6, True), (7, True)],
                         ids=['8probes', '7probes_flux', '8probes_flux_one_step'])
def test_ez_probes_in_blocked_launches(config, n_probes, flux):
    """E_z probes are staged by the blocked kernels at every step of a launch (interior, frame and general tiles):
    the values equal a one-step-per-launch run's of the same kernel variant, which reads each probe's cell from the
    field after every step.  A
    probe is added between chunks.  Eight probes and a flux line exceed the monitors a launch stages: from then on
    that run keeps one step per launch."""
    chunks = [7, 13, 1, 40, 9]
    ref, ref_launches, _ = _ez_probe_run((config[0], 1, config[2]), n_probes, flux, chunks, late=1)
    got, launches, interior = _ez_probe_run(config, n_probes, flux, chunks, late=1)
    if config[0] == 1:
        assert interior > 0, 'the plan has no interior box: the interior kernel is not exercised'
    for (t0, v0), (t1, v1) in zip(ref, got):
        assert v0.shape == v1.shape and v0.shape[0] > 0
        np.testing.assert_array_equal(t1, t0)
        np.testing.assert_array_equal(v1, v0)
    assert got[-1][1].shape == (sum(chunks) - sum(chunks[:2]),)   # the late probe records from its step on
    assert launches[0] < ref_launches[0]   # before the late probe: blocked launches
    if n_probes + 1 + flux <= 8:
        assert launches[3] < ref_launches[3]
    else:
        assert launches[3] == ref_launches[3]


@pytest.mark.parametrize('seed', [0, 1, 2])
def test_random_maps_and_chunks_match_oracle(seed):
    """Seeded boxes and downsample factors; the run advances in chunks of random length, so chunk ends fall both on
    and between DFT sample steps."""
    rng = np.random.default_rng(100 + seed)
    spec = {'sim': {'size_x': 1.4e-6, 'size_y': 1.1e-6, 'dx': 25e-9, 'npml': 8,
                    'boundaries': ['pml', 'periodic_x', 'periodic_y'][seed]},
            'ops': [['add_dielectric_circle', [0.7e-6, 0.55e-6, 0.25e-6], {'eps_r': 3.0}],
                    ['add_line_source', ['y' if seed != 2 else 'x', 0.3e-6], {'wavelength': 700e-9,
                                                                              'bandwidth': 0.6}],
                    ['add_flux_monitor', ['y', 1.0e-6, [0.1e-6, 1.0e-6]], {'wavelengths': [650e-9, 750e-9]}]],
            'dft': []}
    for _ in range(3):
        x0, x1 = sorted(rng.uniform(0.0, 1.4e-6, 2))
        y0, y1 = sorted(rng.uniform(0.0, 1.1e-6, 2))
        spec['dft'].append([x0, y0, x1 - 1e-12, y1 - 1e-12, list(rng.uniform(3.5e14, 5.5e14, int(rng.integers(1, 4)))),
                            int(rng.integers(1, 5))])
    chunks = [int(c) for c in rng.integers(1, 60, 12)]
    spec['checkpoints'] = list(np.cumsum(chunks))
    _, o_maps, snaps = run_oracle_dft(spec)
    sim, _, maps = _build(spec, CONFIGS[seed % 2])
    sim.em.finalize()
    done = 0
    for cp in spec['checkpoints']:
        sim.em.engine.advance(int(cp - done))
        done = cp
        for k, mon in enumerate(maps):
            np.testing.assert_array_equal(mon.ez_dft, snaps[cp][0][k][0])
    sim.em.engine.close()


def test_reset_zeroes_maps_and_reruns_identically():
    spec = CASES_DFT[0]
    sim, _, maps = _build(spec, CONFIGS[0])
    sim.run(n_steps=200, verbose=False, print_every=0)
    first = [m.ez_dft.copy() for m in maps]
    sim.em.engine.reset()
    for m in maps:
        assert not np.any(m.ez_dft)
    sim.em.engine.advance(200)
    for a, m in zip(first, maps):
        np.testing.assert_array_equal(m.ez_dft, a)
    sim.em.engine.close()


def test_batched_advance_refuses_maps():
    spec = CASES_DFT[0]
    sim, _, _ = _build(spec, CONFIGS[0])
    sim.em.finalize()
    advancer = serving.BatchAdvancer(0)
    try:
        advancer.adopt(sim.em.engine)
        with pytest.raises(RuntimeError, match='field-map'):
            advancer.advance([sim.em.engine], 30)
    finally:
        advancer.close()
        sim.em.engine.close()


@pytest.mark.parametrize('seed', [0, 1])
def test_random_poles_and_tfsf_match_oracle(seed):
    """Seeded Drude / Lorentz media and a TFSF box with a map and probes, advanced in chunks of random length, against
    the oracle (no fixture: the oracle is pinned to open_sol on the poles_* and tfsf_* cases)."""
    rng = np.random.default_rng(500 + seed)
    cx, cy = rng.uniform(0.6e-6, 1.0e-6, 2)
    spec = {'sim': {'size_x': 1.6e-6, 'size_y': 1.6e-6, 'dx': 25e-9, 'npml': 10,
                    'boundaries': ['pml', 'periodic_y'][seed]},
            'ops': [['add_dielectric_circle', [0.4e-6, 1.2e-6, 0.12e-6], {'eps_r': 2.0}],
                    ['add_tfsf', [0.3e-6, 0.3e-6, 1.3e-6, 1.3e-6], {'wavelength': float(rng.uniform(650e-9, 900e-9)),
                                                                    'bandwidth': 0.5}],
                    ['add_flux_monitor', ['y', 1.45e-6, [0.1e-6, 1.5e-6]], {'wavelengths': [700e-9]}]],
            'poles': [['drude_circle', [float(cx), float(cy), float(rng.uniform(0.08e-6, 0.2e-6))],
                       [float(rng.uniform(4e15, 9e15)), float(rng.uniform(1e13, 2e14)), 2.0]],
                      ['lorentz_circle', [0.4e-6, 1.2e-6, 0.12e-6], [1.2, 2.5e15, 1e14]]],
            'dft': [[0.1e-6, 0.1e-6, 1.5e-6, 1.5e-6, [4.0e14], 2]],
            'probes': [[float(cx), float(cy), 'ez'], [1.45e-6, 0.8e-6, 'hy']]}
    chunks = [int(c) for c in rng.integers(1, 80, 8)]
    spec['checkpoints'] = list(np.cumsum(chunks))
    o, _, snaps = run_oracle_dft(spec)
    sim, _, maps = _build(spec, CONFIGS[0])
    sim.em.finalize()
    done = 0
    for cp in spec['checkpoints']:
        sim.em.engine.advance(int(cp - done))
        done = cp
        for k, mon in enumerate(maps):
            np.testing.assert_array_equal(mon.ez_dft, snaps[cp][0][k][0])
        assert _digest(sim.em.engine.read_field('ez')) == snaps[cp][2]['ez']
    for (ix, iy, _, times, values), probe in zip(o.probe_records, sim.probes):
        np.testing.assert_array_equal(probe.get_data()[1], np.array(values, dtype=np.float32))
    sim.em.engine.close()


@pytest.mark.parametrize('seed', [0, 1])
def test_random_hz_poles_match_oracle(seed):
    """Seeded Drude / Lorentz media on the H_z engine (face sets of E_x / E_y), a sheet crossing one of them, a map
    and probes, advanced in chunks of random length, against the oracle (pinned to open_sol on the poles_hz_* cases)."""
    rng = np.random.default_rng(700 + seed)
    cx, cy = rng.uniform(0.6e-6, 1.0e-6, 2)
    spec = {'sim': {'size_x': 1.6e-6, 'size_y': 1.6e-6, 'dx': 25e-9, 'npml': 10,
                    'boundaries': ['pml', 'periodic_y'][seed], 'polarization': 'hz'},
            'ops': [['add_dielectric_circle', [0.4e-6, 1.2e-6, 0.12e-6], {'eps_r': 2.0}],
                    ['add_line_source', ['y', float(cx) - 0.05e-6],
                     {'wavelength': float(rng.uniform(650e-9, 900e-9)), 'bandwidth': 0.5,
                      'span': [0.2e-6, 1.4e-6]}],
                    ['add_flux_monitor', ['y', 1.45e-6, [0.1e-6, 1.5e-6]], {'wavelengths': [700e-9]}]],
            'poles': [['drude_circle', [float(cx), float(cy), float(rng.uniform(0.08e-6, 0.2e-6))],
                       [float(rng.uniform(4e15, 9e15)), float(rng.uniform(1e13, 2e14)), 2.0]],
                      ['lorentz_circle', [0.4e-6, 1.2e-6, 0.12e-6], [1.2, 2.5e15, 1e14]]],
            'dft': [[0.1e-6, 0.1e-6, 1.5e-6, 1.5e-6, [4.0e14], 2]],
            'probes': [[float(cx), float(cy), 'ex'], [float(cx), float(cy), 'ey']]}
    chunks = [int(c) for c in rng.integers(1, 80, 8)]
    spec['checkpoints'] = list(np.cumsum(chunks))
    o, _, snaps = run_oracle_dft(spec)
    sim, _, maps = _build(spec, CONFIGS_HZ[0])
    sim.em.finalize()
    done = 0
    for cp in spec['checkpoints']:
        sim.em.engine.advance(int(cp - done))
        done = cp
        for k, mon in enumerate(maps):
            for got, want in zip(map_parts(mon), snaps[cp][0][k]):
                np.testing.assert_array_equal(got, want)
        assert _digest(sim.em.engine.read_field('hz')) == snaps[cp][2]['hz']
    for (ix, iy, _, times, values), probe in zip(o.probe_records, sim.probes):
        np.testing.assert_array_equal(probe.get_data()[1], np.array(values, dtype=np.float32))
    sim.em.engine.close()
