"""GPU parity of the 2D H_z engine (the CUDA path through the C ABI) against open_sol's own outputs and the oracle.

The engine evaluates every cell in the reference's order without fused multiply-add, so these tests assert
bit-identical H_z / E_x / E_y (array_equal, and the SHA-256 digests of open_sol's own fields in tests/golden),
bit-identical complex128 spectra and fluxes, for both kernel sets (variant 1: the interior kernel, TMA-staged in the
lossless one-word-per-cell form or with direct loads in the coefficient form, plus the border kernel; variant 0: the
per-half-step kernels) and for interior row runs per CTA from 1 row up.
"""
import hashlib
import os

import numpy as np
import pytest

from cases import apply_ops
from cases_hz import HZ_CASES
from oracle.hz2d import OracleHz2D

import opensol_b200 as ob

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _fields(sim):
    return {n: sim.em.engine.read_field(n) for n in ('hz', 'ex', 'ey')}


def _oracle_kwargs(spec):
    return {k: v for k, v in spec['sim'].items() if k != 'polarization'}


# (variant, rows per CTA, steps per launch): the per-half-step kernels, and the interior + border kernels with the
# per-grid choice and with interior runs of 1, 2, 7 and 64 rows (ragged last runs, halo rows on every run), one step
# per launch and two (where the two-step interior box fits the grid)
HZ_CONFIGS = [(0, 0, 1), (1, 0, 1), (1, 1, 1), (1, 2, 1), (1, 7, 1), (1, 64, 1), (1, 0, 2), (1, 16, 2), (1, 1, 2)]


@pytest.mark.parametrize('config', HZ_CONFIGS, ids=[f'v{v}_rows{r}_T{t}' for v, r, t in HZ_CONFIGS])
@pytest.mark.parametrize('spec', HZ_CASES, ids=[c['name'] for c in HZ_CASES])
def test_hz_cases_bit_exact_against_reference_fixtures(spec, config):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    sim = ob.Simulation(**spec['sim'], verbose=False)
    mons = apply_ops(sim, spec)
    sim.em.engine.configure(variant=config[0], steps_per_launch=config[2], tile_rows=config[1])
    done = 0
    for cp in spec['checkpoints']:
        sim.run(n_steps=cp - done, verbose=False)
        done = cp
        for name, arr in _fields(sim).items():
            assert _digest(arr) == str(g[f'sha_{name}_{cp}']), f'{name} differs from open_sol at step {cp}'
        for k, mon in enumerate(mons):
            e, h = mon.spectra()
            np.testing.assert_array_equal(e, g[f'spec_e{k}_{cp}'])
            np.testing.assert_array_equal(h, g[f'spec_h{k}_{cp}'])
            np.testing.assert_array_equal(mon.flux(), g[f'flux{k}_{cp}'])


def test_hz_forms_and_face_coefficients():
    """The lossy case runs the coefficient form, the lossless ones the one-word form; the device face coefficients
    equal open_sol's ca_x / cb_x / ca_y / cb_y bit for bit."""
    for spec in HZ_CASES:
        g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
        sim = ob.Simulation(**spec['sim'], verbose=False)
        apply_ops(sim, spec)
        sim.em.finalize()
        eng = sim.em.engine
        lossy = any(op[2].get('sigma_e') for op in spec['ops'] if op[0].startswith('add_dielectric'))
        assert eng.lossless_form() == (not lossy)
        cb_x, cb_y = eng.read_cb()
        np.testing.assert_array_equal(cb_x, g['cb_x'])
        np.testing.assert_array_equal(cb_y, g['cb_y'])


def _random_spec(seed):
    rng = np.random.default_rng(1000 + seed)
    dx = float(rng.choice([15e-9, 20e-9, 25e-9]))
    boundaries = str(rng.choice(['pml', 'periodic_x', 'periodic_y', 'periodic']))
    npml = int(rng.integers(4, 13))
    # up to 300 cells a side: several 128-column strips, ragged last strips and exact multiples of 128
    nx_win = int(rng.choice([int(rng.integers(6, 97)), int(rng.integers(100, 301)), 256 - 2 * npml, 256]))
    ny_win = int(rng.choice([int(rng.integers(6, 97)), int(rng.integers(100, 301)), 128 - 2 * npml, 256]))
    size_x, size_y = nx_win * dx, ny_win * dx
    lossy = rng.random() < 0.4
    ops = []
    for _ in range(int(rng.integers(0, 6))):
        sigma = float(rng.choice([0.0, 2e4])) if lossy else 0.0
        if rng.random() < 0.5:
            ops.append(['add_dielectric_circle', [float(rng.uniform(0, size_x)), float(rng.uniform(0, size_y)),
                                                  float(rng.uniform(0, 0.4 * max(size_x, size_y)))],
                        {'eps_r': float(rng.uniform(1, 12)), 'sigma_e': sigma}])
        else:
            xs, ys = sorted(rng.uniform(0, size_x, 2).tolist()), sorted(rng.uniform(0, size_y, 2).tolist())
            ops.append(['add_dielectric_rectangle', [xs[0], ys[0], xs[1], ys[1]],
                        {'eps_r': float(rng.uniform(1, 12)), 'sigma_e': sigma}])
    for _ in range(int(rng.integers(1, 4))):
        axis = str(rng.choice(['x', 'y']))
        pos = float(rng.uniform(0, size_y if axis == 'x' else size_x))
        length = size_x if axis == 'x' else size_y
        span = None if rng.random() < 0.4 else sorted(rng.uniform(0, length, 2).tolist())
        ops.append(['add_line_source', [axis, pos], {'wavelength': float(rng.uniform(400e-9, 1600e-9)),
                                                     'bandwidth': float(rng.uniform(0.3, 0.9)),
                                                     'amplitude': float(rng.uniform(0.5, 3.0)), 'span': span}])
    for _ in range(int(rng.integers(0, 3))):
        axis = str(rng.choice(['x', 'y']))
        pos = float(rng.uniform(0, size_y if axis == 'x' else size_x))
        length = size_x if axis == 'x' else size_y
        span = sorted(rng.uniform(0, length, 2).tolist())
        ops.append(['add_flux_monitor', [axis, pos, span],
                    {'wavelengths': rng.uniform(400e-9, 1600e-9, int(rng.integers(1, 5))).tolist()}])
    rows = int(rng.choice([0, 1, 3, 16, 100]))
    spec = {'sim': {'size_x': size_x, 'size_y': size_y, 'dx': dx, 'npml': npml, 'boundaries': boundaries},
            'ops': ops, 'steps': int(rng.integers(1, 200)), 'rows': rows, 'variant': int(rng.random() < 0.8)}
    spec['T'] = 2 if spec['variant'] == 1 and rng.random() < 0.5 else 1
    return spec


@pytest.mark.parametrize('seed', range(24))
def test_hz_random_geometries_bit_exact(seed):
    """Every boundary preset, grids from the 2 npml + 2 minimum to 300+ cells (several column strips, ragged and
    exact multiples of the strip), lossless and lossy, 1-3 sheets (spans cut to the CPML), 0-2 flux lines, 1-199
    steps in two chunks, variant 0 or the fused kernel with various row runs, one or two steps per launch."""
    spec = _random_spec(seed)
    sim = ob.Simulation(**spec['sim'], polarization='hz', verbose=False)
    mons = apply_ops(sim, spec)
    sim.em.engine.configure(variant=spec['variant'], steps_per_launch=spec['T'], tile_rows=spec['rows'])
    o = OracleHz2D(**spec['sim'])
    omons = apply_ops(o, spec)
    first = spec['steps'] // 3
    for n in (first, spec['steps'] - first):
        sim.run(n_steps=n, verbose=False)
        o.run(n_steps=n)
    for name, arr in _fields(sim).items():
        np.testing.assert_array_equal(arr, getattr(o, name), err_msg=name)
    for mon, omon in zip(mons, omons):
        e, h = mon.spectra()
        np.testing.assert_array_equal(e, omon.e_acc)
        np.testing.assert_array_equal(h, omon.h_acc)
        np.testing.assert_array_equal(mon.flux(), omon.flux())


def test_hz_magnetic_cells_take_the_coefficient_form():
    """mu_r != 1 on a box: per-cell da / db (coefficient form), against the oracle."""
    args = {'size_x': 2.0e-6, 'size_y': 3.5e-6, 'dx': 25e-9, 'npml': 10, 'boundaries': 'pml'}
    spec = {'ops': [['add_dielectric_circle', [1.0e-6, 1.5e-6, 0.4e-6], {'eps_r': 5.0}],
                    ['add_line_source', ['y', 0.4e-6], {'wavelength': 800e-9}],
                    ['add_flux_monitor', ['y', 1.6e-6, [0.2e-6, 3.3e-6]], {'wavelengths': [700e-9, 900e-9]}]]}
    sim = ob.Simulation(**args, polarization='hz', verbose=False)
    mons = apply_ops(sim, spec)
    o = OracleHz2D(**args)
    omons = apply_ops(o, spec)
    box = (slice(50, 70), slice(60, 120))
    sim.domain.materials.array('mu_r')[box] = np.float32(2.5)
    sim.domain.materials.version += 1
    sim.em.materials_changed(('mu_r',))
    o.mu_r[box] = np.float32(2.5)
    sim.run(n_steps=300, verbose=False)
    o.run(n_steps=300)
    assert not sim.em.engine.lossless_form()
    for name, arr in _fields(sim).items():
        np.testing.assert_array_equal(arr, getattr(o, name), err_msg=name)
    np.testing.assert_array_equal(mons[0].flux(), omons[0].flux())


def test_hz_variants_agree_and_reset():
    spec = HZ_CASES[0]
    results = []
    for variant in (0, 1):
        sim = ob.Simulation(**spec['sim'], verbose=False)
        mons = apply_ops(sim, spec)
        sim.em.engine.configure(variant=variant, steps_per_launch=1, tile_rows=0)
        for n in (1, 9, 90):
            sim.run(n_steps=n, verbose=False)
        results.append((_fields(sim), mons[0].spectra()))
        sim.em.engine.reset()
        sim.em.engine.advance(100)
        again = _fields(sim)
        for name in again:
            np.testing.assert_array_equal(again[name], results[-1][0][name])
    for name in results[0][0]:
        np.testing.assert_array_equal(results[0][0][name], results[1][0][name])
    np.testing.assert_array_equal(results[0][1][0], results[1][1][0])


def test_hz_field_write_read_roundtrip_and_launch_count():
    sim = ob.Simulation(1e-6, 0.5e-6, 25e-9, npml=8, polarization='hz', verbose=False)
    sim.add_flux_monitor('y', 0.5e-6, (0.1e-6, 0.4e-6), wavelengths=[700e-9])
    sim.add_line_source('x', 0.2e-6, wavelength=700e-9)
    sim.em.engine.configure(variant=1, steps_per_launch=1, tile_rows=0)
    sim.em.finalize()
    rng = np.random.default_rng(3)
    values = rng.standard_normal((sim.grid.nx, sim.grid.ny)).astype(np.float32)
    sim.em.engine.write_field('ex', values)
    np.testing.assert_array_equal(sim.em.engine.read_field('ex'), values)
    sim.em.engine.advance(12)
    m = sim.em.engine.sample_interval
    # per step the interior kernel and the border kernel, plus one DFT launch per sample step
    assert sim.em.engine.launch_count() == 12 * 2 + 12 // m


@pytest.mark.parametrize('size, npml, boundaries, rows', [((4.0e-6, 3.2e-6), 10, 'pml', 0),
                                                          ((3.0e-6, 5.12e-6), 12, 'pml', 16),
                                                          ((4.4e-6, 2.88e-6), 8, 'periodic_y', 5),
                                                          ((2.6e-6, 4.0e-6), 10, 'periodic_x', 0)])
def test_hz_two_steps_per_launch(size, npml, boundaries, rows):
    """Two steps per launch (hz2d_interior2_kernel on the interior box, the border in two single steps through the
    scratch set) on lossless grids whose rows are a multiple of 4 cells: dielectric blocks, sheets along both axes
    crossing the interior, two flux lines (a sample step always ends a launch), uneven chunks -- every field, spectrum
    and flux bit-identical to one step per launch and to the oracle, in fewer launches."""
    ops = [['add_dielectric_rectangle', [0.8e-6, 0.4e-6, 1.6e-6, 1.9e-6], {'eps_r': 4.0}],
           ['add_dielectric_circle', [2.0e-6, 1.4e-6, 0.5e-6], {'eps_r': 2.1}],
           ['add_line_source', ['y', 0.45e-6], {'wavelength': 700e-9, 'bandwidth': 0.6}],
           ['add_line_source', ['x', 1.1e-6], {'wavelength': 900e-9, 'bandwidth': 0.5, 'amplitude': 2.0}],
           ['add_flux_monitor', ['y', 2.3e-6, [0.2e-6, 2.4e-6]], {'wavelengths': [650e-9, 800e-9, 1000e-9]}],
           ['add_flux_monitor', ['x', 0.7e-6, [0.2e-6, 2.4e-6]], {'wavelengths': [900e-9]}]]
    args = {'size_x': size[0], 'size_y': size[1], 'dx': 20e-9, 'npml': npml, 'boundaries': boundaries}
    runs = []
    for T in (1, 2):
        sim = ob.Simulation(**args, polarization='hz', verbose=False)
        mons = apply_ops(sim, {'ops': ops})
        sim.em.engine.configure(variant=1, steps_per_launch=T, tile_rows=rows)
        assert sim.grid.ny % 4 == 0
        launches = 0
        for n in (37, 1, 2, 160):
            sim.run(n_steps=n, verbose=False)
            launches += sim.em.engine.launch_count()
        assert sim.em.engine.lossless_form()
        runs.append((_fields(sim), [m.spectra() for m in mons], [m.flux() for m in mons], launches))
    o = OracleHz2D(**args)
    omons = apply_ops(o, {'ops': ops})
    o.run(n_steps=200)
    assert runs[1][3] < runs[0][3]   # the two-step launches ran
    for name in runs[0][0]:
        np.testing.assert_array_equal(runs[1][0][name], runs[0][0][name], err_msg=name)
        np.testing.assert_array_equal(runs[1][0][name], getattr(o, name), err_msg=name)
    for (e1, h1), (e2, h2), omon in zip(runs[0][1], runs[1][1], omons):
        np.testing.assert_array_equal(e2, e1)
        np.testing.assert_array_equal(h2, h1)
        np.testing.assert_array_equal(e2, omon.e_acc)
    for f1, f2 in zip(runs[0][2], runs[1][2]):
        np.testing.assert_array_equal(f2, f1)


def test_hz_probes_two_steps_per_launch():
    """Field probes with two steps per launch: the first step's value of a cell inside the two-step box comes from
    hz2d_probe_mid_kernel (stepped again from the launch's input), of a cell in the border's first-step region from
    the scratch set.  Probes of each component in the box, on the box's outer ring, in the CPML and on the grid
    corners, one added between chunks: the series equal one step per launch bit for bit, in fewer launches."""
    from opensol_b200.monitors import FieldProbe
    ops = [['add_dielectric_rectangle', [0.8e-6, 0.4e-6, 1.6e-6, 1.9e-6], {'eps_r': 4.0}],
           ['add_line_source', ['y', 0.45e-6], {'wavelength': 700e-9, 'bandwidth': 0.6}],
           ['add_line_source', ['x', 1.1e-6], {'wavelength': 900e-9, 'bandwidth': 0.5, 'amplitude': 2.0}],
           ['add_flux_monitor', ['y', 2.3e-6, [0.2e-6, 2.4e-6]], {'wavelengths': [650e-9, 800e-9]}]]
    args = {'size_x': 4.0e-6, 'size_y': 3.2e-6, 'dx': 20e-9, 'npml': 10, 'boundaries': 'pml'}
    runs = []
    for T in (1, 2):
        sim = ob.Simulation(**args, polarization='hz', verbose=False)
        apply_ops(sim, {'ops': ops})
        eng = sim.em.engine
        nx, ny = sim.grid.nx, sim.grid.ny
        cells = [(nx // 2, ny // 2, 'hz'), (nx // 2 + 1, ny // 2 + 1, 'ex'), (100, 60, 'ey'), (12, 50, 'hz'),
                 (110, 16, 'ex'), (110, 163, 'ey'), (3, 40, 'ey')]
        probes = []
        for ix, iy, comp in cells:
            probes.append(FieldProbe(ix, iy, comp))
            eng.attach_probe(probes[-1])
        eng.configure(variant=1, steps_per_launch=T, tile_rows=0)
        launches = 0
        for k, n in enumerate((37, 1, 2, 160)):
            sim.run(n_steps=n, verbose=False)
            launches += eng.launch_count()
            if k == 0:
                probes.append(FieldProbe(0, 0, 'hz'))
                eng.attach_probe(probes[-1])
        assert eng.lossless_form() and ny % 4 == 0
        if T == 2:
            assert eng.hz_plan()[0] > 0
        runs.append(([p.get_data() for p in probes], launches, _fields(sim)))
        eng.close()
    assert runs[1][1] < runs[0][1]   # the two-step launches ran
    for (t0, v0), (t1, v1) in zip(runs[0][0], runs[1][0]):
        assert v0.shape == v1.shape and v0.shape[0] > 0
        np.testing.assert_array_equal(t1, t0)
        np.testing.assert_array_equal(v1, v0)
    assert runs[1][0][-1][1].shape == (163,)
    for name in runs[0][2]:
        np.testing.assert_array_equal(runs[1][2][name], runs[0][2][name], err_msg=name)
