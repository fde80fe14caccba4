"""GPU parity of the 2D E_z engine (the CUDA path through the C ABI) against the oracle and open_sol's own outputs.

Bar: fluxes and field snapshots within 1e-5 relative (float32) of the reference CPU backend.
The engine evaluates every cell in the reference's order without fused multiply-add, so these tests assert the
stronger property: bit-identical fields (array_equal, and the SHA-256 digests of open_sol's own fields in
tests/golden), bit-identical complex128 spectra and fluxes.  FLUX_RTOL documents the contract bar where a
tolerance-based check is used.
"""
import hashlib
import os

import numpy as np
import pytest

from cases import CASES, apply_ops
from oracle.fdtd2d import OracleEz2D

import opensol_b200 as ob
from opensol_b200 import workloads

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
FLUX_RTOL = 1e-5
FRAME_KIND = 'ez2d_frame_step_kernel | ez2d_tb_kernel (general)'


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _fields(sim):
    return {n: sim.em.engine.read_field(n) for n in ('ez', 'hx', 'hy')}


@pytest.mark.parametrize('spec', CASES, ids=[c['name'] for c in CASES])
def test_cases_bit_exact_against_reference_fixtures(spec):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    sim = ob.Simulation(**spec['sim'], verbose=False)
    mons = apply_ops(sim, spec)
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
    # the float64-stepper reference of the same case: the float32 flux error against it, stated
    if spec['name'] == 'c1':
        f32 = mons[0].flux()
        f64 = g[f"f64_flux0_{spec['checkpoints'][-1]}"]
        rel = np.abs(f32 - f64) / np.abs(f64)
        assert np.all(rel < FLUX_RTOL), rel


@pytest.mark.parametrize('spec', CASES, ids=[c['name'] for c in CASES])
def test_cases_bit_exact_against_oracle(spec):
    sim = ob.Simulation(**spec['sim'], verbose=False)
    mons = apply_ops(sim, spec)
    o = OracleEz2D(**spec['sim'])
    omons = apply_ops(o, spec)
    n = spec['checkpoints'][-1]
    sim.run(n_steps=n, verbose=False)
    o.run(n_steps=n)
    for name, arr in _fields(sim).items():
        np.testing.assert_array_equal(arr, getattr(o, name))
    for mon, omon in zip(mons, omons):
        e, h = mon.spectra()
        np.testing.assert_array_equal(e, omon.e_acc)
        np.testing.assert_array_equal(h, omon.h_acc)


# (variant, steps per launch, interior tile rows): per-step kernels, and the blocked kernels at every T with tile
# heights from a few rows (many ragged tiles, tiles shorter than T) to 128
KERNEL_CONFIGS = [(0, 1, 128), (1, 1, 128), (1, 2, 32), (1, 3, 7), (1, 3, 128), (1, 4, 128), (1, 4, 3), (2, 3, 128),
                  (2, 4, 16)]


@pytest.mark.parametrize('config', KERNEL_CONFIGS, ids=[f'v{v}_T{t}_rows{r}' for v, t, r in KERNEL_CONFIGS])
@pytest.mark.parametrize('spec', CASES, ids=[c['name'] for c in CASES])
def test_kernel_configs_bit_exact(spec, config):
    """Every kernel variant and launch shape gives open_sol's fields and spectra bit for bit."""
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    sim = ob.Simulation(**spec['sim'], verbose=False)
    sim.em.engine.configure(*config)
    mons = apply_ops(sim, spec)
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


def test_autotune_keeps_state_and_results():
    """The tile-height autotuner times trial launches on the live fields without changing them; the run afterwards is
    still open_sol's bit for bit."""
    spec = CASES[0]
    g = np.load(os.path.join(GOLDEN, 'c1.npz'))
    sim = ob.Simulation(**spec['sim'], verbose=False)
    mons = apply_ops(sim, spec)
    sim.run(n_steps=150, verbose=False)
    before = _fields(sim)
    rows, ms = sim.em.engine.autotune(candidates=(3, 16, 64), repeats=2)
    assert rows in (3, 16, 64) and ms > 0
    for name, arr in _fields(sim).items():
        np.testing.assert_array_equal(arr, before[name])
    sim.run(n_steps=150, verbose=False)
    for name, arr in _fields(sim).items():
        assert _digest(arr) == str(g[f'sha_{name}_300'])
    e, h = mons[0].spectra()
    np.testing.assert_array_equal(e, g['spec_e0_300'])


def test_interior_and_general_kernels_both_run():
    """The headline grid uses the interior kernel for nearly all cells and, per blocked launch of T steps, T
    single-step frame launches for the rest."""
    args = workloads.roofline_2d_sim_args()
    sim = ob.Simulation(**args, verbose=False)
    workloads.apply(sim, workloads.roofline_2d_ops())
    sim.em.finalize()
    sim.em.engine.configure(steps_per_launch=4)
    cells, tiles_in, tiles_gen = sim.em.engine.plan_info(4)
    assert tiles_in > 0 and tiles_gen > 0
    assert cells > 0.98 * sim.grid.nx * sim.grid.ny
    sim.em.engine.set_profiling(True)
    sim.run(n_steps=52, verbose=False)
    times = sim.em.engine.kernel_times()
    assert times['ez2d_interior_kernel'][1] == 13 and times[FRAME_KIND][1] == 13 * 4
    assert times['ez2d_flux_staged_kernel'][1] == 2 * 4
    sim.clear()


def _random_spec(seed):
    rng = np.random.default_rng(seed)
    dx = float(rng.choice([15e-9, 20e-9, 25e-9]))
    boundaries = str(rng.choice(['pml', 'periodic_x', 'periodic_y', 'periodic']))
    npml = int(rng.integers(4, 13))
    nx_win, ny_win = int(rng.integers(6, 97)), int(rng.integers(6, 97))
    size_x, size_y = nx_win * dx, ny_win * dx
    ops = []
    for _ in range(int(rng.integers(0, 6))):
        if rng.random() < 0.5:
            ops.append(['add_dielectric_circle', [float(rng.uniform(0, size_x)), float(rng.uniform(0, size_y)),
                                                  float(rng.uniform(0, 0.4 * max(size_x, size_y)))],
                        {'eps_r': float(rng.uniform(1, 12)), 'sigma_e': float(rng.choice([0.0, 2e4]))}])
        else:
            xs, ys = sorted(rng.uniform(0, size_x, 2).tolist()), sorted(rng.uniform(0, size_y, 2).tolist())
            ops.append(['add_dielectric_rectangle', [xs[0], ys[0], xs[1], ys[1]], {'eps_r': float(rng.uniform(1, 12))}])
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
    return {'sim': {'size_x': size_x, 'size_y': size_y, 'dx': dx, 'npml': npml, 'boundaries': boundaries},
            'ops': ops, 'steps': int(rng.integers(1, 260))}


@pytest.mark.parametrize('seed', range(24))
def test_random_geometries_bit_exact(seed):
    """Ragged, tiny (down to the 2 npml + 2 minimum) and non-square grids, every boundary preset, 0-3 sources (lossy
    cells, spans cut to the CPML), 0-2 monitors, 1-259 steps in two chunks."""
    spec = _random_spec(seed)
    sim = ob.Simulation(**spec['sim'], verbose=False)
    mons = apply_ops(sim, spec)
    o = OracleEz2D(**spec['sim'])
    omons = apply_ops(o, spec)
    first = spec['steps'] // 3
    for n in (first, spec['steps'] - first):
        sim.run(n_steps=n, verbose=False)
        o.run(n_steps=n)
    for name, arr in _fields(sim).items():
        np.testing.assert_array_equal(arr, getattr(o, name))
    for mon, omon in zip(mons, omons):
        e, h = mon.spectra()
        np.testing.assert_array_equal(e, omon.e_acc)
        np.testing.assert_array_equal(h, omon.h_acc)
        np.testing.assert_array_equal(mon.flux(), omon.flux())


def test_minimum_cpml_grid():
    """A 2 npml + 2 cell axis (the smallest CPMLSided accepts) on both axes."""
    dx, npml = 25e-9, 6
    args = {'size_x': 2 * dx, 'size_y': 2 * dx, 'dx': dx, 'npml': npml, 'boundaries': 'pml'}
    spec = {'ops': [['add_line_source', ['x', dx], {'wavelength': 500e-9}]]}
    sim = ob.Simulation(**args, verbose=False)
    apply_ops(sim, spec)
    o = OracleEz2D(**args)
    apply_ops(o, spec)
    assert (sim.grid.nx, sim.grid.ny) == (2 * npml + 2, 2 * npml + 2)
    sim.run(n_steps=80, verbose=False)
    o.run(n_steps=80)
    for name, arr in _fields(sim).items():
        np.testing.assert_array_equal(arr, getattr(o, name))


def test_empty_simulation_and_zero_steps():
    sim = ob.Simulation(1e-6, 1e-6, 25e-9, npml=8, verbose=False)
    mon = sim.add_flux_monitor('x', 0.5e-6, (0, 1e-6), wavelengths=[800e-9])
    assert sim.run(n_steps=0, verbose=False) == 0
    sim.run(n_steps=25, verbose=False)
    assert mon.sample_interval == 1
    for arr in _fields(sim).values():
        assert not arr.any()
    assert not mon.flux().any()


def test_chunking_and_reset_do_not_change_results():
    spec = CASES[1]
    sim = ob.Simulation(**spec['sim'], verbose=False)
    mons = apply_ops(sim, spec)
    for n in (1, 7, 50, 142):
        sim.run(n_steps=n, verbose=False)
    chunked = _fields(sim), mons[0].spectra()
    sim.em.engine.reset()
    sim.em.engine.advance(200)
    single = _fields(sim), mons[0].spectra()
    for name in chunked[0]:
        np.testing.assert_array_equal(chunked[0][name], single[0][name])
    np.testing.assert_array_equal(chunked[1][0], single[1][0])


def test_field_write_read_roundtrip():
    sim = ob.Simulation(1e-6, 0.5e-6, 25e-9, npml=8, verbose=False)
    sim.em.finalize()
    rng = np.random.default_rng(3)
    values = rng.standard_normal((sim.grid.nx, sim.grid.ny)).astype(np.float32)
    sim.em.engine.write_field('hx', values)
    np.testing.assert_array_equal(sim.em.engine.read_field('hx'), values)


def test_duration_run_matches_reference_ticks_and_flux():
    spec = CASES[0]
    g = np.load(os.path.join(GOLDEN, 'c1.npz'))
    sim = ob.Simulation(**spec['sim'], verbose=False)
    mons = apply_ops(sim, spec)
    assert sim.run(duration=spec['duration'], verbose=False) == int(g['duration_steps'])
    np.testing.assert_array_equal(mons[0].flux(), g['flux0_1370'])


def test_roofline_workload_full_size_bit_exact():
    """The 8192^2 benchmark grid (2000 cylinders, 4 x 16-frequency lines) for 600 steps against the oracle on the host:
    every field and every monitor's complex128 E / H spectra bit-identical at full size.  By step 600 the pulse has
    crossed the lo-x flux line and reached the first cylinders, and 23 DFT samples have been taken."""
    args = workloads.roofline_2d_sim_args()
    ops = workloads.roofline_2d_ops()
    sim = ob.Simulation(**args, verbose=False)
    mons = workloads.apply(sim, ops)
    o = OracleEz2D(**args)
    omons = workloads.apply(o, ops)
    n = 600
    sim.run(n_steps=n, verbose=False)
    o.run(n_steps=n)
    assert sim.grid.nx == sim.grid.ny == 8192
    assert mons[0].sample_interval == o.sample_interval
    for name, arr in _fields(sim).items():
        np.testing.assert_array_equal(arr, getattr(o, name))
    crossed = 0
    for mon, omon in zip(mons, omons):
        e, h = mon.spectra()
        np.testing.assert_array_equal(e, omon.e_acc)
        np.testing.assert_array_equal(h, omon.h_acc)
        np.testing.assert_array_equal(mon.flux(), omon.flux())
        crossed += bool(np.abs(e).max() > 0)
    assert crossed >= 1
    sim.clear()


def test_roofline_workload_linearity():
    """Size-independent property at full size: the update is linear, so doubling the source amplitude doubles every
    field and quadruples every flux.  Not bit for bit: a power-of-two scale commutes with rounding only for normal
    numbers, and the leading edge of the pulse passes through subnormal values (~1e-38) whose rounding seeds ulp-level
    differences; the bar is float32 rounding (LINEARITY_RTOL of the largest value)."""
    LINEARITY_RTOL = 1e-5
    args = workloads.roofline_2d_sim_args()
    out = []
    for amplitude in (1.0, 2.0):
        sim = ob.Simulation(**args, verbose=False)
        mons = workloads.apply(sim, workloads.roofline_2d_ops(amplitude=amplitude))
        sim.run(n_steps=600, verbose=False)
        out.append((sim.em.engine.read_field('ez'), [m.flux() for m in mons]))
        sim.clear()
    scale = np.abs(out[1][0]).max()
    assert scale > 0
    assert np.abs(out[1][0] - 2.0 * out[0][0]).max() <= LINEARITY_RTOL * scale
    flux_scale = max(float(np.abs(f).max()) for f in out[1][1])
    for f1, f2 in zip(out[0][1], out[1][1]):
        assert np.abs(f2 - 4.0 * f1).max() <= LINEARITY_RTOL * flux_scale


def test_roofline_workload_deterministic():
    """Two runs of the full-size workload give bit-identical fields and fluxes (no races, no atomics order)."""
    args = workloads.roofline_2d_sim_args()
    out = []
    for _ in range(2):
        sim = ob.Simulation(**args, verbose=False)
        mons = workloads.apply(sim, workloads.roofline_2d_ops())
        sim.run(n_steps=400, verbose=False)
        out.append((sim.em.engine.read_field('ez'), sim.em.engine.read_field('hy'), [m.flux() for m in mons]))
        sim.clear()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    for f1, f2 in zip(out[0][2], out[1][2]):
        np.testing.assert_array_equal(f1, f2)


FP64_FLUX_RTOL = 1e-5   # float32 run against the float64 oracle run, relative to each monitor's peak flux


def test_roofline_workload_full_run_against_fixture():
    """The whole 10,000-step 8192^2 benchmark run against tests/golden/c2_full.npz (open_sol's own float32 run and
    the oracle's, which agree byte for byte; tests/golden/make_golden_c2_full.py): E_z, H_x, H_y and every monitor's
    complex128 E / H spectra bit-identical (SHA-256) at steps 600 and 10,000, the four 16-frequency fluxes equal.  The
    error of those float32 fluxes against the float64 oracle run is stated and held to FP64_FLUX_RTOL."""
    g = np.load(os.path.join(GOLDEN, 'c2_full.npz'))
    sim = ob.Simulation(**workloads.roofline_2d_sim_args(), verbose=False)
    mons = workloads.apply(sim, workloads.roofline_2d_ops())
    done = 0
    for cp in (600, 10_000):
        sim.run(n_steps=cp - done, verbose=False, print_every=0)
        done = cp
        for name, arr in _fields(sim).items():
            assert _digest(arr) == str(g[f'sha_{name}_{cp}']), f'{name} at step {cp}'
        for k, mon in enumerate(mons):
            e, h = mon.spectra()
            assert _digest(e) == str(g[f'sha_spec_e{k}_{cp}']), f'E spectra of monitor {k} at step {cp}'
            assert _digest(h) == str(g[f'sha_spec_h{k}_{cp}']), f'H spectra of monitor {k} at step {cp}'
            np.testing.assert_array_equal(mon.flux(), g[f'flux{k}_{cp}'])
    assert int(g['sample_interval']) == mons[0].sample_interval
    errors = []
    for k, mon in enumerate(mons):
        f64 = g[f'f64_flux{k}_10000']
        errors.append(float(np.abs(mon.flux() - f64).max() / np.abs(f64).max()))
    print(f'float32 vs float64 flux error per monitor (relative to its peak): {errors}')
    assert max(errors) <= FP64_FLUX_RTOL
    sim.clear()
