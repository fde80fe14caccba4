"""The B200 engine's host-side setup (its own restatement of open_sol's setup, in opensol_b200/) against the oracle on
the CPU: grid and dt, curl spacings, CPML rows, calibrated source profiles, DFT sample interval, per-step source
values and phase tables, the runner's tick count.  No device is touched."""
import numpy as np
import pytest

from cases import CASES, apply_ops
from oracle.fdtd2d import OracleEz2D, dft_phases

import opensol_b200 as ob
from opensol_b200.boundaries import BoundaryConfig, resolve_boundary


def _pair(spec):
    sim = ob.Simulation(**spec['sim'], verbose=False)
    apply_ops(sim, spec)
    sim.em.finalize_host()
    o = OracleEz2D(**spec['sim'])
    apply_ops(o, spec)
    o.finalize()
    return sim, o


@pytest.mark.parametrize('spec', CASES, ids=[c['name'] for c in CASES])
def test_setup_rows_match_oracle(spec):
    sim, o = _pair(spec)
    eng = sim.em.engine
    assert (eng.nx, eng.ny) == (o.domain.nx, o.domain.ny)
    assert eng.dt == o.domain.dt
    for name, values in eng.rows.curl.items():
        np.testing.assert_array_equal(values, o.curl[name])
    assert [s.face for s in eng.rows.sides] == [s.name for s in o.cpml_sides]
    for mine, ref in zip(eng.rows.sides, o.cpml_sides):
        for attr in ('b_e', 'a_e', 'inv_e', 'b_h', 'a_h', 'inv_h'):
            np.testing.assert_array_equal(getattr(mine, attr), getattr(ref, attr))
    for mine, ref in zip(sim.em.sources, o.sources):
        assert (mine.axis, mine.position, mine.span) == (ref.axis, ref.position, (ref.lo, ref.hi))
        np.testing.assert_array_equal(mine.profile, ref.profile)
    assert eng.sample_interval == o.sample_interval
    for mine, ref in zip(sim.em.monitors, o.monitors):
        assert (mine.axis, mine.position, mine.span) == (ref.normal_axis, ref.position, (ref.lo, ref.hi))
        np.testing.assert_array_equal(mine.frequencies, ref.frequencies)
    np.testing.assert_array_equal(sim.domain.materials.eps_r, o.eps_r)
    sigma = sim.domain.materials.get('sigma_e')
    np.testing.assert_array_equal(np.zeros_like(o.sigma_e) if sigma is None else sigma, o.sigma_e)


@pytest.mark.parametrize('spec', CASES, ids=[c['name'] for c in CASES])
def test_chunk_tables_match_oracle(spec):
    sim, o = _pair(spec)
    eng = sim.em.engine
    n = spec['checkpoints'][0]
    values, first_q, n_q, phases, t_end = eng.chunk_tables(n)
    ref_values, times_full = o.source_values(n)
    for mine, ref in zip(values, ref_values):
        np.testing.assert_array_equal(mine, ref)
    assert t_end == times_full[-1]
    m = o.sample_interval
    assert first_q == 1 and n_q == n // m
    offset = 0
    for mon in o.monitors:
        nf = mon.frequencies.size
        table = phases[offset:offset + n_q * nf * 2].reshape(n_q, nf, 2)
        for q in range(n_q):
            ref = dft_phases(2.0 * np.pi * mon.frequencies, times_full[(q + 1) * m - 1], mon.dt * m)
            np.testing.assert_array_equal(table[q], ref)
        offset += n_q * nf * 2


def test_calibration_reads_cb_formula():
    """The profile's cb factor is the engine's float32 dt / (eps_r eps0) (fdtd_ez_2d_kernels.py:314-319)."""
    from opensol_b200.sources import e_coefficients_host
    spec = CASES[1]
    sim, o = _pair(spec)
    ca, cb = e_coefficients_host(o.eps_r, o.sigma_e, o.domain.dt)
    np.testing.assert_array_equal(cb, o.cb)
    np.testing.assert_array_equal(ca, o.ca)


def test_duration_tick_count_without_device(monkeypatch):
    """Simulation.run(duration=80 fs) hands the runner's 1370 ticks to advance_ticks in print_every chunks."""
    spec = CASES[0]
    sim = ob.Simulation(**spec['sim'], verbose=False)
    apply_ops(sim, spec)
    calls = []
    monkeypatch.setattr(sim.em, 'finalize', lambda: sim.em.finalize_host())
    monkeypatch.setattr(sim.em.engine, 'advance', lambda n: calls.append(n))
    monkeypatch.setattr(sim.runner, 'flush', lambda: None)
    ticks = sim.run(duration=spec['duration'], verbose=False)
    assert ticks == 1370 and sum(calls) == 1370 and calls == [500, 500, 370]


def test_boundary_presets_and_validation():
    assert resolve_boundary('periodic_y', 15).periodic_y
    with pytest.raises(ValueError, match='Unknown boundary preset'):
        resolve_boundary('nope', 15)
    with pytest.raises(ValueError, match='must be paired'):
        BoundaryConfig('periodic', 'cpml', 'cpml', 'cpml')
    bc = BoundaryConfig.all_pml(10)
    bc.cpml_kappa_max = 0.5
    with pytest.raises(ValueError, match='cpml_kappa_max'):
        bc._validate()
    with pytest.raises(NotImplementedError):
        ob.Simulation(1e-6, 1e-6, 25e-9, boundaries='pec', verbose=False)


def test_simulation_argument_errors():
    with pytest.raises(ValueError, match='needs'):
        ob.Simulation(None, 1e-6, 25e-9)
    sim = ob.Simulation(1e-6, 1e-6, 25e-9, npml=8, verbose=False)
    with pytest.raises(ValueError, match='exactly one'):
        sim.run()
    with pytest.raises(ValueError, match='exactly one of wavelength'):
        sim.add_line_source('x', 0.5e-6)
    with pytest.raises(ValueError, match='outside physical domain'):
        sim.add_flux_monitor('x', 2e-6, (0, 1e-6), wavelengths=[1e-6])
    with pytest.raises(ValueError, match='circle radius'):
        sim.add_dielectric_circle(0.5e-6, 0.5e-6, -1.0, eps_r=2.0)


def test_courant_check_refuses_unstable_cells():
    sim = ob.Simulation(1e-6, 1e-6, 25e-9, npml=8, verbose=False)
    sim.add_dielectric_rectangle(0.2e-6, 0.2e-6, 0.4e-6, 0.4e-6, eps_r=0.5)
    with pytest.raises(ValueError, match='unstable'):
        sim.em.finalize_host()


def test_box_masks_equal_full_grid_masks():
    """Bounding-box masks set exactly the cells of open_sol's full-grid float32 expressions."""
    d = ob.Domain.uniform(2.0e-6, 1.5e-6, 20e-9, npml=10, verbose=False)
    X = d._centers_f32[0][:, None]
    Y = d._centers_f32[1][None, :]
    rng = np.random.default_rng(7)
    for _ in range(40):
        cx, cy = rng.uniform(-0.1e-6, 2.1e-6), rng.uniform(-0.1e-6, 1.6e-6)
        r = rng.uniform(0.0, 0.5e-6)
        full = (X - cx) ** 2 + (Y - cy) ** 2 <= r ** 2
        np.testing.assert_array_equal(d.circle_mask(cx, cy, r).full(full.shape), full)
        x0, x1, y0, y1 = rng.uniform(-0.1e-6, 2.1e-6, 2).tolist() + rng.uniform(-0.1e-6, 1.6e-6, 2).tolist()
        full = (X >= min(x0, x1)) & (X < max(x0, x1)) & (Y >= min(y0, y1)) & (Y < max(y0, y1))
        np.testing.assert_array_equal(d.rect_mask(x0, y0, x1, y1).full(full.shape), full)
