"""os_fdtd2d_advance_noalloc against os_fdtd2d_advance, both through the C ABI.

Two identical simulations (seeded cylinders, a line source, four flux lines, CPML on every side) advance the same two
chunks in a row, one handle through each entry point; fields and complex128 spectra must be bit-identical after
each chunk.  The second allocation-free call must leave the device's free memory unchanged (the first one may load
the module that holds the scratch array; the check assumes nothing else allocates on the device meanwhile), and a
chunk whose tables exceed the fixed scratch is rejected before anything runs.  The same equality is checked on a TFSF
case (the per-step kernels, TFSF rows of the value table), an H_z case with a field map and an E_z case with a field
map (phase tables of maps after those of the flux lines).  Collected last (file name) so that it also runs after every
other GPU test in one process.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import opensol_b200 as ob
from cases import apply_ops
from cases_dft import case as dft_case
from opensol_b200 import _native, workloads
from test_oracle_golden_dft import field_names, map_parts

pytestmark = pytest.mark.gpu

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'include', 'opensol_fdtd.h')


def _max_floats():
    with open(HEADER) as f:
        return int(re.search(r'#define OS_FDTD_NOALLOC_MAX_FLOATS (\d+)', f.read()).group(1))


def _sim(cells=384):
    sim = ob.Simulation(**workloads.roofline_2d_sim_args(total_cells=cells), verbose=False)
    mons = workloads.apply(sim, workloads.roofline_2d_ops(total_cells=cells, n_cylinders=40, seed=7))
    sim.em.finalize()
    return sim, mons


def _advance_noalloc(engine, n_steps):
    """One chunk through os_fdtd2d_advance_noalloc, with the same host tables engine.advance would upload."""
    values, first_q, n_q, phases, t_end = engine.chunk_tables(n_steps)
    rc = _native.load().os_fdtd2d_advance_noalloc(
        engine.handle, n_steps, _native.fptr(values) if values.size else None, first_q, n_q,
        _native.fptr(phases) if phases.size else None)
    _native.check(rc)
    engine.n_step += n_steps
    engine.time = t_end


def _state(engine, mons):
    engine.synchronize()
    fields = {n: engine.read_field(n) for n in ('ez', 'hx', 'hy')}
    spectra = [m.spectra() for m in mons]
    return fields, spectra


def _assert_same(a, b):
    for name in a[0]:
        np.testing.assert_array_equal(a[0][name], b[0][name], err_msg=name)
    for (ea, ha), (eb, hb) in zip(a[1], b[1]):
        np.testing.assert_array_equal(ea, eb)
        np.testing.assert_array_equal(ha, hb)


def test_noalloc_matches_advance_on_two_calls_in_a_row():
    import torch
    ref_sim, ref_mons = _sim()
    sim, mons = _sim()
    ref, eng = ref_sim.em.engine, sim.em.engine
    assert len(ref_mons) == 4 and eng.n_step == 0
    chunks = (301, 250)        # 301 is not a multiple of the steps per launch: a shorter last launch
    for k, n in enumerate(chunks):
        ref.advance(n)
        ref.synchronize()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _advance_noalloc(eng, n)
        free_after = torch.cuda.mem_get_info()[0]
        if k > 0:   # the first call per device may load the module that holds the scratch array
            assert free_after == free_before, (free_before, free_after)
        _assert_same(_state(ref, ref_mons), _state(eng, mons))
    assert eng.n_step == sum(chunks)
    assert any(float(np.abs(e).max()) > 0 for e, _ in (m.spectra() for m in mons))


def test_noalloc_rejects_tables_beyond_the_scratch():
    sim, mons = _sim(cells=128)
    eng = sim.em.engine
    n_sources = len(eng._lines)
    assert n_sources >= 1
    too_many = _max_floats() // n_sources + 1       # the source values alone exceed the scratch
    values, first_q, n_q, phases, _ = eng.chunk_tables(too_many)
    lib = _native.load()
    rc = lib.os_fdtd2d_advance_noalloc(eng.handle, too_many, _native.fptr(values), first_q, n_q,
                                       _native.fptr(phases))
    assert rc == _native.OS_ERR_INVALID
    assert 'fixed scratch' in _native.last_error()
    steps = ctypes.c_int64()
    _native.check(lib.os_fdtd2d_step_count(eng.handle, ctypes.byref(steps)))
    assert steps.value == 0
    np.testing.assert_array_equal(eng.read_field('ez'), 0)


def _case_sim(name):
    spec = dft_case(name)
    sim = ob.Simulation(**spec['sim'], verbose=False)
    fluxes = apply_ops(sim, spec)
    maps = [sim.em.add_dft_monitor(x0, y0, x1, y1, frequencies=f, downsample=ds)
            for x0, y0, x1, y1, f, ds in spec['dft']]
    sim.em.finalize()
    return sim, spec, fluxes, maps


def _case_state(sim, spec, fluxes, maps):
    engine = sim.em.engine
    engine.synchronize()
    return ([engine.read_field(n) for n in field_names(spec)], [m.spectra() for m in fluxes],
            [part for m in maps for part in map_parts(m)])


@pytest.mark.parametrize('name', ['tfsf_cylinder', 'dft_hz_pml', 'dft_pml'])
def test_noalloc_matches_advance_on_other_paths(name):
    ref = _case_sim(name)
    got = _case_sim(name)
    for n in (97, 64):
        ref[0].em.engine.advance(n)
        _advance_noalloc(got[0].em.engine, n)
        a, b = _case_state(*ref), _case_state(*got)
        for x, y in zip(a[0], b[0]):
            np.testing.assert_array_equal(x, y)
        for (ea, ha), (eb, hb) in zip(a[1], b[1]):
            np.testing.assert_array_equal(ea, eb)
            np.testing.assert_array_equal(ha, hb)
        for x, y in zip(a[2], b[2]):
            np.testing.assert_array_equal(x, y)
    assert any(float(np.abs(f).max()) > 0 for f in a[0])


def test_noalloc_counts_phases_only_when_given_and_refuses_huge_counts():
    """A chunk that takes no DFT sample, given a huge sample count but no phase table, runs as os_fdtd2d_advance
    does (nothing is uploaded for it); step or sample counts whose tables would overflow the scratch, however large,
    are refused before anything runs."""
    sim, mons = _sim(cells=128)
    eng = sim.em.engine
    m = eng.sample_interval
    assert m > 2
    values, _, _, _, t_end = eng.chunk_tables(m - 1)            # ends before the first sample
    lib = _native.load()
    _native.check(lib.os_fdtd2d_advance_noalloc(eng.handle, m - 1, _native.fptr(values), 1, 10 ** 9, None))
    eng.n_step += m - 1
    eng.time = t_end
    ref, ref_mons = _sim(cells=128)
    ref.em.engine.advance(m - 1)
    for name in ('ez', 'hx', 'hy'):
        np.testing.assert_array_equal(eng.read_field(name), ref.em.engine.read_field(name))
    for n_steps, n_samples in ((2 ** 62, 2 ** 62 // m + 2), (m, 2 ** 61)):   # each covers its chunk's samples
        values, first_q, _, phases, _ = eng.chunk_tables(4)
        rc = lib.os_fdtd2d_advance_noalloc(eng.handle, n_steps, _native.fptr(values), first_q, n_samples,
                                           _native.fptr(phases))
        assert rc == _native.OS_ERR_INVALID
        assert 'fixed scratch' in _native.last_error()
    steps = ctypes.c_int64()
    _native.check(lib.os_fdtd2d_step_count(eng.handle, ctypes.byref(steps)))
    assert steps.value == m - 1
