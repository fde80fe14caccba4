"""os_fdtd2d_advance_noalloc against os_fdtd2d_advance, both through the C ABI.

Two identical simulations (seeded cylinders, a line source, four flux lines, CPML on every side) advance the same two
chunks in a row, one handle through each entry point; fields and complex128 spectra must be bit-identical after
each chunk.  The second allocation-free call must leave the device's free memory unchanged (the first one may load
the module that holds the scratch array), and a chunk whose tables exceed the fixed scratch is rejected before
anything runs.  Collected last (file name) so that it also runs after every other GPU test in one process.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import opensol_b200 as ob
from opensol_b200 import _native, workloads

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
