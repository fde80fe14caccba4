"""The bounded waits of the staged interior kernel give up without harming the device: the engine's test hook makes
one warp wait, at most 1 ms, on an mbarrier that no copy and no thread completes.  The advance's next synchronising
call reports the timeout (RuntimeError naming the bounded wait; the status is OS_ERR_CUDA), the context stays usable,
and after reset() the same engine gives the fields and fluxes of a clean run bit for bit."""
import numpy as np
import pytest

import opensol_b200 as ob
from opensol_b200 import workloads

pytestmark = pytest.mark.gpu
CELLS = 512
STEPS = 60


def _sim():
    sim = ob.Simulation(**workloads.roofline_2d_sim_args(total_cells=CELLS), verbose=False)
    mons = workloads.apply(sim, workloads.roofline_2d_ops(total_cells=CELLS, n_cylinders=30, seed=5))
    sim.em.finalize()
    return sim, mons


def _state(sim, mons):
    engine = sim.em.engine
    engine.synchronize()
    return [engine.read_field(n) for n in ('ez', 'hx', 'hy')], [m.flux() for m in mons]


def test_wait_runs_out_reports_and_recovers():
    clean_sim, clean_mons = _sim()
    clean_sim.em.engine.advance(STEPS)
    clean = _state(clean_sim, clean_mons)
    sim, mons = _sim()
    engine = sim.em.engine
    interior_cells, _, _ = engine.plan_info()
    assert interior_cells > 0            # the blocked interior kernel runs on this grid
    engine.set_stall_probe(1_000_000)    # 1 ms
    engine.advance(STEPS)
    with pytest.raises(RuntimeError, match='bounded wait'):
        engine.synchronize()
    engine.synchronize()                 # the flag was cleared: the next call succeeds
    engine.set_stall_probe(0)
    engine.reset()
    engine.advance(STEPS)
    fields, fluxes = _state(sim, mons)
    for a, b in zip(fields, clean[0]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(fluxes, clean[1]):
        np.testing.assert_array_equal(a, b)
    assert np.abs(fields[0]).max() > 0
