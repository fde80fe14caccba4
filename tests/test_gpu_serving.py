"""The continuous-batching serving loop (opensol_b200.serving) on the GPU: every job's fluxes are bit-identical when
served in the mix and when run alone; admission respects the slot count and the memory budget; the batched advance
matches os_fdtd2d_advance field for field."""
import numpy as np
import pytest

from opensol_b200 import serving

pytestmark = pytest.mark.gpu


def _small_specs(n=7, seed=3):
    specs = serving.make_job_specs(n_jobs=n, rate=0.0, seed=seed, side_range=(40, 150), steps_range=(150, 700))
    return specs


def test_mix_equals_alone():
    specs = _small_specs()
    loop = serving.ServingLoop(max_active=3, chunk_steps=96, tile_rows=16)
    results = {r.job_id: r for r in loop.run(specs, realtime=False)}
    loop.close()
    assert sorted(results) == [s.job_id for s in specs]
    assert loop.peak_active == 3
    for spec in specs:
        alone, _ = serving.run_alone(spec, tile_rows=16)
        for mine, ref in zip(results[spec.job_id].fluxes, alone):
            np.testing.assert_array_equal(mine, ref)
        assert any(np.abs(f).max() > 0 for f in alone)


def test_memory_budget_limits_admission():
    specs = _small_specs(n=5, seed=4)
    budget = 2.5 * max(s.device_bytes() for s in specs)
    loop = serving.ServingLoop(memory_budget=budget, max_active=16, chunk_steps=128, tile_rows=32)
    results = loop.run(specs, realtime=False)
    loop.close()
    assert len(results) == len(specs)
    assert loop.peak_bytes <= budget
    assert loop.peak_active < len(specs)   # the budget, not the 16 slots, held jobs back


def test_batched_fields_equal_single_advance():
    """Fields of three jobs after one batched chunk equal those of each job advanced alone by os_fdtd2d_advance."""
    specs = _small_specs(n=3, seed=5)
    batch = serving.BatchAdvancer()
    sims = [serving.build_job(s, tile_rows=16)[0] for s in specs]
    for sim in sims:
        batch.adopt(sim.em.engine)
    batch.advance([sim.em.engine for sim in sims], 131)
    ms, launches = batch.last_ms()
    assert ms > 0 and launches >= 2 * (131 // 3)
    for spec, sim in zip(specs, sims):
        ref, _ = serving.build_job(spec, tile_rows=16)
        ref.em.engine.advance(131)
        for name in ('ez', 'hx', 'hy'):
            np.testing.assert_array_equal(sim.em.engine.read_field(name), ref.em.engine.read_field(name))
        assert sim.em.engine.n_step == ref.em.engine.n_step == 131
    batch.close()


def test_mix_equals_alone_at_stream_sizes():
    """Ten jobs of the serving stream's own kind at sizes 256-1024 cells a side (+30 CPML cells: row lengths that are
    not multiples of 4 included), 600-1500 steps, served together with at most 6 active at once and 256-step ticks
    (jobs join and leave mid-run): every job's fluxes bit-identical to its run alone."""
    specs = serving.make_job_specs(n_jobs=10, rate=0.0, seed=11, side_range=(256, 1024), steps_range=(600, 1500))
    assert any((s.side + 2 * s.npml) % 4 for s in specs)
    loop = serving.ServingLoop(max_active=6, chunk_steps=256)
    results = {r.job_id: r for r in loop.run(specs, realtime=False)}
    loop.close()
    assert sorted(results) == [s.job_id for s in specs]
    assert loop.peak_active == 6
    for spec in specs:
        alone, _ = serving.run_alone(spec)
        for mine, ref in zip(results[spec.job_id].fluxes, alone):
            np.testing.assert_array_equal(mine, ref)
