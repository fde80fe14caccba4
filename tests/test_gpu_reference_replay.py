"""The reference-kernel replay (open_sol's own RawKernels compiled unchanged, replayed with its step sequence; the
GPU baseline the engine's speed is compared with) computes open_sol's step: on an all-CPML case with a cylinder, a
lossy block, a line source and two flux lines, its fields after 120 and 300 steps agree with the oracle's within
float32 rounding (the replayed kernels contract multiply-adds into FMA, as NVRTC compiles them by default, so they
are not bit-identical): FIELD_RTOL of the run's peak field, FLUX_RTOL of the peak flux."""
import numpy as np
import pytest

from cases import apply_ops, case
from oracle import replay_ez2d
from oracle.fdtd2d import OracleEz2D

pytestmark = pytest.mark.gpu
FIELD_RTOL = 1e-5
FLUX_RTOL = 1e-5


def test_replay_follows_the_oracle():
    ok, why = replay_ez2d.available()
    if not ok:
        pytest.skip(why)
    spec = case('pml_small')
    o = OracleEz2D(**spec['sim'])
    oracle_monitors = apply_ops(o, spec)
    o.finalize()
    replay_source = OracleEz2D(**spec['sim'])
    apply_ops(replay_source, spec)
    replay = replay_ez2d.ReferenceReplayEz2D(replay_source)
    replay.reset()
    peak = {'ez': 0.0, 'hx': 0.0, 'hy': 0.0}
    try:
        done = 0
        for checkpoint in (120, 300):
            ms = replay.run(checkpoint - done)
            o.run(n_steps=checkpoint - done)
            done = checkpoint
            assert ms > 0
            for name in peak:
                want = getattr(o, name)
                peak[name] = max(peak[name], float(np.abs(want).max()))
                got = replay.field(name)
                assert np.abs(got - want).max() <= FIELD_RTOL * peak[name], name
            for k, mon in enumerate(oracle_monitors):
                want = mon.flux()
                scale = float(np.abs(want).max())
                assert scale > 0
                assert np.abs(replay.flux(k) - want).max() <= FLUX_RTOL * scale
        assert min(peak.values()) > 0
    finally:
        replay.close()
