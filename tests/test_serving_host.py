"""Host side of the serving loop (no device): the seeded request stream and the per-job memory estimate."""
import numpy as np

from opensol_b200 import serving


def test_request_stream_is_seeded_and_in_range():
    a = serving.make_job_specs(n_jobs=64, rate=20.0, seed=7)
    b = serving.make_job_specs(n_jobs=64, rate=20.0, seed=7)
    assert [(s.side, s.steps, s.arrival, s.wavelength, s.rectangles) for s in a] == \
        [(s.side, s.steps, s.arrival, s.wavelength, s.rectangles) for s in b]
    assert all(256 <= s.side <= 2048 and 2000 <= s.steps <= 20000 for s in a)
    assert all(1 <= len(s.rectangles) <= 40 for s in a)
    assert all(1000e-9 <= s.wavelength <= 1600e-9 for s in a)
    arrivals = np.array([s.arrival for s in a])
    assert np.all(np.diff(arrivals) > 0)
    rate = len(a) / arrivals[-1]
    assert 10.0 < rate < 40.0


def test_device_bytes_covers_the_field_sets():
    spec = serving.make_job_specs(n_jobs=1, seed=1)[0]
    n = spec.side + 2 * spec.npml
    assert spec.device_bytes() >= 28 * n * n
