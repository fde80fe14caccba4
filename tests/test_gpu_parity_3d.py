"""GPU parity of the 3D engine (the CUDA path through the C ABI) against the oracle and open_sol's own outputs.

The kernels evaluate every cell in the reference's order without fused multiply-add, so fields, complex128 spectra
and fluxes are asserted bit-identical to the oracle and to open_sol's numpy twins (SHA-256 digests in tests/golden);
open_sol's default numba twins compute the coefficients in float64, and the fields stay within 1e-5 of the run's
peak field of them, fluxes within 1e-5 relative (FIELD_RTOL, FLUX_RTOL).
"""
import hashlib
import os

import numpy as np
import pytest

from builders3d import build_product
from cases3d import CASES3D
from test_oracle_golden3d import build_oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
FIELDS = ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')
FIELD_RTOL = 1e-5
FLUX_RTOL = 1e-5


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize('spec', CASES3D, ids=[c['name'] for c in CASES3D])
def test_cases_against_reference_fixtures_and_oracle(spec):
    g = np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))
    physics, monitors = build_product(spec)
    o = build_oracle(spec)
    engine = physics.engine
    assert engine.material_id is not None and _digest(engine.material_id) == str(g['sha_material_id'])
    assert physics.sources[0].weight == g['dipole_weight'][0]
    assert monitors[0].sample_interval == int(g['sample_interval'])
    done = 0
    for cp in spec['checkpoints']:
        physics.run(cp - done)
        o.run(cp - done)
        done = cp
        fields = engine.state()
        for name in FIELDS:
            np.testing.assert_array_equal(fields[name], o.fields[name], err_msg=f'{name} at step {cp}')
            assert _digest(fields[name]) == str(g[f'numpy_sha_{name}_{cp}']), (name, cp)
        for k, (mon, omon) in enumerate(zip(monitors, o.monitors)):
            planes = mon.planes() if hasattr(mon, 'planes') else [mon]
            oplanes = omon.planes() if hasattr(omon, 'planes') else [omon]
            for plane, oplane in zip(planes, oplanes):
                for (e, h), opair in zip(plane.spectra(), oplane.pairs):
                    np.testing.assert_array_equal(e, opair['e_dft'])
                    np.testing.assert_array_equal(h, opair['h_dft'])
            flux = mon.flux()
            np.testing.assert_array_equal(flux, g[f'numpy_flux{k}_{cp}'])
            np.testing.assert_allclose(flux, g[f'numba_flux{k}_{cp}'], rtol=FLUX_RTOL, atol=0)


@pytest.mark.parametrize('spec', CASES3D, ids=[c['name'] for c in CASES3D])
def test_chunking_and_reset(spec):
    """One chunk, many one-step chunks and a run after reset() give the same fields."""
    physics, _ = build_product(spec)
    engine = physics.engine
    n = spec['checkpoints'][0]
    physics.run(n)
    whole = engine.state()
    engine.reset()
    for _ in range(n):
        physics.step()
    stepped = engine.state()
    for name in FIELDS:
        np.testing.assert_array_equal(whole[name], stepped[name])
    assert engine.n_step == n


def test_field_roundtrip_and_launches():
    spec = CASES3D[0]
    physics, _ = build_product(spec)
    engine = physics.engine
    rng = np.random.default_rng(3)
    values = rng.standard_normal(engine.shape).astype(np.float32)
    engine.write_field('hy', values)
    np.testing.assert_array_equal(engine.read_field('hy'), values)
    engine.set_variant(1)
    engine.reset()
    physics.run(30)
    engine.synchronize()
    m = physics.monitors[0].sample_interval
    _, fused = engine.interior()
    assert fused   # the fused kernel, and H then E of the x, y and z faces in three launches each: 7 per step
    assert engine.launch_count() == 7 * 30 + 30 // m
    engine.set_variant(3)   # the lean form needs rows of at least 144 cells: this grid runs the in-place form
    engine.reset()
    physics.run(30)
    assert not engine.interior()[1]
    assert engine.launch_count() == 2 * 30 + 30 // m
    engine.set_variant(0)
    engine.reset()
    physics.run(30)
    assert engine.launch_count() == 2 * 30 + 30 // m
    assert engine.last_advance_ms() > 0.0


# c3_mixed with a z extent of 160 cells (a multiple of 4, at least 144): the lean form runs on it, with lossy and
# magnetic blocks (every coefficient path), a periodic axis and pec / pmc faces
MIXED_NZ160 = dict(CASES3D[1], name='c3_mixed_nz160', window=(16, 20, 150))
FORM_SPECS = CASES3D + [MIXED_NZ160]


@pytest.mark.parametrize('spec', FORM_SPECS, ids=[c['name'] for c in FORM_SPECS])
def test_step_forms_bit_identical(spec):
    """The fused forms (two field and psi sets; the lean form where the z extent is a multiple of 4, else the
    in-place form) in every launch shape and the in-place two-kernel form give bit-identical fields and fluxes,
    chunked into uneven advances (the set holding the current state alternates between chunks)."""
    from cases3d import grid_shape
    shape = grid_shape(spec)
    lean = shape[2] % 4 == 0 and shape[2] >= 144 and shape[1] >= 17
    runs = []
    for variant, config in ((0, 0), (1, 0), (1, 1), (1, 2), (1, 3), (1, 4), (3, 0), (3, 1), (3, 2), (3, 3), (3, 4)):
        physics, monitors = build_product(spec)
        engine = physics.engine
        engine.set_variant(variant)
        engine.set_fused_config(config)
        box, fused = engine.interior()
        assert fused == (variant == 1 or (variant == 3 and lean))
        assert all(hi > lo for lo, hi in zip(box[::2], box[1::2]))
        for n in (7, 1, 12, 5):
            physics.run(n)
        runs.append((engine.state(), [np.asarray(m.flux()) for m in monitors]))
    for run in runs[1:]:
        for name in FIELDS:
            np.testing.assert_array_equal(runs[0][0][name], run[0][name], err_msg=name)
        for f0, f1 in zip(runs[0][1], run[1]):
            np.testing.assert_array_equal(f0, f1)


def test_x_chunk_does_not_change_results():
    """The number of x planes a block streams is a launch shape only: 1, 5, 24 planes and the whole grid give
    bit-identical fields and fluxes."""
    spec = CASES3D[0]
    physics, _ = build_product(spec)
    engine = physics.engine
    n = spec['checkpoints'][0]
    runs = []
    for planes in (engine.shape[0], 1, 5, 24):
        engine.reset()
        engine.set_x_chunk(planes)
        physics.run(n)
        runs.append((engine.state(), [np.asarray(m.flux()) for m in physics.monitors]))
    for state, fluxes in runs[1:]:
        for name in FIELDS:
            np.testing.assert_array_equal(state[name], runs[0][0][name])
        for f, f0 in zip(fluxes, runs[0][1]):
            np.testing.assert_array_equal(f, f0)


def test_workload_512_deterministic_across_x_chunks():
    """Size-independent property at the benchmark size (512^3, 500 spheres, dipole, flux box): two runs, with 24- and
    7-plane x chunks, give bit-identical fields and box flux (no races, no order dependence)."""
    from opensol_b200 import workloads
    out = []
    for planes in (24, 7):
        physics, box = workloads.roofline_3d_physics()
        physics.finalize()
        physics.engine.set_x_chunk(planes)
        physics.run(200)
        out.append((physics.engine.read_field('ez'), physics.engine.read_field('hx'), np.asarray(box.flux())))
        del physics, box
    assert np.abs(out[0][0]).max() > 0
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


def test_workload_512_against_oracle():
    """The 3D benchmark workload at its full size (512^3 incl. CPML 12, 500 spheres, z dipole, 8-frequency flux box)
    for 200 steps (7 DFT samples) against the oracle on the host: the painted eps_r, all six fields, every plane's
    complex128 spectra and the box flux bit-identical."""
    from cases3d import roofline_3d_oracle
    from opensol_b200 import workloads
    physics, box = workloads.roofline_3d_physics()
    physics.finalize()
    physics.engine.set_variant(2)   # the staged fused form on the full grid; every form gives the same bits
    o, obox = roofline_3d_oracle()
    np.testing.assert_array_equal(physics.domain.materials.array('eps_r'), o.materials['eps_r'])
    assert box.sample_interval == obox.sample_interval
    n = 200
    physics.run(n)
    o.run(n)
    engine = physics.engine
    for name in FIELDS:
        np.testing.assert_array_equal(engine.read_field(name), o.fields[name], err_msg=name)
    assert np.abs(o.fields['ez']).max() > 0
    for plane, oplane in zip(box.planes(), obox.planes()):
        for (e, h), opair in zip(plane.spectra(), oplane.pairs):
            np.testing.assert_array_equal(e, opair['e_dft'])
            np.testing.assert_array_equal(h, opair['h_dft'])
    np.testing.assert_array_equal(np.asarray(box.flux()), np.asarray(obox.flux()))


@pytest.mark.parametrize('total', [64, 96])
def test_staged_form_bit_identical(total):
    """The fused form with planes staged in shared memory by tensor copies (variant 2; here the 3D workload on 64^3
    and 96^3 grids) in every launch shape gives the fields and box flux of the in-place two-kernel form bit for bit,
    over uneven chunks and short and long x chunks."""
    from opensol_b200 import workloads
    n_spheres = max(1, int(round(500 * (total / 512) ** 3)))
    runs = []
    for variant, config, chunk in ((0, 0, 24), (2, 0, 24), (2, 1, 7), (2, 2, 24), (2, 3, 1), (2, 4, 50)):
        physics, box = workloads.roofline_3d_physics(total_cells=total, n_spheres=n_spheres)
        physics.finalize()
        engine = physics.engine
        engine.set_variant(variant)
        engine.set_fused_config(config)
        engine.set_x_chunk(chunk)
        for n in (13, 1, 40):
            physics.run(n)
        runs.append((engine.state(), np.asarray(box.flux())))
        del physics, box
    assert np.abs(runs[0][0]['ez']).max() > 0
    for state, flux in runs[1:]:
        for name in FIELDS:
            np.testing.assert_array_equal(state[name], runs[0][0][name], err_msg=name)
        np.testing.assert_array_equal(flux, runs[0][1])


FP64_FLUX_RTOL_3D = 1e-5   # float32 box flux against the float64 3D oracle run, relative to its peak


def test_workload_512_full_run_against_fixture():
    """The whole 2000-step 512^3 workload against tests/golden/c3_full.npz (the oracle's float32 and float64 runs,
    tests/golden/make_golden_c3_full.py): the six fields and every plane's complex128 spectra bit-identical (SHA-256)
    at steps 200 and 2000, the box flux equal; the error of the float32 box flux against the float64 run is stated and
    held to FP64_FLUX_RTOL_3D."""
    from opensol_b200 import workloads
    g = np.load(os.path.join(GOLDEN, 'c3_full.npz'))
    physics, box = workloads.roofline_3d_physics()
    physics.finalize()
    assert box.sample_interval == int(g['sample_interval'])
    engine = physics.engine
    done = 0
    for cp in (200, 2000):
        physics.run(cp - done)
        done = cp
        for name in FIELDS:
            assert _digest(engine.read_field(name)) == str(g[f'sha_{name}_{cp}']), (name, cp)
        for p_, plane in enumerate(box.planes()):
            for q, (e, h) in enumerate(plane.spectra()):
                assert _digest(e) == str(g[f'sha_spec_e{p_}{q}_{cp}']), (p_, q, cp)
                assert _digest(h) == str(g[f'sha_spec_h{p_}{q}_{cp}']), (p_, q, cp)
        np.testing.assert_array_equal(np.asarray(box.flux()), g[f'flux_{cp}'])
    f64 = g['f64_flux_2000']
    error = float(np.abs(np.asarray(box.flux()) - f64).max() / np.abs(f64).max())
    print(f'float32 vs float64 box flux error (relative to its peak): {error:.3e}')
    assert error <= FP64_FLUX_RTOL_3D


@pytest.mark.parametrize('total', [160, 200])
def test_lean_form_bit_identical(total):
    """The lean staged fused form (variant 3: four cells a thread, packed arithmetic; here the 3D workload on 160^3
    and 200^3 grids, two and three tiles along z with partial last tiles) in every launch shape gives the fields and
    box flux of the in-place two-kernel form bit for bit, over uneven chunks and short and long x chunks."""
    from opensol_b200 import workloads
    n_spheres = max(1, int(round(500 * (total / 512) ** 3)))
    runs = []
    for variant, config, chunk in ((0, 0, 24), (3, 0, 24), (3, 1, 7), (3, 2, 1), (3, 3, 50), (3, -1, 2), (3, 3, 63),
                                   (3, 4, 24), (3, 4, 1), (3, 4, 63)):
        physics, box = workloads.roofline_3d_physics(total_cells=total, n_spheres=n_spheres)
        physics.finalize()
        engine = physics.engine
        engine.set_variant(variant)
        engine.set_fused_config(config)
        engine.set_x_chunk(chunk)
        assert engine.interior()[1] == (variant == 3)
        for n in (13, 1, 40):
            physics.run(n)
        runs.append((engine.state(), np.asarray(box.flux())))
        del physics, box
    assert np.abs(runs[0][0]['ez']).max() > 0
    for state, flux in runs[1:]:
        for name in FIELDS:
            np.testing.assert_array_equal(state[name], runs[0][0][name], err_msg=name)
        np.testing.assert_array_equal(flux, runs[0][1])
