"""The 3D engine's host-side setup (opensol_b200's own restatement) against open_sol's fixtures on the CPU: grid and
dt, kappa-folded curl spacings, CPML layer rows, material index and tables (exact levels and the re-quantisation
path), dipole placement and dual volume, flux plane geometry.  No device is touched."""
import os

import numpy as np
import pytest

from cases3d import CASES3D, DX, boundary_faces, paint, window_size
from make_golden3d import binned_index_cases
from oracle.fdtd3d import OracleEM3D

import opensol_b200 as ob
from opensol_b200.engine3d import FDTDEngine3D, face_shares
from opensol_b200.material_index3d import build_material_index
from opensol_b200.monitors3d import FluxBox3D, PlaneFlux3D, face_samples
from opensol_b200.physics3d import nearest_face

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _domain(spec):
    sx, sy, sz = window_size(spec)
    config = ob.BoundaryConfig3D(boundary_faces(spec), npml=spec['npml'])
    domain = ob.Domain3D.uniform(sx, sy, sz, DX, npml_sides=config.npml_sides, boundary_config=config)
    for name, values in paint(spec).items():
        domain.materials.array(name)[...] = values
    return domain, config


@pytest.fixture(scope='module', params=[c['name'] for c in CASES3D])
def case(request):
    spec = next(c for c in CASES3D if c['name'] == request.param)
    return spec, np.load(os.path.join(GOLDEN, f"{spec['name']}.npz"))


def test_grid_rows_and_materials(case):
    spec, g = case
    domain, config = _domain(spec)
    engine = FDTDEngine3D(domain, config)
    assert engine.shape == tuple(g['shape'])
    assert np.float32(engine.dt) == g['dt']
    for axis in range(3):
        np.testing.assert_array_equal(engine.inv_e[axis], g[f'inv_e{axis}'])
        np.testing.assert_array_equal(engine.inv_h[axis], g[f'inv_h{axis}'])
    assert sorted(f'cpml_{axis}{kind}' for axis in engine.cpml for kind in 'eh') == \
        sorted(k[:-8] for k in g.files if k.startswith('cpml_') and k.endswith('_row_map'))
    for axis, layer in engine.cpml.items():
        for kind in 'eh':
            key = f'cpml_{axis}{kind}'
            np.testing.assert_array_equal(getattr(layer, f'row_map_{kind}'), g[key + '_row_map'])
            np.testing.assert_array_equal(getattr(layer, f'b_{kind}'), g[key + '_b'])
            np.testing.assert_array_equal(getattr(layer, f'gain_{kind}'), g[key + '_gain'])
    ids, n_ids = engine.build_materials_host()
    import hashlib
    assert hashlib.sha256(ids.tobytes()).hexdigest() == str(g['sha_material_id'])
    for mine, key in (('t_ez', 'table_eps_z'), ('t_sig', 'table_sigma'), ('t_mu', 'table_mu'),
                      ('t_sm', 'table_sigma_m')):
        np.testing.assert_array_equal(engine.tables[mine], g[key])
    # the oracle's shares are the reference's face_shares: the engine's must equal them
    sx, sy, sz = window_size(spec)
    o = OracleEM3D(sx, sy, sz, DX, faces=boundary_faces(spec), npml=spec['npml'])
    for axis in range(3):
        for mine, theirs in zip(engine.shares[axis], o.shares[axis]):
            np.testing.assert_array_equal(mine, theirs)


def test_dipole_and_monitor_geometry(case):
    spec, g = case
    domain, config = _domain(spec)
    physics = ob.EMPhysics3D(domain)
    sx, sy, sz = window_size(spec)
    d = spec['dipole']
    x, y, z = (f * s for f, s in zip(d['at'], (sx, sy, sz)))
    axis = 'xyz'.index(d['orientation'])
    cell = list(domain.pos_to_cell(x, y, z))
    cell[axis] = nearest_face(domain.cell_edges()[axis], (x, y, z)[axis], domain.physical_window()[axis])
    assert tuple(cell) == tuple(g['dipole_cell'])
    assert physics.engine.face_dual_volume(axis, cell) == float(g['dipole_volume'])
    engine = physics.engine
    k = 0
    if spec['flux_box'] is not None:
        b = spec['flux_box']
        lo = tuple(f * s for f, s in zip(b['lo'], (sx, sy, sz)))
        hi = tuple(f * s for f, s in zip(b['hi'], (sx, sy, sz)))
        bounds = [(physics._nearest_edge(a, min(lo[a], hi[a])), physics._nearest_edge(a, max(lo[a], hi[a])))
                  for a in range(3)]
        box = FluxBox3D(bounds, ob.monitors.resolve_frequencies(list(b['wavelengths']), None), engine.dt,
                        engine.widths, engine.shape, engine.periodic)
        planes = np.asarray([(p.normal_axis, p.edge, *sum(p.bounds, ())) for p in box.planes()])
        np.testing.assert_array_equal(planes, g['monitor0_planes'])
        np.testing.assert_array_equal(box.frequencies, g['monitor0_frequencies'])
        k = 1
    for p in spec['flux_planes']:
        a = 'xyz'.index(p['normal'])
        bounds = [(w.start, w.stop) for w in domain.physical_window()]
        size = (sx, sy, sz)[a]
        bounds[a] = (physics._nearest_edge(a, p['at'] * size),) * 2
        plane = PlaneFlux3D(a, bounds[a][0], bounds, ob.monitors.resolve_frequencies(list(p['wavelengths']), None),
                            engine.dt, engine.widths, engine.shape, engine.periodic)
        np.testing.assert_array_equal(np.asarray([(plane.normal_axis, plane.edge, *sum(plane.bounds, ()))]),
                                      g[f'monitor{k}_planes'])
        k += 1


def test_face_samples_weights():
    widths = np.full(10, 2.0e-8)
    for first, last in ((0, 10), (2, 7), (1, 2), (3, 9)):
        faces, weights = face_samples(widths, first, last)
        edges = np.arange(max(first, 1), last + 1)
        expected = [0.5 * ((widths[e - 1] if e > first else 0.0) + (widths[e] if e < last else 0.0)) for e in edges]
        assert faces == slice(int(edges[0]) - 1, int(edges[-1]))
        np.testing.assert_array_equal(weights, expected)


def test_material_index_requantisation():
    g = np.load(os.path.join(GOLDEN, 'material_index3d.npz'))
    for case, (limit, arrays) in enumerate(binned_index_cases()):
        ids, tables, errors, deltas = build_material_index(arrays, arrays['eps_r'].shape, limit)
        np.testing.assert_array_equal(ids, g[f'case{case}_ids'])
        for name, table in tables.items():
            np.testing.assert_array_equal(table, g[f'case{case}_table_{name}'])
        assert set(errors) == {k[len(f'case{case}_error_'):] for k in g.files if k.startswith(f'case{case}_error_')}
        for name in errors:
            assert errors[name] == float(g[f'case{case}_error_{name}'])
            assert deltas[name] == float(g[f'case{case}_delta_{name}'])


def test_material_ids_are_lexicographic_ranks_of_level_tuples():
    """With exact levels, a cell's id is the rank of its tuple of level numbers (arrays that vary, in order) among the
    occurring tuples, and the tables give back each array's value: checked against numpy's row-wise unique for one
    to six varying arrays (four or more take the ranked radix groups)."""
    rng = np.random.default_rng(12)
    names = ('eps_r', 'sigma_e', 'mu_r', 'eps_xx', 'eps_yy', 'sigma_m')
    for k in range(1, 7):
        shape = (9, 7, 11)
        arrays = {n: rng.choice(rng.uniform(1.0, 9.0, 4).astype(np.float32), size=shape) for n in names[:k]}
        arrays['mu_r'] = arrays.get('mu_r', np.ones(shape, np.float32))
        ids, tables, errors, _ = build_material_index(arrays, shape)
        varying = [n for n in arrays if np.unique(arrays[n]).size > 1]
        tuples = np.stack([np.searchsorted(np.unique(arrays[n]), arrays[n].ravel()) for n in varying], axis=1)
        _, expected = np.unique(tuples, axis=0, return_inverse=True)
        np.testing.assert_array_equal(ids.ravel(), expected.ravel())
        for n, a in arrays.items():
            np.testing.assert_array_equal(tables[n][ids], a)
        assert errors == {}


def test_face_shares_uniform_and_graded():
    lo, hi = face_shares(np.full(5, 3.0), periodic=False)
    assert np.all(lo == 0.5) and np.all(hi == 0.5)
    lo, hi = face_shares(np.array([1.0, 3.0, 1.0]), periodic=True)
    np.testing.assert_array_equal(lo, np.float32([0.25, 0.75, 0.5]))
    np.testing.assert_array_equal(hi, np.float32([0.75, 0.25, 0.5]))


def test_boundary_config_validation():
    with pytest.raises(ValueError, match='periodic faces must be paired'):
        ob.BoundaryConfig3D({'x_lo': 'periodic'})
    with pytest.raises(ValueError, match='must be one of'):
        ob.BoundaryConfig3D({'z_hi': 'open'})
    with pytest.raises(NotImplementedError):
        FDTDEngine3D(*_domain_mirror())


def _domain_mirror():
    config = ob.BoundaryConfig3D({'x_lo': 'symmetric'}, npml=4)
    domain = ob.Domain3D.uniform(4e-7, 4e-7, 4e-7, DX, npml_sides=config.npml_sides, boundary_config=config)
    return domain, config
