"""The 3D cases of tests/golden/cases3d.py built on the B200 engine's public API (Domain3D, BoundaryConfig3D,
EMPhysics3D) and on the oracle, from the same painted material arrays."""
from cases3d import DX, boundary_faces, paint, window_size


def build_product(spec, device=0, finalize=True):
    import opensol_b200 as ob
    sx, sy, sz = window_size(spec)
    config = ob.BoundaryConfig3D(boundary_faces(spec), npml=spec['npml'])
    domain = ob.Domain3D.uniform(sx, sy, sz, DX, npml_sides=config.npml_sides, boundary_config=config)
    for name, values in paint(spec).items():
        domain.materials.array(name)[...] = values
    physics = ob.EMPhysics3D(domain, device=device)
    d = spec['dipole']
    physics.add_dipole(*(f * s for f, s in zip(d['at'], (sx, sy, sz))), orientation=d['orientation'],
                       dipole_moment=d['moment'], wavelength=d['wavelength'], bandwidth=d['bandwidth'])
    monitors = []
    if spec['flux_box'] is not None:
        b = spec['flux_box']
        monitors.append(physics.add_flux_box(tuple(f * s for f, s in zip(b['lo'], (sx, sy, sz))),
                                             tuple(f * s for f, s in zip(b['hi'], (sx, sy, sz))),
                                             wavelengths=list(b['wavelengths'])))
    for p in spec['flux_planes']:
        size = {'x': sx, 'y': sy, 'z': sz}[p['normal']]
        monitors.append(physics.add_flux_plane(p['normal'], p['at'] * size, wavelengths=list(p['wavelengths'])))
    if finalize:
        physics.finalize()
    return physics, monitors
