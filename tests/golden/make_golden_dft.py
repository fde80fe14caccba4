"""Generate the field-map (running DFT) fixtures of tests/golden/ by running open_sol itself (CPU backend) on the
cases of cases_dft.py.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden_dft.py /path/to/reference [case names]

Each case writes <name>.npz: per field-map monitor its sample boxes (x / y sample slice starts, strides, counts) and
its complex64 spectra at every checkpoint (E_z; or H_z, E_x, E_y for the H_z cases), the flux monitor's complex128 spectra, the DFT sample interval,
SHA-256 digests of the fields at every checkpoint, and per field probe its times and float32 values at the end.
"""
import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def digest(array):
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def run_case(spec):
    import numpy as np
    from open_sol import Simulation
    from cases import apply_ops
    from open_sol.physics.em.materials import DrudePole, LorentzPole
    from cases_dft import apply_poles
    sim = Simulation(**spec['sim'])
    fluxes = apply_ops(sim, spec)
    apply_poles(sim.em, spec, DrudePole, LorentzPole, sim.domain.circle_mask)
    maps = [sim.em.add_dft_monitor(x0, y0, x1, y1, frequencies=freqs, downsample=ds)
            for x0, y0, x1, y1, freqs, ds in spec['dft']]
    probes = [sim.em.add_field_probe(x, y, comp) for x, y, comp in spec.get('probes', [])]
    out = {}
    done = 0
    for cp in spec['checkpoints']:
        sim.run(n_steps=cp - done, print_every=0)
        done = cp
        fields = sim.em.fields
        names = ('ez', 'hx', 'hy') if spec['sim'].get('polarization', 'ez') == 'ez' else ('hz', 'ex', 'ey')
        for name in names:
            out[f'sha_{name}_{cp}'] = digest(np.array(getattr(fields, name)))
        for k, mon in enumerate(maps):
            if mon.polarization == 'ez':
                out[f'map{k}_{cp}'] = np.array(mon.ez_dft)
            else:
                for part in ('hz', 'ex', 'ey'):
                    out[f'map{k}_{part}_{cp}'] = np.array(getattr(mon, f'{part}_dft'))
        for k, mon in enumerate(fluxes):
            out[f'spec_e{k}_{cp}'] = np.array(mon._spectra.spectra[0])
    for k, mon in enumerate(maps):
        xs, ys = mon.x_samples, mon.y_samples
        out[f'map{k}_box'] = np.array([xs.start, xs.stop, mon.downsample, mon.mx, ys.start, ys.stop, mon.my])
    for k, probe in enumerate(probes):
        times, values = probe.get_data()
        out[f'probe{k}_t'], out[f'probe{k}_v'] = np.asarray(times), np.asarray(values)
        out[f'probe{k}_cell'] = np.array([probe.ix, probe.iy])
    out['sample_interval'] = np.int64(maps[0].sample_interval)
    out['n_step'] = np.int64(sim.em.engine.n_step)
    return out


def main():
    reference = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('OPENSOL_REFERENCE')
    if not reference:
        raise SystemExit('usage: make_golden_dft.py /path/to/reference')
    os.environ.setdefault('NUMBA_CACHE_DIR', os.path.join(tempfile.gettempdir(), 'opensol_numba_cache'))
    sys.dont_write_bytecode = True
    sys.path.insert(0, reference)
    sys.path.insert(0, HERE)
    import numpy as np
    from cases_dft import CASES_DFT, CASES_DFT_HZ
    only = set(sys.argv[2:])   # case names to regenerate (default: all)
    index_path = os.path.join(HERE, 'index_dft.json')
    index = {}
    if only and os.path.exists(index_path):
        with open(index_path) as f:
            index = json.load(f)['cases']
    for spec in CASES_DFT + CASES_DFT_HZ:
        if only and spec['name'] not in only:
            continue
        out = run_case(spec)
        np.savez_compressed(os.path.join(HERE, f"{spec['name']}.npz"), **out)
        index[spec['name']] = sorted(out)
        print(f"{spec['name']}: {len(out)} entries, m {int(out['sample_interval'])}")
    with open(index_path, 'w') as f:
        json.dump({'generated_by': 'tests/golden/make_golden_dft.py (open_sol CPU backend)', 'cases': index}, f,
                  indent=1)


if __name__ == '__main__':
    main()
