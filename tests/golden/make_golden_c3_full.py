"""Generate tests/golden/c3_full.npz: the whole 512^3 3D workload (opensol_b200.workloads.roofline_3d_physics: 500
seeded dielectric spheres, a centred 1310 nm z dipole, a closed 8-frequency flux box, CPML 12 on every face) run for
2,000 steps on the CPU by the oracle (tests/golden/cases3d.roofline_3d_oracle), in its float32 build (the engine's
arithmetic) and its float64 build (the run the float32 flux's error is stated against).

Stored, at steps 200 and 2,000: SHA-256 digests of the six float32 fields and of the flux box's complex128 E / H
spectra (every plane, both pairs), the box flux (8,) of the float32 run and of the float64 run; the DFT sample
interval.  The fields themselves (3.2 GB) are not stored; the digests pin them bit for bit.

    python tests/golden/make_golden_c3_full.py

About an hour on 8 host cores.
"""
import hashlib
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CHECKPOINTS = (200, 2_000)
FIELDS = ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')


def digest(array):
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def run(precision):
    import numpy as np
    from cases3d import roofline_3d_oracle
    o, box = roofline_3d_oracle(precision)
    out, done = {}, 0
    for cp in CHECKPOINTS:
        t = time.time()
        o.run(cp - done)
        done = cp
        print(f'{precision}: step {cp} ({time.time() - t:.0f} s)', flush=True)
        if precision == 'single':
            for name in FIELDS:
                out[f'sha_{name}_{cp}'] = digest(o.fields[name])
            for p, plane in enumerate(box.planes()):
                for q, pair in enumerate(plane.pairs):
                    out[f'sha_spec_e{p}{q}_{cp}'] = digest(pair['e_dft'])
                    out[f'sha_spec_h{p}{q}_{cp}'] = digest(pair['h_dft'])
        out[f'flux_{cp}'] = np.asarray(box.flux(), np.float64)
    out['sample_interval'] = np.int64(box.sample_interval)
    out['n_step'] = np.int64(o.n_step)
    return out


def main():
    import numpy as np
    sys.dont_write_bytecode = True
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    out = run('single')
    double = run('double')
    for cp in CHECKPOINTS:
        out[f'f64_flux_{cp}'] = double[f'flux_{cp}']
    path = os.path.join(HERE, 'c3_full.npz')
    np.savez_compressed(path, **out)
    f32, f64 = out['flux_2000'], out['f64_flux_2000']
    print(f'float32 vs float64 box flux at 2000 steps: max error relative to the peak '
          f'{np.abs(f32 - f64).max() / np.abs(f64).max():.3e}')
    print(f'wrote {path} ({len(out)} entries)')


if __name__ == '__main__':
    main()
