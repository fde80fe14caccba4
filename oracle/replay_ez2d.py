"""ORACLE -- BENCH / TEST INFRASTRUCTURE ONLY.

Nothing in the product (``opensol_b200``) imports this module.  bench.py's reference-replay leg and tests/ use it to
time open_sol's own GPU step of the 2D E_z engine (its cupy RawKernel path, which needs cupy and so cannot run in this
image) on the same grid as the engine: the reference's update_h_kernel / update_e_kernel compiled unchanged
(oracle/make_ref_replay.py) and replayed with the reference's launch shapes and sequence by oracle/replay_ez2d.cu,
the setup arrays taken from the oracle (which reproduces open_sol's setup bit for bit).  Device buffers are torch
tensors (plumbing only).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from oracle.fdtd2d import FACES

_HERE = os.path.dirname(os.path.abspath(__file__))
CUBIN = os.path.join(_HERE, '_ref', 'ez2d_rawkernels.cubin')
LIB = os.path.join(_HERE, '_build', 'libreplay_ez2d.so')
_P = ctypes.c_void_p


class _Side(ctypes.Structure):
    _fields_ = [('axis', ctypes.c_int), ('npml', ctypes.c_int), ('e_row0', ctypes.c_int), ('h_row0', ctypes.c_int),
                ('sign', ctypes.c_float)] + [(n, _P) for n in ('b_e', 'a_e', 'inv_e', 'b_h', 'a_h', 'inv_h', 'psi_e',
                                                                'psi_h')]


class _Monitor(ctypes.Structure):
    _fields_ = [('normal_axis', ctypes.c_int), ('position', ctypes.c_int), ('lo', ctypes.c_int),
                ('hi', ctypes.c_int), ('nf', ctypes.c_int), ('omega', _P), ('dt_m', ctypes.c_double),
                ('phases', _P), ('e_acc', _P), ('h_acc', _P)]


class _Config(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int), ('ny', ctypes.c_int)] + \
               [(n, _P) for n in ('ez', 'hx', 'hy', 'ca', 'cb', 'da', 'db', 'inv_dx_e', 'inv_dx_h', 'inv_dy_e',
                                  'inv_dy_h')] + \
               [('n_sides', ctypes.c_int), ('sides', _Side * 4), ('src_axis', ctypes.c_int),
                ('src_position', ctypes.c_int), ('src_lo', ctypes.c_int), ('src_hi', ctypes.c_int),
                ('profile', _P), ('n_monitors', ctypes.c_int), ('monitors', _Monitor * 8),
                ('sample_interval', ctypes.c_int)]


def available():
    """(True, '') when the reference's kernels were compiled here, else (False, why)."""
    if not os.path.exists(CUBIN):
        return False, ('the reference kernels were not compiled (oracle/make_ref_replay.py needs the reference '
                       'source tree)')
    return True, ''


def load_library():
    if not os.path.exists(LIB):
        subprocess.run(['make', '-s', '-C', _HERE, 'replay'], check=True)
    lib = ctypes.CDLL(LIB)
    lib.replay_ez2d_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Config), ctypes.POINTER(_P)]
    lib.replay_ez2d_reset.argtypes = [_P]
    lib.replay_ez2d_run.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)]
    lib.replay_ez2d_destroy.argtypes = [_P]
    lib.replay_ez2d_destroy.restype = None
    lib.replay_ez2d_last_error.restype = ctypes.c_char_p
    return lib


class ReferenceReplayEz2D:
    """open_sol's GPU step replayed on `device` for a finalized OracleEz2D `oracle` with CPML on every side or none,
    at most one line source and up to 8 flux monitors (the benchmark workloads' features)."""

    def __init__(self, oracle, device=0):
        import torch
        ok, why = available()
        if not ok:
            raise RuntimeError(why)
        if not oracle._finalized:
            oracle.finalize()
        if len(oracle.sources) > 1 or oracle.tfsf or oracle.poles or oracle.maps or oracle.probes:
            raise ValueError('the replay covers line sources (at most one) and flux monitors only')
        if any(kind != 'cpml' for kind in oracle.domain.faces.values()):
            raise ValueError('the replay covers domains with CPML on every side')
        self.oracle = oracle
        self.lib = load_library()
        self.device = torch.device('cuda', device)
        torch.cuda.set_device(self.device)
        d = oracle.domain
        self.nx, self.ny = d.nx, d.ny
        keep = self._keep = []

        def dev(array, dtype=None):
            t = torch.from_numpy(np.ascontiguousarray(array if dtype is None else array.astype(dtype))).to(self.device)
            keep.append(t)
            return t

        cfg = _Config()
        cfg.nx, cfg.ny = self.nx, self.ny
        self.fields = {n: torch.zeros((self.nx, self.ny), dtype=torch.float32, device=self.device)
                       for n in ('ez', 'hx', 'hy')}
        for n, t in self.fields.items():
            setattr(cfg, n, t.data_ptr())
        for n in ('ca', 'cb', 'da', 'db'):
            setattr(cfg, n, dev(getattr(oracle, n), np.float32).data_ptr())
        for n in ('inv_dx_e', 'inv_dx_h', 'inv_dy_e', 'inv_dy_h'):
            setattr(cfg, n, dev(oracle.curl[n], np.float32).data_ptr())
        cfg.n_sides = len(oracle.cpml_sides)
        for k, side in enumerate(sorted(oracle.cpml_sides, key=lambda s: FACES.index(s.name))):
            rec = cfg.sides[k]
            rec.axis = 0 if side.name[0] == 'x' else 1
            rec.npml = d.npml
            rec.e_row0, rec.h_row0 = side.e_rows.start, side.h_rows.start
            rec.sign = 1.0 if rec.axis == 0 else -1.0
            for n in ('b_e', 'a_e', 'inv_e', 'b_h', 'a_h', 'inv_h'):
                setattr(rec, n, dev(getattr(side, n), np.float32).data_ptr())
            shape = (d.npml, self.ny) if rec.axis == 0 else (self.nx, d.npml)
            rec.psi_e = dev(np.zeros(shape, np.float32)).data_ptr()
            rec.psi_h = dev(np.zeros(shape, np.float32)).data_ptr()
        if oracle.sources:
            src = oracle.sources[0]
            cfg.src_axis = 0 if src.axis == 'x' else 1
            cfg.src_position, cfg.src_lo, cfg.src_hi = src.position, src.lo, src.hi
            cfg.profile = dev(src.profile, np.float32).data_ptr()
        else:
            cfg.src_axis = -1
        self.spectra = []
        cfg.n_monitors = len(oracle.monitors)
        for k, mon in enumerate(oracle.monitors):
            rec = cfg.monitors[k]
            rec.normal_axis = 0 if mon.normal_axis == 'x' else 1
            rec.position, rec.lo, rec.hi = mon.position, mon.lo, mon.hi
            rec.nf = mon.frequencies.size
            rec.omega = dev(2.0 * np.pi * mon.frequencies, np.float64).data_ptr()
            rec.dt_m = float(mon.dt) * oracle.sample_interval
            rec.phases = dev(np.zeros((rec.nf, 2), np.float32)).data_ptr()
            e = torch.zeros((rec.nf, mon.hi - mon.lo), dtype=torch.complex128, device=self.device)
            h = torch.zeros_like(e)
            self.spectra.append((e, h))
            rec.e_acc, rec.h_acc = e.data_ptr(), h.data_ptr()
        cfg.sample_interval = oracle.sample_interval
        self.cfg = cfg
        torch.cuda.synchronize(self.device)
        handle = _P()
        if self.lib.replay_ez2d_create(CUBIN.encode(), ctypes.byref(cfg), ctypes.byref(handle)):
            raise RuntimeError(self.lib.replay_ez2d_last_error().decode())
        self.handle = handle
        self.n_step = 0
        self.time = 0.0

    def _schedule(self, n_steps):
        """Per-step float32 source values and the clock after each sampled step (the oracle's own clock rules)."""
        dt = float(self.oracle.domain.dt)
        values = np.zeros(max(n_steps, 1), np.float32)
        samples = []
        t = self.time
        src = self.oracle.sources[0] if self.oracle.sources else None
        m = self.oracle.sample_interval
        for k in range(n_steps):
            if src is not None:
                values[k] = np.float32(src.amplitude * src.temporal(t + 0.5 * dt))
            t = t + dt
            if (self.n_step + k + 1) % m == 0:
                samples.append(t)
        return values, np.asarray(samples if samples else [0.0], np.float64), t

    def run(self, n_steps):
        """Advance n_steps; returns the device milliseconds of the whole run (CUDA events on the replay stream)."""
        values, samples, t_end = self._schedule(n_steps)
        ms = ctypes.c_float()
        if self.lib.replay_ez2d_run(self.handle, self.n_step, n_steps,
                                    values.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                    samples.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(ms)):
            raise RuntimeError(self.lib.replay_ez2d_last_error().decode())
        self.n_step += n_steps
        self.time = t_end
        return float(ms.value)

    def reset(self):
        if self.lib.replay_ez2d_reset(self.handle):
            raise RuntimeError(self.lib.replay_ez2d_last_error().decode())
        self.n_step, self.time = 0, 0.0

    def field(self, name):
        return self.fields[name].cpu().numpy()

    def flux(self, k):
        """Flux of monitor k from the replayed spectra (the oracle monitor's own readout formula)."""
        mon = self.oracle.monitors[k]
        e, h = (s.cpu().numpy() for s in self.spectra[k])
        saved = mon.e_acc, mon.h_acc
        try:
            mon.e_acc, mon.h_acc = e, h
            return np.asarray(mon.flux())
        finally:
            mon.e_acc, mon.h_acc = saved

    def close(self):
        if getattr(self, 'handle', None):
            self.lib.replay_ez2d_destroy(self.handle)
            self.handle = None
