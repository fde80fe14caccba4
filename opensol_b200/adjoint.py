"""Gradient of a 2D FDTD flux objective with respect to eps_r on a design box, by the discrete adjoint on the device,
behind a torch.autograd.Function (no open_sol counterpart: open_sol has no FDTD adjoint).

Forward: the simulation runs from rest for n_steps on the engine's fast kernels, saving its full state (fields and
CPML psi) every `checkpoint_every` steps in device memory; J = monitor.flux()[freq_index].  Backward: from the last
segment to the first, the segment is recomputed from its checkpoint while E on the design box is recorded, then the
exact transpose of every step runs backward through it (opensol_b200/csrc/fdtd2d_adjoint.cuh), the DFT samples of
the objective's monitor entering as adjoint sources.  Inside the design box (no source, no CPML, lossless) a step is
E^{n+1} = E^n + cb curl H with cb = dt / (eps_r eps0), so dJ/deps_r = -(1 / eps_r) sum_n lambda_E^{n+1} (E^{n+1} -
E^n).  Cost: one forward, one recomputation, one adjoint sweep.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _native
from .constants import DTYPE


class FluxAdjoint2D:
    """d(flux)/d(eps_r) on cells box = (i0, i1, j0, j1) of a finalized 2D simulation `sim` whose monitor `monitor`
    defines J = monitor.flux()[freq_index] after n_steps.  The box must avoid CPML, sources and monitors and be
    lossless (sigma_e = 0)."""

    def __init__(self, sim, monitor, freq_index, box, n_steps, checkpoint_every=256):
        self.sim = sim
        self.engine = sim.em.engine
        self.monitor = monitor
        self.freq_index = int(freq_index)
        self.box = tuple(int(b) for b in box)
        self.n_steps = int(n_steps)
        self.K = int(checkpoint_every)
        self.n_slots = max(1, math.ceil(self.n_steps / self.K))
        i0, i1, j0, j1 = self.box
        self.box_slices = (slice(i0, i1), slice(j0, j1))
        engine = self.engine
        engine.sync_device()
        out = ctypes.c_void_p()
        _native.check(_native.load().os_fdtd2d_adjoint_create(engine.handle, i0, i1, j0, j1, self.n_slots, self.K,
                                                              ctypes.byref(out)))
        self._handle = out
        self._tables = None
        self._slot_tables = None   # per checkpoint segment: the chunk tables of its steps (clock from rest)

    def close(self):
        if self._handle is not None:
            _native.load().os_fdtd2d_adjoint_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- forward
    def set_design(self, eps_box):
        """Write eps_r on the box (the device coefficients follow at the next sync)."""
        eps_box = np.asarray(eps_box, dtype=DTYPE)
        materials = self.sim.domain.materials
        materials.array('eps_r')[self.box_slices] = eps_box
        materials.version += 1   # an in-place write: the engine re-uploads the coefficients at the next sync
        self.sim.em.materials_changed(('eps_r',))

    def _prepare_tables(self):
        """The source values and DFT phases of the whole run and of each checkpoint segment, for a run from rest.
        They depend on the clock, the sources' waveforms and the monitors' frequencies only, not on eps_r, so they are
        built once and reused by every forward."""
        engine = self.engine
        engine.reset()
        self._tables = engine.chunk_tables(self.n_steps)
        slots = []
        for slot in range(self.n_slots):
            n = min(self.K, self.n_steps - slot * self.K)
            tables = engine.chunk_tables(n)
            slots.append(tables)
            engine.n_step += n          # the clock of the next segment's tables (no device work)
            engine.time = tables[-1]
        engine.reset()
        self._slot_tables = slots

    def forward(self, eps_box=None):
        """Run from rest; returns J."""
        if eps_box is not None:
            self.set_design(eps_box)
        engine = self.engine
        self.sim.em.finalize()
        if self._slot_tables is None:
            self._prepare_tables()
        engine.reset()
        lib = _native.load()
        for slot in range(self.n_slots):
            _native.check(lib.os_fdtd2d_adjoint_save(self._handle, slot))
            engine.advance(min(self.K, self.n_steps - slot * self.K), self._slot_tables[slot])
        return float(self.monitor.flux()[self.freq_index])

    # ---- backward
    def _adjoint_sources(self):
        """Per DFT sample of the monitor: (step index, dJ/de, dJ/dh) on its line cells."""
        mon = self.monitor
        values, first_q, n_q, phases, _ = self._tables
        m = self.engine.sample_interval
        offset = 0
        for other in self.engine._monitors:
            if other is mon:
                break
            offset += n_q * other.n_freqs * 2
        table = phases[offset:offset + n_q * mon.n_freqs * 2].reshape(n_q, mon.n_freqs, 2)
        f = mon.frequencies[self.freq_index]
        r = np.exp(1j * np.pi * f * mon.dt)
        e_spec, h_spec = mon.spectra()
        E_c, H_c = e_spec[self.freq_index], h_spec[self.freq_index]
        scale = np.cos(np.pi * f * mon.dt) * mon._flux_sign * mon._cell_widths
        out = []
        for qi in range(n_q):
            q = first_q + qi
            ph = (table[qi, self.freq_index, 0].astype(np.float64)
                  + 1j * table[qi, self.freq_index, 1].astype(np.float64))
            de = scale * np.real(ph * np.conj(H_c * r))
            dh = scale * np.real(E_c * np.conj(ph * r))
            out.append((q * m - 1, de, dh))
        return out

    def backward(self):
        """dJ/deps_r on the box (float64), after forward()."""
        if self._tables is None:
            raise RuntimeError('FluxAdjoint2D.backward needs a forward run first')
        lib = _native.load()
        values = self._tables[0]
        sources = self._adjoint_sources()
        # the adjoint is linear: run it with sources of unit size and scale the gradient back (float32 headroom)
        peak = max((max(float(np.abs(de).max()), float(np.abs(dh).max())) for _, de, dh in sources), default=0.0)
        if peak == 0.0:
            return np.zeros((self.box[1] - self.box[0], self.box[3] - self.box[2]))
        monitor_id = self.engine._monitor_ids[id(self.monitor)]
        _native.check(lib.os_fdtd2d_adjoint_reset(self._handle))
        for slot in range(self.n_slots - 1, -1, -1):
            step0 = slot * self.K
            n = min(self.K, self.n_steps - step0)
            seg = [(k - step0, de / peak, dh / peak) for k, de, dh in sources if step0 <= k < step0 + n]
            steps = (ctypes.c_int32 * max(1, len(seg)))(*[k for k, _, _ in seg])
            src_e = np.ascontiguousarray(np.stack([de for _, de, _ in seg]) if seg else np.zeros((1, 1)), DTYPE)
            src_h = np.ascontiguousarray(np.stack([dh for _, _, dh in seg]) if seg else np.zeros((1, 1)), DTYPE)
            seg_values = np.ascontiguousarray(values[:, step0:step0 + n], DTYPE)
            _native.check(lib.os_fdtd2d_adjoint_segment(
                self._handle, slot, step0, n, _native.fptr(seg_values) if seg_values.size else None, monitor_id,
                len(seg), steps, _native.fptr(src_e), _native.fptr(src_h)))
        grad = np.empty((self.box[1] - self.box[0], self.box[3] - self.box[2]), np.float64)
        _native.check(lib.os_fdtd2d_adjoint_gradient(self._handle, _native.dptr(grad)))
        eps = self.sim.domain.materials.array('eps_r')[self.box_slices].astype(np.float64)
        self.engine.n_step = self.n_steps
        return -grad * peak / eps


def flux_objective(adjoint):
    """A torch.autograd.Function applying `adjoint` (a FluxAdjoint2D): f(eps_box) = J, df/deps_box by the adjoint."""
    import torch

    class _FluxObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, eps_box):
            value = adjoint.forward(eps_box.detach().cpu().numpy())
            ctx.device, ctx.dtype = eps_box.device, eps_box.dtype
            return torch.tensor(value, dtype=torch.float64, device=eps_box.device)

        @staticmethod
        def backward(ctx, grad_output):
            grad = adjoint.backward()
            return (grad_output.to(torch.float64) * torch.from_numpy(grad).to(ctx.device)).to(ctx.dtype)

    return _FluxObjective.apply
