"""Batched ensemble of independent Kerr-Schild boxes (new; the reference
advances one level at a time).

Every member is one whole-domain box with its own operator settings (mass,
spin, EOS, floors, excision, accretion sphere, grid spacing); all members
share one precision.  `Ensemble.advance(steps)` runs `steps` classic RK4
steps of every member in one persistent kernel launch (optionally replayed
from a CUDA graph), each member with its own CFL step
dt = min(cfl / max inverse dt, max_dt): the step of `advance_rk4_cfl`,
reproduced to rounding."""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L


class Ensemble:
    def __init__(self, members, cfl=0.25, max_dt=0.0, time=0.0):
        """members: sequence of (operator, LevelBox); the LevelBox states are
        advanced in place and must stay alive as long as the ensemble.
        max_dt: one cap for all members or one per member (<= 0: none)."""
        self._lib = L.load()
        self._members = list(members)
        n = len(self._members)
        if n < 1:
            raise ValueError("an ensemble needs at least one member")
        arr = (L.EnsembleMember * n)()
        caps = (list(max_dt) if hasattr(max_dt, "__len__")
                else [max_dt] * n)
        if len(caps) != n:
            raise ValueError("one max_dt per member")
        for i, (op, lv) in enumerate(self._members):
            if not (lv.state.is_cuda and lv.state.dtype == torch.float64
                    and lv.state.is_contiguous()):
                raise ValueError("member states must be contiguous CUDA "
                                 "float64 tensors")
            m = arr[i]
            m.params = op.params
            m.box = lv.c_box()
            m.state = lv.state.data_ptr()
            m.state_comp_stride = lv.comp_stride()
            for d in range(3):
                m.inverse_dx[d] = 1.0 / op.dx
            m.cfl = cfl
            m.max_dt = float(caps[i])
            m.time = time
        self._arr = arr
        h = C.c_void_p()
        st = self._lib.grhd_ensemble_create(arr, n, C.byref(h))
        self._h = h
        self._check(st)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.grhd_ensemble_destroy(h)
            self._h = None

    close = __del__

    def _check(self, status):
        L.check(self._lib, self._h, status, self._lib.grhd_ensemble_last_error)

    @staticmethod
    def _stream():
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def __len__(self):
        return len(self._members)

    def advance(self, steps, use_graph=True):
        self._check(self._lib.grhd_ensemble_advance(
            self._h, int(steps), int(bool(use_graph)), self._stream()))

    def autotune(self, trial_steps=1) -> dict:
        t = L.EnsembleTuning()
        self._check(self._lib.grhd_ensemble_autotune(
            self._h, int(trial_steps), C.byref(t), self._stream()))
        return {"zchunk": t.zchunk, "blocks_per_sm": t.blocks_per_sm,
                "ms_per_step": t.ms_per_step}

    @property
    def tuning(self) -> dict:
        t = L.EnsembleTuning()
        mx = C.c_int()
        self._check(self._lib.grhd_ensemble_get_tuning(self._h, C.byref(t),
                                                       C.byref(mx)))
        return {"zchunk": t.zchunk, "blocks_per_sm": t.blocks_per_sm,
                "ms_per_step": t.ms_per_step,
                "max_blocks_per_sm": mx.value}

    def set_tuning(self, zchunk, blocks_per_sm):
        t = L.EnsembleTuning(int(zchunk), int(blocks_per_sm), 0.0)
        self._check(self._lib.grhd_ensemble_set_tuning(self._h, C.byref(t)))

    def member_info(self, i) -> dict:
        t, mi, m, integ = (C.c_double() for _ in range(4))
        d = L.Diagnostics()
        self._check(self._lib.grhd_ensemble_member_info(
            self._h, int(i), C.byref(t), C.byref(mi), C.byref(m),
            C.byref(integ), C.byref(d)))
        return {"time": t.value, "max_inverse_dt": mi.value,
                "mdot": m.value, "mdot_integral": integ.value,
                "diagnostics": d}

    def reset_accretion(self):
        self._check(self._lib.grhd_ensemble_reset_accretion(self._h))

    def invalidate(self):
        self._check(self._lib.grhd_ensemble_invalidate(self._h))

    def set_barrier_test(self, extra_arrivals, timeout_seconds):
        """Test hook: barriers wait for blocks that never arrive, so every
        wait runs out after timeout_seconds; (0, 4.0) restores."""
        self._check(self._lib.grhd_ensemble_set_barrier_test(
            self._h, int(extra_arrivals), float(timeout_seconds)))

    def launch_count(self) -> int:
        return int(self._lib.grhd_ensemble_launch_count(self._h))
