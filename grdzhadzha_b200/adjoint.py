"""Discrete adjoint of the FP64 Kerr-Schild operator (new; the reference has
no adjoint) over the C ABI.

`TorusAccretionAdjoint` evaluates
    J(theta) = integral over `steps` RK4 steps of the rest-mass accretion
               rate through the sphere r < accretion_radius
for a torus initial state with parameters
    theta = [amplitude, entropy, spin, mode_1, ..., mode_5]
(grhd_adjoint_torus) and its gradient dJ/dtheta by the checkpointed
discrete adjoint (grhd_adjoint_forward / grhd_adjoint_backward).  The step
size is fixed, so J is differentiated along a fixed step sequence.

`AccretionIntegral` wraps the forward/backward pair in a
torch.autograd.Function for the gradient test; the computation stays in
libgrhd_b200.so.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L
from .operator import LevelBox, _ptr, _stream

THETA_NAMES = ("amplitude", "entropy", "spin", "mode_1", "mode_2", "mode_3",
               "mode_4", "mode_5")


def default_torus(**overrides) -> L.AdjointTorus:
    lib = L.load()
    t = L.AdjointTorus()
    lib.grhd_default_adjoint_torus(C.byref(t))
    for k, v in overrides.items():
        if k in ("mode_amplitude", "mode_phase"):
            for m in range(5):
                getattr(t, k)[m] = v[m]
        else:
            setattr(t, k, v)
    return t


class TorusAccretionAdjoint:
    def __init__(self, operator, level: LevelBox, steps: int,
                 checkpoint_every: int, dt: float, torus=None):
        """operator: an FP64 Kerr-Schild operator with accretion_radius > 0
        (its spin is replaced by theta's); level: the whole-domain box (its
        state tensor is not used by the forward/backward pair)."""
        self._lib = L.load()
        self.op = operator
        self.level = level
        self.steps, self.every, self.dt = steps, checkpoint_every, dt
        self.torus = torus if torus is not None else default_torus()
        if self.torus.entropy <= 0.0:
            K = C.c_double()
            self._check(self._lib.grhd_adjoint_unit_entropy(
                C.byref(operator.params), C.byref(self.torus), C.byref(K)))
            self.torus.entropy = K.value
        h = C.c_void_p()
        box = level.c_box()
        st = self._lib.grhd_adjoint_create(C.byref(operator.params),
                                           C.byref(box), steps,
                                           checkpoint_every, dt, C.byref(h))
        self._h = h
        self._check(st)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.grhd_adjoint_destroy(h)
            self._h = None

    def _check(self, status):
        if status != L.GRHD_OK:
            h = getattr(self, "_h", None)
            L.check(self._lib, h if h else None, status,
                    self._lib.grhd_adjoint_last_error if h else None)

    # theta <-> grhd_adjoint_torus
    def theta(self) -> list:
        t = self.torus
        return [t.amplitude, t.entropy, t.spin] + list(t.mode_amplitude)

    def torus_of(self, theta) -> L.AdjointTorus:
        t = L.AdjointTorus()
        C.memmove(C.byref(t), C.byref(self.torus), C.sizeof(t))
        th = [float(x) for x in theta]
        t.amplitude, t.entropy, t.spin = th[0], th[1], th[2]
        for m in range(5):
            t.mode_amplitude[m] = th[3 + m]
        return t

    def launch_count(self) -> int:
        return int(self._lib.grhd_adjoint_launch_count(self._h))

    def forward(self, theta=None) -> float:
        t = self.torus_of(self.theta() if theta is None else theta)
        J = C.c_double()
        self._check(self._lib.grhd_adjoint_forward(self._h, C.byref(t),
                                                   C.byref(J), _stream()))
        return J.value

    def backward(self, lambda0: torch.Tensor | None = None) -> list:
        g = (C.c_double * 8)()
        lp, ls = None, 0
        if lambda0 is not None:
            lp, ls = _ptr(lambda0), lambda0[0].numel()
        self._check(self._lib.grhd_adjoint_backward(self._h, g, lp, ls,
                                                    _stream()))
        return list(g)

    def tangent(self, direction, theta=None) -> tuple:
        """Tangent-linear sweep (grhd_adjoint_tangent): (J, dJ) with dJ =
        sum_k direction[k] dJ/dtheta_k along the same discrete steps and
        branches as the adjoint, so dJ = <backward(), direction> to
        rounding.  Overwrites the forward's tape."""
        t = self.torus_of(self.theta() if theta is None else theta)
        v = (C.c_double * 8)(*[float(x) for x in direction])
        J, dJ = C.c_double(), C.c_double()
        self._check(self._lib.grhd_adjoint_tangent(
            self._h, C.byref(t), v, C.byref(J), C.byref(dJ), _stream()))
        return J.value, dJ.value

    def initial_state(self, theta=None, level: LevelBox | None = None):
        lv = level or LevelBox(lo=self.level.lo, hi=self.level.hi,
                               ghost=self.level.ghost,
                               device=self.level.state.device)
        t = self.torus_of(self.theta() if theta is None else theta)
        self._check(self._lib.grhd_adjoint_initial_data(
            self._h, C.byref(t), _ptr(lv.state), lv.comp_stride(), None, 0,
            _stream()))
        return lv

    def tangents(self, theta=None) -> torch.Tensor:
        """dU0/dtheta over the interior: (8, 5, nz, ny, nx)."""
        z, y, x = self.level.interior_shape
        out = torch.zeros((8, 5, z, y, x), dtype=torch.float64,
                          device=self.level.state.device)
        t = self.torus_of(self.theta() if theta is None else theta)
        self._check(self._lib.grhd_adjoint_initial_data(
            self._h, C.byref(t), None, 0, _ptr(out), x * y * z, _stream()))
        return out

    def rhs_vjp(self, level: LevelBox, rhs_bar: torch.Tensor,
                mdot_bar: float = 0.0):
        """(dRHS/dU)^T rhs_bar + mdot_bar dMdot/dU over the interior
        conserved variables, and the spin derivative, at the operator's
        spin."""
        out = torch.zeros_like(rhs_bar)
        sb = C.c_double()
        self._check(self._lib.grhd_adjoint_rhs_vjp(
            self._h, _ptr(level.state), level.comp_stride(), _ptr(rhs_bar),
            rhs_bar[0].numel(), float(mdot_bar), _ptr(out), out[0].numel(),
            C.byref(sb), _stream()))
        return out, sb.value

    def step_vjp(self, level: LevelBox, state_bar_next: torch.Tensor,
                 mdot_integral_bar: float = 0.0):
        """The adjoint of U^n for one RK4 step of size dt given that of
        U^{n+1} (interior conserved variables) and the weight of the step's
        accretion integral; and the spin derivative."""
        out = torch.zeros_like(state_bar_next)
        sb = C.c_double()
        self._check(self._lib.grhd_adjoint_step_vjp(
            self._h, _ptr(level.state), level.comp_stride(),
            _ptr(state_bar_next), state_bar_next[0].numel(),
            float(mdot_integral_bar), _ptr(out), out[0].numel(),
            C.byref(sb), _stream()))
        return out, sb.value


class AccretionIntegral(torch.autograd.Function):
    """J(theta) with the discrete adjoint as its backward (gradient test
    only)."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, adjoint: TorusAccretionAdjoint):
        J = adjoint.forward(theta.detach().cpu().tolist())
        ctx.adjoint = adjoint
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_J):
        g = torch.tensor(ctx.adjoint.backward(), dtype=torch.float64)
        return grad_J * g, None
