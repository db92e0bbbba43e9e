"""Python mirror of the reference operator classes over the C ABI.

Names, arguments and error behaviour follow GRDzhadzha's
Source/Matter/GRHD/FixedBGFArrayBoxFiniteVolume.hpp:

  FixedBGLevelDataFiniteVolumeOperator(eos, background, dx, center,
      atmosphere, limiter_theta, use_reconstruction, recovery_options,
      use_static_metric_sources)                                   :446-614
  TimeDependentFixedBGLevelDataFiniteVolumeOperator(eos, background_factory,
      dx, center, atmosphere, limiter_theta, use_reconstruction,
      recovery_options, use_static_metric_sources,
      use_metric_volume_time_sources, metric_time_derivative_step)  :677-830

A level here is one box (`LevelBox`) holding a CUDA float64 tensor of shape
(11, nz + 2g, ny + 2g, nx + 2g) in the FArrayBox component order
D, S1, S2, S3, tau, rho, eps, pressure, v1, v2, v3.  torch only supplies the
device memory and the stream; all arithmetic runs in libgrhd_b200.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import torch

from . import _lib as L

D, S1, S2, S3, TAU, RHO, EPS, PRESSURE, V1, V2, V3 = range(11)


# ---------------------------------------------------------------- options


@dataclass
class IdealGasEOS:
    """IdealGasEOS.hpp:10-53"""
    adiabatic_index: float = 5.0 / 3.0


@dataclass
class AtmosphereOptions:
    """Atmosphere.hpp:16-22"""
    rho_floor: float = 1.0e-12
    pressure_floor: float = 1.0e-12
    max_velocity_squared: float = 1.0 - 1.0e-12
    metric_source_atmosphere_factor: float = 1.0 + 1.0e-12


@dataclass
class RecoveryOptions:
    """Valencia.hpp:17-23"""
    max_iterations: int = 50
    tolerance: float = 1.0e-12
    pressure_floor: float = 1.0e-12
    max_velocity_squared: float = 1.0 - 1.0e-12


@dataclass
class KerrSchild:
    """KerrSchild.hpp:22-90 (params_t + dx).  The hole sits at the
    operator centre; `center` is kept for interface parity."""
    mass: float = 1.0
    spin: float = 0.0
    center: Sequence[float] = (0.0, 0.0, 0.0)
    dx: float = 1.0

    def __post_init__(self):
        if self.spin > self.mass or self.spin < -self.mass:
            raise ValueError("The dimensionless spin parameter must be in the "
                             "range -1.0 < spin < 1.0")


@dataclass
class CircularBinaryPN:
    """CircularBinaryPN.hpp:29-57 (params_t + dx).  Used directly as the
    time-dependent operator's background factory: factory(t) is this
    binary with params.time + t (Tests/GRHDFixedBGTest/GRHDFixedBGTest.cpp:
    435-446)."""
    mass_1: float = 0.5
    mass_2: float = 0.5
    separation: float = 10.0
    angular_velocity: float = 0.0
    phase: float = 0.0
    time: float = 0.0
    softening_radius: float = 0.5
    center: Sequence[float] = (0.0, 0.0, 0.0)
    dx: float = 1.0

    def __post_init__(self):
        if (self.mass_1 <= 0.0 or self.mass_2 <= 0.0 or self.separation <= 0.0
                or self.softening_radius < 0.0):
            raise ValueError("Invalid CircularBinaryPN parameters")


# ------------------------------------------------------------------ level


@dataclass
class LevelBox:
    """One box of a level: interior [lo, hi], ghost width, problem domain
    and the device state tensor over the ghosted box."""
    lo: tuple
    hi: tuple
    ghost: int = 2
    domain_lo: tuple | None = None
    domain_hi: tuple | None = None
    state: torch.Tensor | None = field(default=None, repr=False)
    device: str = "cuda"
    ncomp: int = 11  # 36 (CCZ4 + GRHD) for LevelDataFiniteVolumeOperator

    def __post_init__(self):
        if self.domain_lo is None:
            self.domain_lo = tuple(self.lo)
        if self.domain_hi is None:
            self.domain_hi = tuple(self.hi)
        if self.state is None:
            g = self.ghost
            n = [self.hi[d] - self.lo[d] + 1 + 2 * g for d in range(3)]
            self.state = torch.zeros((self.ncomp, n[2], n[1], n[0]),
                                     dtype=torch.float64, device=self.device)

    @classmethod
    def cube(cls, n, ghost=2, device="cuda"):
        nn = (n, n, n) if isinstance(n, int) else tuple(n)
        return cls(lo=(0, 0, 0), hi=tuple(x - 1 for x in nn), ghost=ghost,
                   device=device)

    @property
    def interior_shape(self):
        return tuple(self.hi[d] - self.lo[d] + 1 for d in (2, 1, 0))

    @property
    def num_cells(self) -> int:
        s = self.interior_shape
        return s[0] * s[1] * s[2]

    def interior(self, comps=slice(0, 11)) -> torch.Tensor:
        g = self.ghost
        z, y, x = self.interior_shape
        return self.state[comps, g:g + z, g:g + y, g:g + x]

    def c_box(self) -> L.Box:
        b = L.Box()
        for d in range(3):
            b.lo[d], b.hi[d] = self.lo[d], self.hi[d]
            b.domain_lo[d], b.domain_hi[d] = self.domain_lo[d], self.domain_hi[d]
        b.ghost = self.ghost
        return b

    def comp_stride(self) -> int:
        return self.state[0].numel()

    def new_rhs(self) -> torch.Tensor:
        return torch.zeros((5,) + self.interior_shape, dtype=torch.float64,
                           device=self.state.device)


def level_exchange(boxes) -> None:
    """LevelData<FArrayBox>::exchange() over the LevelBoxes of one level
    (grhd_level_exchange_components): ghost cells inside the problem domain
    take all components of the box that owns them (11 GRHD ones, or 36 for
    the operator on CCZ4-stored geometry)."""
    lib = L.load()
    n = len(boxes)
    arr = (L.Box * n)(*[b.c_box() for b in boxes])
    ptrs = (C.c_void_p * n)(*[_ptr(b.state).value for b in boxes])
    strides = (C.c_int64 * n)(*[b.comp_stride() for b in boxes])
    ncomp = {int(b.state.shape[0]) for b in boxes}
    if len(ncomp) != 1:
        raise ValueError("the boxes of a level hold the same components")
    err = C.create_string_buffer(256)
    st = lib.grhd_level_exchange_components(arr, ptrs, strides, n,
                                            ncomp.pop(), err, 256, _stream())
    if st != L.GRHD_OK:
        cls = L.InvalidArgument if st == L.GRHD_ERR_INVALID_ARG \
            else L.GRHDError
        e = cls(st, None)
        e.args = (err.value.decode(),)
        raise e


def kitp_config(**kw) -> L.KitpConfig:
    """The disk driver's source-term settings (SimulationConfig,
    Main_GRHDLevelDataBinaryPNKITPDisk.cpp:63-71 defaults) with
    overrides."""
    lib = L.load()
    c = L.KitpConfig()
    lib.grhd_default_kitp_config(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _ptr(t: torch.Tensor):
    if not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA float64 tensor")
    return C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


# --------------------------------------------------------------- operators


class _OperatorBase:
    def __init__(self, eos, background, dx, center, atmosphere,
                 limiter_theta, use_reconstruction, recovery_options,
                 use_static_metric_sources, use_metric_volume_time_sources,
                 metric_time_derivative_step, excision_radius,
                 accretion_radius=0.0, precision="fp64"):
        if not dx > 0.0:
            raise ValueError("GRHD grid spacing must be positive")
        self._lib = L.load()
        p = L.Params()
        self._lib.grhd_default_params(C.byref(p))
        if isinstance(background, KerrSchild):
            p.background = L.GRHD_BG_KERR_SCHILD
            p.ks_mass, p.ks_spin = background.mass, background.spin
        elif isinstance(background, CircularBinaryPN):
            p.background = L.GRHD_BG_BINARY_PN
            p.pn_mass_1, p.pn_mass_2 = background.mass_1, background.mass_2
            p.pn_separation = background.separation
            p.pn_angular_velocity = background.angular_velocity
            p.pn_phase, p.pn_time = background.phase, background.time
            p.pn_softening_radius = background.softening_radius
        else:
            raise TypeError("background must be KerrSchild or CircularBinaryPN")
        p.adiabatic_index = eos.adiabatic_index
        p.dx = dx
        for d in range(3):
            p.center[d] = center[d]
        a = atmosphere or AtmosphereOptions()
        p.rho_floor, p.pressure_floor = a.rho_floor, a.pressure_floor
        p.max_velocity_squared = a.max_velocity_squared
        p.metric_source_atmosphere_factor = a.metric_source_atmosphere_factor
        r = recovery_options or RecoveryOptions()
        p.recovery_max_iterations = r.max_iterations
        p.recovery_tolerance = r.tolerance
        p.recovery_pressure_floor = r.pressure_floor
        p.recovery_max_velocity_squared = r.max_velocity_squared
        p.limiter_theta = limiter_theta
        p.use_reconstruction = int(use_reconstruction)
        p.use_static_metric_sources = int(use_static_metric_sources)
        p.use_metric_volume_time_sources = int(use_metric_volume_time_sources)
        p.metric_time_derivative_step = metric_time_derivative_step
        p.excision_radius = excision_radius
        p.accretion_radius = accretion_radius
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        p.precision = (L.GRHD_PRECISION_MIXED if precision == "mixed"
                       else L.GRHD_PRECISION_FP64)
        self.precision = precision
        self.params = p
        self.dx = dx
        self.eos = eos
        self.background = background
        ctx = C.c_void_p()
        L.check(self._lib, None, self._lib.grhd_create(C.byref(p),
                                                       C.byref(ctx)))
        self._ctx = ctx

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx:
            self._lib.grhd_destroy(ctx)
            self._ctx = None

    def _inv(self, inverse_dx_U):
        v = inverse_dx_U if inverse_dx_U is not None else [1.0 / self.dx] * 3
        return (C.c_double * 3)(*v)

    def _check(self, status):
        L.check(self._lib, self._ctx, status)

    # ---- methods of the reference operator ----

    def _compute_rhs(self, rhs, state: LevelBox, inverse_dx_U, time):
        b = state.c_box()
        self._check(self._lib.grhd_compute_rhs(
            self._ctx, _ptr(rhs), rhs[0].numel(), _ptr(state.state),
            state.comp_stride(), C.byref(b), self._inv(inverse_dx_U), time,
            _stream()))

    def _recover_primitives(self, state: LevelBox, time):
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_recover_primitives(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            time, C.byref(d), _stream()))
        return d

    def _update_conserved(self, state, rhs, dt, recovery_time, recover):
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_update_conserved(
            self._ctx, _ptr(state.state), state.comp_stride(), _ptr(rhs),
            rhs[0].numel(), C.byref(b), dt, recovery_time, int(recover),
            C.byref(d), _stream()))
        return d

    def _compute_max_inverse_dt(self, state, inverse_dx_U, time):
        out = C.c_double()
        b = state.c_box()
        self._check(self._lib.grhd_compute_max_inverse_dt(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), time, C.byref(out), _stream()))
        return out.value

    def _compute_stable_dt(self, state, inverse_dx_U, cfl, time):
        if not cfl > 0.0:
            raise L.InvalidArgument(L.GRHD_ERR_INVALID_ARG, None)
        out = C.c_double()
        b = state.c_box()
        self._check(self._lib.grhd_compute_stable_dt(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), cfl, time, C.byref(out), _stream()))
        return out.value

    def _advance(self, fn, state, inverse_dx_U, time, dt):
        d = L.Diagnostics()
        b = state.c_box()
        self._check(fn(self._ctx, _ptr(state.state), state.comp_stride(),
                       C.byref(b), self._inv(inverse_dx_U), time, dt,
                       C.byref(d), _stream()))
        return d

    def ssprk2_stage(self, stage, state: LevelBox, stage_state: LevelBox,
                     dt, inverse_dx_U=None, time=0.0):
        """One of the two halves of advance_ssprk2 (:563-589) for a level
        whose ghosts the caller exchanges before each (grhd_ssprk2_stage):
        1: stage_state = state + dt L(state); 2: state = (state +
        stage_state + dt L(stage_state)) / 2; each recovered."""
        if tuple(stage_state.lo) != tuple(state.lo) or \
                tuple(stage_state.hi) != tuple(state.hi):
            raise ValueError("state and stage state cover different boxes")
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_ssprk2_stage(
            self._ctx, int(stage), _ptr(state.state), state.comp_stride(),
            _ptr(stage_state.state), stage_state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), time, dt, C.byref(d), _stream()))
        return d

    def advance_level_ssprk2(self, boxes, stage_boxes, dt, inverse_dx_U=None,
                             time=0.0):
        """advance_ssprk2 of a level of several boxes on this device: the
        reference's sequence (:563-589) with LevelData::exchange() before
        each RHS (grhd_level_exchange).  stage_boxes: one scratch LevelBox
        per box, same boxes."""
        level_exchange(boxes)
        for b, sb in zip(boxes, stage_boxes):
            self.ssprk2_stage(1, b, sb, dt, inverse_dx_U, time)
        level_exchange(stage_boxes)
        for b, sb in zip(boxes, stage_boxes):
            self.ssprk2_stage(2, b, sb, dt, inverse_dx_U, time)

    def ccz4_state(self, state: LevelBox, time=0.0) -> LevelBox:
        """A 36-component LevelBox for LevelDataFiniteVolumeOperator: the
        CCZ4 variables of this operator's analytic background over the
        ghosted box (as the reference's store_ccz4_background_vars,
        Tests/GRHDFixedBGTest/GRHDFixedBGTest.cpp:97-134: chi =
        det(gamma)^(-1/3), h = gamma chi, A = K_ij chi - K h / 3, trace K,
        lapse, shift; the others zero), then the 11 GRHD components of
        `state`.  The metric comes from grhd_eval_background."""
        g = state.ghost
        dev = state.state.device
        idx = [torch.arange(state.lo[d] - g, state.hi[d] + g + 1,
                            dtype=torch.float64, device=dev)
               for d in range(3)]
        z, y, x = torch.meshgrid(idx[2], idx[1], idx[0], indexing="ij")
        c = self.params.center
        xyz = torch.stack([(x + 0.5) * self.dx - c[0],
                           (y + 0.5) * self.dx - c[1],
                           (z + 0.5) * self.dx - c[2]], dim=-1).reshape(-1, 3)
        xyz = xyz.contiguous()
        out = torch.empty((xyz.shape[0], 64), dtype=torch.float64, device=dev)
        self._check(self._lib.grhd_eval_background(
            self._ctx, xyz.shape[0], _ptr(xyz), time, _ptr(out), _stream()))
        gm = out[:, 0:9].reshape(-1, 3, 3)
        Kt = out[:, 9:18].reshape(-1, 3, 3)
        trK, lapse, shift = out[:, 18], out[:, 19], out[:, 20:23]
        det = (gm[:, 0, 0] * gm[:, 1, 1] * gm[:, 2, 2]
               + 2 * gm[:, 0, 1] * gm[:, 0, 2] * gm[:, 1, 2]
               - gm[:, 0, 0] * gm[:, 1, 2] * gm[:, 1, 2]
               - gm[:, 1, 1] * gm[:, 0, 2] * gm[:, 0, 2]
               - gm[:, 2, 2] * gm[:, 0, 1] * gm[:, 0, 1])
        chi = torch.pow(det, -1.0 / 3.0)
        shape = state.state.shape[1:]
        lv = LevelBox(lo=state.lo, hi=state.hi, ghost=g,
                      domain_lo=state.domain_lo, domain_hi=state.domain_hi,
                      device=str(dev), ncomp=36)
        v = lv.state
        v[0] = chi.reshape(shape)
        pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
        for q, (a, b) in enumerate(pairs):
            h = gm[:, a, b] * chi
            v[1 + q] = h.reshape(shape)
            v[8 + q] = (Kt[:, a, b] * chi - trK * h / 3.0).reshape(shape)
        v[7] = trK.reshape(shape)
        v[18] = lapse.reshape(shape)
        for d in range(3):
            v[19 + d] = shift[:, d].reshape(shape)
        v[25:] = state.state
        return lv

    # ---- initial data (FixedBGTorus.hpp, Michel test) ----

    def fill_torus(self, state: LevelBox, inner_radius, pressure_max_radius,
                   rho_peak=1.0, total_mass=1.0, max_velocity_squared=None,
                   time=0.0):
        """make_fixed_bg_torus_parameters + fill_fixed_bg_torus_level_data
        (FixedBGTorus.hpp:291-409) on the device; returns the torus
        parameters (ell, surface_potential, polytropic_constant,
        max_enthalpy)."""
        c = L.TorusConfig()
        self._lib.grhd_default_torus_config(C.byref(c))
        c.total_mass, c.inner_radius = total_mass, inner_radius
        c.pressure_max_radius, c.rho_peak = pressure_max_radius, rho_peak
        if max_velocity_squared is not None:
            c.max_velocity_squared = max_velocity_squared
        out = L.TorusParams()
        b = state.c_box()
        self._check(self._lib.grhd_torus_initial_data(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            C.byref(c), time, C.byref(out), _stream()))
        return out

    def fill_michel(self, state: LevelBox, sonic_radius=8.0,
                    sonic_density=1.0e-6, atmosphere_radius=4.0,
                    mass=1.0, root_tolerance=1.0e-13):
        """fill_michel_state (Tests/GRHDLevelDataMichelAccretion:312-372)."""
        c = L.MichelConfig(mass, sonic_radius, sonic_density,
                           atmosphere_radius, root_tolerance)
        b = state.c_box()
        self._check(self._lib.grhd_michel_initial_data(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            C.byref(c), _stream()))

    def fill_kitp_disk(self, state: LevelBox, time=0.0, **config):
        """The binary disk drivers' Keplerian disk (kitp_primitive +
        fill_kitp_level_data, Main_GRHDLevelDataBinaryPNKITPDisk.cpp:
        398-555) on the device, SimulationConfig defaults (:56-61) with
        `config` overrides (mach, aspect_ratio, cavity_radius_factor,
        cavity_delta, outer_cutoff_radius, rho_peak, mode_amplitude[4],
        mode_phase[4]); needs the CircularBinaryPN background."""
        c = L.KitpDiskConfig()
        self._lib.grhd_default_kitp_disk_config(C.byref(c))
        for k, v in config.items():
            if k in ("mode_amplitude", "mode_phase"):
                arr = getattr(c, k)
                for i, x in enumerate(v):
                    arr[i] = x
            else:
                setattr(c, k, v)
        b = state.c_box()
        self._check(self._lib.grhd_kitp_disk_initial_data(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            C.byref(c), time, _stream()))

    def perturb_density(self, state: LevelBox, amplitude, seed, time=0.0):
        b = state.c_box()
        self._check(self._lib.grhd_perturb_density(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            amplitude, seed, time, _stream()))

    def disk_diagnostics(self, state: LevelBox, time=0.0) -> list:
        """compute_diagnostics of the example drivers
        (Main_GRHDLevelDataKerrSchildDisk.cpp:223-290): [mass, disk_mass,
        tau, max_rho, max_pressure, max_velocity, max_lorentz_factor]."""
        out = (C.c_double * 7)()
        b = state.c_box()
        self._check(self._lib.grhd_disk_diagnostics(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            time, out, _stream()))
        return list(out)

    # ---- the binary-PN disk driver's source terms ----

    def kitp_viscous_rhs(self, rhs: torch.Tensor, state: LevelBox,
                         config=None, time=0.0):
        """add_kitp_viscous_rhs (Examples/GRHDLevelDataBinaryPNKITPDisk/
        Main_GRHDLevelDataBinaryPNKITPDisk.cpp:772-806): rhs -= the
        alpha-viscosity stress divergence in x and y."""
        cfg = config if config is not None else kitp_config()
        b = state.c_box()
        self._check(self._lib.grhd_kitp_viscous_rhs(
            self._ctx, _ptr(rhs), rhs[0].numel(), _ptr(state.state),
            state.comp_stride(), C.byref(b), C.byref(cfg), time, _stream()))

    def kitp_sink_rhs(self, rhs: torch.Tensor, state: LevelBox, config=None,
                      time=0.0):
        """add_kitp_sink_rhs (:567-610)."""
        cfg = config if config is not None else kitp_config()
        b = state.c_box()
        self._check(self._lib.grhd_kitp_sink_rhs(
            self._ctx, _ptr(rhs), rhs[0].numel(), _ptr(state.state),
            state.comp_stride(), C.byref(b), C.byref(cfg), time, _stream()))

    def kitp_advance_ssprk2(self, state: LevelBox, time, dt, config=None,
                            inverse_dx_U=None):
        """advance_kitp_ssprk2 (Main_GRHDLevelDataBinaryPNKITPDisk.cpp:
        842-876), the disk driver's step (grhd_kitp_advance_ssprk2)."""
        cfg = config if config is not None else kitp_config()
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_kitp_advance_ssprk2(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), C.byref(cfg), time, dt, C.byref(d),
            _stream()))
        return d

    def kitp_sink_decay(self, state: LevelBox, time, dt, config=None):
        """apply_kitp_sink_decay (:612-662) with the bodies at `time`."""
        cfg = config if config is not None else kitp_config()
        b = state.c_box()
        self._check(self._lib.grhd_kitp_sink_decay(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            C.byref(cfg), time, dt, _stream()))

    # ---- instrumentation ----

    def profile(self, enable=True):
        self._check(self._lib.grhd_profile_enable(self._ctx, int(enable)))

    def profile_read(self):
        """{class: (ms, launches)} since the last read."""
        ms = (C.c_double * L.NUM_KERNEL_CLASSES)()
        n = (C.c_longlong * L.NUM_KERNEL_CLASSES)()
        self._check(self._lib.grhd_profile_read(self._ctx, ms, n))
        return {name: (ms[i], n[i])
                for i, name in enumerate(L.KERNEL_CLASSES)}

    def accretion(self, reset=False):
        """(Mdot of the last RHS evaluation, its time integral since the
        last reset) through the sphere r < accretion_radius (new)."""
        m, i = C.c_double(), C.c_double()
        self._check(self._lib.grhd_accretion(self._ctx, C.byref(m),
                                             C.byref(i), int(reset)))
        return m.value, i.value

    def launch_count(self) -> int:
        return int(self._lib.grhd_launch_count(self._ctx))

    def advance_rk4(self, state, inverse_dx_U=None, time=0.0, dt=None):
        """New: classic RK4 with post-stage recovery (no reference
        counterpart)."""
        return self._advance(self._lib.grhd_advance_rk4, state, inverse_dx_U,
                             time, dt)

    def advance_rk4_cfl(self, state, cfl, time=0.0, max_dt=0.0,
                        max_inverse_dt=0.0, inverse_dx_U=None):
        """New: one RK4 step with dt = min(cfl / max_inverse_dt, max_dt),
        the driver pattern compute_stable_dt + advance.  Pass the
        max_inverse_dt this method returned for the same unmodified state
        (0 recomputes it).  Returns (dt, next max_inverse_dt, diagnostics)."""
        if not cfl > 0.0:
            raise L.InvalidArgument(L.GRHD_ERR_INVALID_ARG, None)
        mi = C.c_double(max_inverse_dt)
        dt = C.c_double()
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_advance_rk4_cfl(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), time, cfl, max_dt, C.byref(mi),
            C.byref(dt), C.byref(d), _stream()))
        return dt.value, mi.value, d

    def advance_rk4_cfl_steps(self, state, cfl, steps, time=0.0, max_dt=0.0,
                              max_inverse_dt=0.0, inverse_dx_U=None):
        """New: `steps` advance_rk4_cfl steps in one call
        (grhd_advance_rk4_cfl_steps); the per-cell pass of each step's
        first RHS rides on the previous step's last stage.  Returns
        (time reached, next max_inverse_dt, diagnostics of all steps)."""
        if not cfl > 0.0:
            raise L.InvalidArgument(L.GRHD_ERR_INVALID_ARG, None)
        mi = C.c_double(max_inverse_dt)
        tout = C.c_double(time)
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_advance_rk4_cfl_steps(
            self._ctx, _ptr(state.state), state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), time, cfl, max_dt, int(steps),
            C.byref(mi), C.byref(tout), C.byref(d), _stream()))
        return tout.value, mi.value, d

    def advance_rk4_cfl_host(self, host_state, box, cfl, time=0.0,
                             max_dt=0.0, max_inverse_dt=0.0,
                             inverse_dx_U=None):
        """New: advance_rk4_cfl of a state in host memory
        (grhd_advance_rk4_cfl_host): host_state is a CPU float64 tensor of
        the whole-domain LevelBox `box`'s shape (pinned for fast copies),
        updated in place.  Returns (dt, next max_inverse_dt, diagnostics,
        host-to-device bytes, device-to-host bytes)."""
        if not cfl > 0.0:
            raise L.InvalidArgument(L.GRHD_ERR_INVALID_ARG, None)
        if host_state.device.type != "cpu" or \
                host_state.dtype != torch.float64 or \
                not host_state.is_contiguous():
            raise L.InvalidArgument(L.GRHD_ERR_INVALID_ARG, None)
        mi = C.c_double(max_inverse_dt)
        dt = C.c_double()
        d = L.Diagnostics()
        hb, db = C.c_longlong(), C.c_longlong()
        b = box.c_box()
        self._check(self._lib.grhd_advance_rk4_cfl_host(
            self._ctx, C.c_void_p(host_state.data_ptr()),
            host_state[0].numel(), C.byref(b), self._inv(inverse_dx_U),
            time, cfl, max_dt, C.byref(mi), C.byref(dt), C.byref(d),
            C.byref(hb), C.byref(db), _stream()))
        return dt.value, mi.value, d, hb.value, db.value


class FixedBGLevelDataFiniteVolumeOperator(_OperatorBase):
    """FixedBGFArrayBoxFiniteVolume.hpp:446-614 (static background)."""

    def __init__(self, eos, background, dx, center,
                 atmosphere=None, limiter_theta=1.5, use_reconstruction=True,
                 recovery_options=None, use_static_metric_sources=True,
                 excision_radius=0.0, accretion_radius=0.0,
                 precision="fp64"):
        super().__init__(eos, background, dx, center, atmosphere,
                         limiter_theta, use_reconstruction, recovery_options,
                         use_static_metric_sources, False, 1.0e-3,
                         excision_radius, accretion_radius, precision)

    def compute_rhs(self, rhs, state, domain=None, inverse_dx_U=None):
        self._compute_rhs(rhs, state, inverse_dx_U, 0.0)

    def recover_primitives(self, state):
        return self._recover_primitives(state, 0.0)

    def update_conserved(self, state, rhs, dt,
                         recover_primitives_after_update=True):
        return self._update_conserved(state, rhs, dt, 0.0,
                                      recover_primitives_after_update)

    def compute_max_inverse_dt(self, state, domain_box=None,
                               inverse_dx_U=None):
        return self._compute_max_inverse_dt(state, inverse_dx_U, 0.0)

    def compute_stable_dt(self, state, domain_box=None, inverse_dx_U=None,
                          cfl=None):
        return self._compute_stable_dt(state, inverse_dx_U, cfl, 0.0)

    def advance_ssprk2(self, state, domain=None, inverse_dx_U=None, dt=None):
        return self._advance(self._lib.grhd_advance_ssprk2, state,
                             inverse_dx_U, 0.0, dt)


class TimeDependentFixedBGLevelDataFiniteVolumeOperator(_OperatorBase):
    """FixedBGFArrayBoxFiniteVolume.hpp:677-830 (background factory of
    time; the CircularBinaryPN parameters act as the factory)."""

    def __init__(self, eos, background_factory, dx, center,
                 atmosphere=None, limiter_theta=1.5, use_reconstruction=True,
                 recovery_options=None, use_static_metric_sources=True,
                 use_metric_volume_time_sources=True,
                 metric_time_derivative_step=1.0e-3, excision_radius=0.0,
                 accretion_radius=0.0, precision="fp64"):
        super().__init__(eos, background_factory, dx, center, atmosphere,
                         limiter_theta, use_reconstruction, recovery_options,
                         use_static_metric_sources,
                         use_metric_volume_time_sources,
                         metric_time_derivative_step, excision_radius,
                         accretion_radius, precision)

    def compute_rhs(self, rhs, state, domain=None, inverse_dx_U=None,
                    time=0.0):
        self._compute_rhs(rhs, state, inverse_dx_U, time)

    def recover_primitives(self, state, time=0.0):
        return self._recover_primitives(state, time)

    def update_conserved(self, state, rhs, dt, recovery_time=0.0,
                         recover_primitives_after_update=True):
        return self._update_conserved(state, rhs, dt, recovery_time,
                                      recover_primitives_after_update)

    def compute_max_inverse_dt(self, state, domain_box=None,
                               inverse_dx_U=None, time=0.0):
        return self._compute_max_inverse_dt(state, inverse_dx_U, time)

    def compute_stable_dt(self, state, domain_box=None, inverse_dx_U=None,
                          cfl=None, time=0.0):
        return self._compute_stable_dt(state, inverse_dx_U, cfl, time)

    def advance_ssprk2(self, state, domain=None, inverse_dx_U=None, time=0.0,
                       dt=None):
        return self._advance(self._lib.grhd_advance_ssprk2, state,
                             inverse_dx_U, time, dt)


class LevelDataFiniteVolumeOperator:
    """LevelDataFiniteVolumeOperator (FArrayBoxFiniteVolume.hpp:1215-1364):
    the Valencia operator on a metric the grid holds in GRChombo's CCZ4
    variables (grhd_ccz4_*).  States are LevelBoxes of
    ncomp = GRHD_CCZ4_NUM_VARS components (25 CCZ4, then 11 GRHD); FP64."""

    NUM_VARS = 36
    GRHD_OFFSET = 25

    def __init__(self, eos, atmosphere=None, limiter_theta=1.5,
                 use_reconstruction=True, recovery_options=None,
                 use_static_metric_sources=True):
        self._lib = L.load()
        p = L.Params()
        self._lib.grhd_default_params(C.byref(p))
        p.adiabatic_index = eos.adiabatic_index
        p.dx = 1.0  # unused: the spacing comes with inverse_dx_U
        a = atmosphere or AtmosphereOptions()
        p.rho_floor, p.pressure_floor = a.rho_floor, a.pressure_floor
        p.max_velocity_squared = a.max_velocity_squared
        p.metric_source_atmosphere_factor = a.metric_source_atmosphere_factor
        r = recovery_options or RecoveryOptions()
        p.recovery_max_iterations = r.max_iterations
        p.recovery_tolerance = r.tolerance
        p.recovery_pressure_floor = r.pressure_floor
        p.recovery_max_velocity_squared = r.max_velocity_squared
        p.limiter_theta = limiter_theta
        p.use_reconstruction = int(use_reconstruction)
        p.use_static_metric_sources = int(use_static_metric_sources)
        p.use_metric_volume_time_sources = 0
        self.params = p
        self.eos = eos
        ctx = C.c_void_p()
        L.check(self._lib, None, self._lib.grhd_create(C.byref(p),
                                                       C.byref(ctx)))
        self._ctx = ctx

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx:
            self._lib.grhd_destroy(ctx)

    def _check(self, status):
        L.check(self._lib, self._ctx, status)

    @staticmethod
    def _inv(inverse_dx_U):
        if inverse_dx_U is None:
            raise ValueError("inverse_dx_U is required")
        return (C.c_double * 3)(*inverse_dx_U)

    def _state(self, state: LevelBox):
        if state.state.shape[0] != self.NUM_VARS:
            raise ValueError(f"expected a {self.NUM_VARS}-component state")
        return _ptr(state.state)

    def compute_rhs(self, rhs, state: LevelBox, domain=None,
                    inverse_dx_U=None):
        b = state.c_box()
        self._check(self._lib.grhd_ccz4_compute_rhs(
            self._ctx, _ptr(rhs), rhs[0].numel(), self._state(state),
            state.comp_stride(), C.byref(b), self._inv(inverse_dx_U),
            _stream()))

    def recover_primitives(self, state: LevelBox):
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_ccz4_recover_primitives(
            self._ctx, self._state(state), state.comp_stride(), C.byref(b),
            C.byref(d), _stream()))
        return d

    def update_conserved(self, state: LevelBox, rhs, dt,
                         recover_primitives_after_update=True):
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_ccz4_update_conserved(
            self._ctx, self._state(state), state.comp_stride(), _ptr(rhs),
            rhs[0].numel(), C.byref(b), dt,
            int(recover_primitives_after_update), C.byref(d), _stream()))
        return d

    def compute_max_inverse_dt(self, state: LevelBox, domain_box=None,
                               inverse_dx_U=None):
        out = C.c_double()
        b = state.c_box()
        self._check(self._lib.grhd_ccz4_compute_max_inverse_dt(
            self._ctx, self._state(state), state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), C.byref(out), _stream()))
        return out.value

    def compute_stable_dt(self, state: LevelBox, domain_box=None,
                          inverse_dx_U=None, cfl=None):
        if cfl is None or not cfl > 0.0:
            raise L.InvalidArgument(L.GRHD_ERR_INVALID_ARG, None)
        m = self.compute_max_inverse_dt(state, domain_box, inverse_dx_U)
        return cfl / max(m, 1.0e-14)

    def ssprk2_stage(self, stage, state: LevelBox, stage_state: LevelBox,
                     dt, inverse_dx_U=None):
        """One half of advance_ssprk2 for a level whose ghosts the caller
        exchanges before each (grhd_ccz4_ssprk2_stage)."""
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_ccz4_ssprk2_stage(
            self._ctx, int(stage), self._state(state), state.comp_stride(),
            self._state(stage_state), stage_state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), dt, C.byref(d), _stream()))
        return d

    def advance_level_ssprk2(self, boxes, stage_boxes, dt, inverse_dx_U=None):
        """advance_ssprk2 (:1323-1348) of a level of several boxes on this
        device, LevelData::exchange() of all 36 components before each
        RHS."""
        level_exchange(boxes)
        for b, sb in zip(boxes, stage_boxes):
            self.ssprk2_stage(1, b, sb, dt, inverse_dx_U)
        level_exchange(stage_boxes)
        for b, sb in zip(boxes, stage_boxes):
            self.ssprk2_stage(2, b, sb, dt, inverse_dx_U)

    def advance_ssprk2(self, state: LevelBox, domain=None, inverse_dx_U=None,
                       dt=None):
        d = L.Diagnostics()
        b = state.c_box()
        self._check(self._lib.grhd_ccz4_advance_ssprk2(
            self._ctx, self._state(state), state.comp_stride(), C.byref(b),
            self._inv(inverse_dx_U), dt, C.byref(d), _stream()))
        return d
