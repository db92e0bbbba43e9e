"""ctypes binding of the C ABI in include/grhd_b200.h.

The shared library is built in-tree (grdzhadzha_b200/libgrhd_b200.so, see
grdzhadzha_b200/build.py).  There is no fallback: if the library is missing
or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgrhd_b200.so")

GRHD_OK = 0
GRHD_ERR_RECOVERY = 1
GRHD_ERR_INVALID_ARG = 2
GRHD_ERR_CUDA = 3
GRHD_ERR_SETUP = 4

GRHD_BG_KERR_SCHILD = 0
GRHD_BG_BINARY_PN = 1

GRHD_PRECISION_FP64 = 0
GRHD_PRECISION_MIXED = 1

NUM_STATE_COMPS = 11
NUM_CONSERVED = 5


class Params(C.Structure):
    _fields_ = [
        ("background", C.c_int),
        ("ks_mass", C.c_double), ("ks_spin", C.c_double),
        ("pn_mass_1", C.c_double), ("pn_mass_2", C.c_double),
        ("pn_separation", C.c_double), ("pn_angular_velocity", C.c_double),
        ("pn_phase", C.c_double), ("pn_time", C.c_double),
        ("pn_softening_radius", C.c_double),
        ("adiabatic_index", C.c_double),
        ("dx", C.c_double),
        ("center", C.c_double * 3),
        ("rho_floor", C.c_double), ("pressure_floor", C.c_double),
        ("max_velocity_squared", C.c_double),
        ("metric_source_atmosphere_factor", C.c_double),
        ("recovery_max_iterations", C.c_int),
        ("recovery_tolerance", C.c_double),
        ("recovery_pressure_floor", C.c_double),
        ("recovery_max_velocity_squared", C.c_double),
        ("limiter_theta", C.c_double),
        ("use_reconstruction", C.c_int),
        ("use_static_metric_sources", C.c_int),
        ("use_metric_volume_time_sources", C.c_int),
        ("metric_time_derivative_step", C.c_double),
        ("excision_radius", C.c_double),
        ("accretion_radius", C.c_double),
        ("precision", C.c_int),
    ]


class Box(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3), ("ghost", C.c_int),
                ("domain_lo", C.c_int * 3), ("domain_hi", C.c_int * 3)]


class Diagnostics(C.Structure):
    _fields_ = [("num_cells", C.c_longlong),
                ("num_failed_recoveries", C.c_longlong),
                ("num_floored_primitives", C.c_longlong),
                ("num_conserved_resets", C.c_longlong)]


class TorusConfig(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "total_mass", "inner_radius", "pressure_max_radius", "rho_peak",
        "max_velocity_squared", "radial_derivative_fraction",
        "radial_derivative_min_step", "angular_momentum_min_factor",
        "angular_momentum_max_factor")] + [
        ("angular_momentum_samples", C.c_int),
        ("angular_momentum_bisection_iterations", C.c_int),
        ("angular_momentum_tolerance", C.c_double)]


class TorusParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "ell", "surface_potential", "polytropic_constant", "max_enthalpy")]


class MichelConfig(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "mass", "sonic_radius", "sonic_density", "atmosphere_radius",
        "root_tolerance")]


NUM_KERNEL_CLASSES = 5
KERNEL_CLASSES = ("ghosts", "cells", "faces", "stage", "cfl")


class EnsembleMember(C.Structure):
    _fields_ = [("params", Params), ("box", Box), ("state", C.c_void_p),
                ("state_comp_stride", C.c_int64),
                ("inverse_dx", C.c_double * 3), ("cfl", C.c_double),
                ("max_dt", C.c_double), ("time", C.c_double)]


class EnsembleTuning(C.Structure):
    _fields_ = [("zchunk", C.c_int), ("blocks_per_sm", C.c_int),
                ("ms_per_step", C.c_double)]


class Error(C.Structure):
    _fields_ = [("status", C.c_int), ("where", C.c_int),
                ("cell", C.c_int * 3), ("residual", C.c_double),
                ("message", C.c_char * 256)]


# Every symbol include/grhd_b200.h declares, with its ctypes signature.
_P = C.POINTER
_dp = _P(C.c_double)
_vp = C.c_void_p
class KitpDiskConfig(C.Structure):
    _fields_ = [("mach", C.c_double), ("aspect_ratio", C.c_double),
                ("cavity_radius_factor", C.c_double),
                ("cavity_delta", C.c_double),
                ("outer_cutoff_radius", C.c_double),
                ("rho_peak", C.c_double),
                ("mode_amplitude", C.c_double * 4),
                ("mode_phase", C.c_double * 4)]


class CheckpointHeader(C.Structure):
    """grhd_checkpoint_header (the KITPCHK1 header fields)."""
    _fields_ = [("num_components", C.c_int), ("num_cells", C.c_int),
                ("num_z_cells", C.c_int), ("num_ghosts", C.c_int),
                ("steps", C.c_int), ("frame_index", C.c_int),
                ("time", C.c_double), ("next_output_time", C.c_double),
                ("next_checkpoint_time", C.c_double),
                ("recovery_totals", C.c_longlong * 4),
                ("diagnostics", C.c_double * 7),
                ("diagnostic_counts", C.c_longlong * 3)]


class KitpConfig(C.Structure):
    """grhd_kitp_config: the binary-PN disk driver's source-term settings."""
    _fields_ = [(n, C.c_double) for n in (
        "alpha_viscosity", "viscosity_beta", "rho_floor", "sink_size",
        "sink_rate", "sink_shape")]


class AdjointTorus(C.Structure):
    """grhd_adjoint_torus: the eight differentiable parameters (amplitude,
    entropy, spin, mode_amplitude[5]) and the fixed ones."""
    _fields_ = [("amplitude", C.c_double), ("entropy", C.c_double),
                ("spin", C.c_double), ("mode_amplitude", C.c_double * 5),
                ("mode_phase", C.c_double * 5),
                ("inner_radius", C.c_double),
                ("pressure_max_radius", C.c_double),
                ("max_velocity_squared", C.c_double)]


SIGNATURES = {
    "grhd_abi_version": (C.c_int, []),
    "grhd_default_params": (None, [_P(Params)]),
    "grhd_create": (C.c_int, [_P(Params), _P(C.c_void_p)]),
    "grhd_destroy": (None, [_vp]),
    "grhd_last_error": (C.c_int, [_vp, _P(Error)]),
    "grhd_status_string": (C.c_char_p, [C.c_int]),
    "grhd_compute_rhs": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_int64,
                                   _P(Box), _dp, C.c_double, _vp]),
    "grhd_compute_rhs_static": (C.c_int, [_vp, _vp, C.c_int64, _vp,
                                          C.c_int64, _P(Box), _dp,
                                          C.c_double, _vp]),
    "grhd_static_scratch_fill": (C.c_int, [_vp, C.c_double, _vp]),
    "grhd_recover_primitives": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                          C.c_double, _P(Diagnostics), _vp]),
    "grhd_update_conserved": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_int64,
                                        _P(Box), C.c_double, C.c_double,
                                        C.c_int, _P(Diagnostics), _vp]),
    "grhd_compute_max_inverse_dt": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                              _dp, C.c_double, _dp, _vp]),
    "grhd_compute_stable_dt": (C.c_int, [_vp, _vp, C.c_int64, _P(Box), _dp,
                                         C.c_double, C.c_double, _dp, _vp]),
    "grhd_advance_ssprk2": (C.c_int, [_vp, _vp, C.c_int64, _P(Box), _dp,
                                      C.c_double, C.c_double,
                                      _P(Diagnostics), _vp]),
    "grhd_advance_rk4_cfl_steps": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                             _dp, C.c_double, C.c_double,
                                             C.c_double, C.c_int, _dp, _dp,
                                             _P(Diagnostics), _vp]),
    "grhd_advance_rk4_cfl_host": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                            _dp, C.c_double, C.c_double,
                                            C.c_double, _dp, _dp,
                                            _P(Diagnostics),
                                            _P(C.c_longlong),
                                            _P(C.c_longlong), _vp]),
    "grhd_ssprk2_stage": (C.c_int, [_vp, C.c_int, _vp, C.c_int64, _vp,
                                    C.c_int64, _P(Box), _dp, C.c_double,
                                    C.c_double, _P(Diagnostics), _vp]),
    "grhd_advance_rk4": (C.c_int, [_vp, _vp, C.c_int64, _P(Box), _dp,
                                   C.c_double, C.c_double, _P(Diagnostics),
                                   _vp]),
    "grhd_advance_rk4_cfl": (C.c_int, [_vp, _vp, C.c_int64, _P(Box), _dp,
                                       C.c_double, C.c_double, C.c_double,
                                       _dp, _dp, _P(Diagnostics), _vp]),
    "grhd_eval_background": (C.c_int, [_vp, C.c_int64, _vp, C.c_double, _vp,
                                       _vp]),
    "grhd_eval_con2prim": (C.c_int, [_vp, C.c_int64, _vp, _vp, _vp, _vp, _vp,
                                     _vp, _vp]),
    "grhd_eval_arith": (C.c_int, [_vp, C.c_int64, _vp, _vp, _vp, _vp]),
    "grhd_face_zchunk": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.c_int)]),
    "grhd_default_torus_config": (None, [_P(TorusConfig)]),
    "grhd_torus_initial_data": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                          _P(TorusConfig), C.c_double,
                                          _P(TorusParams), _vp]),
    "grhd_michel_initial_data": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                           _P(MichelConfig), _vp]),
    "grhd_perturb_density": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                       C.c_double, C.c_uint64, C.c_double,
                                       _vp]),
    "grhd_profile_enable": (C.c_int, [_vp, C.c_int]),
    "grhd_profile_read": (C.c_int, [_vp, _P(C.c_double), _P(C.c_longlong)]),
    "grhd_launch_count": (C.c_longlong, [_vp]),
    "grhd_accretion": (C.c_int, [_vp, _dp, _dp, C.c_int]),
    "grhd_ensemble_create": (C.c_int, [_P(EnsembleMember), C.c_int,
                                       _P(_vp)]),
    "grhd_ensemble_destroy": (None, [_vp]),
    "grhd_ensemble_last_error": (C.c_int, [_vp, _P(Error)]),
    "grhd_ensemble_get_tuning": (C.c_int, [_vp, _P(EnsembleTuning),
                                           _P(C.c_int)]),
    "grhd_ensemble_set_tuning": (C.c_int, [_vp, _P(EnsembleTuning)]),
    "grhd_ensemble_autotune": (C.c_int, [_vp, C.c_int, _P(EnsembleTuning),
                                         _vp]),
    "grhd_ensemble_advance": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "grhd_ensemble_member_info": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp,
                                            _dp, _P(Diagnostics)]),
    "grhd_ensemble_reset_accretion": (C.c_int, [_vp]),
    "grhd_ensemble_invalidate": (C.c_int, [_vp]),
    "grhd_ensemble_set_barrier_test": (C.c_int, [_vp, C.c_uint,
                                                 C.c_double]),
    "grhd_ensemble_launch_count": (C.c_longlong, [_vp]),
    "grhd_disk_diagnostics": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                        C.c_double, _dp, _vp]),
    "grhd_level_exchange": (C.c_int, [_P(Box), _P(C.c_void_p),
                                      _P(C.c_int64), C.c_int, C.c_char_p,
                                      C.c_int, _vp]),
    "grhd_ccz4_compute_rhs": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_int64,
                                        _P(Box), _dp, _vp]),
    "grhd_ccz4_recover_primitives": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                               _P(Diagnostics), _vp]),
    "grhd_ccz4_update_conserved": (C.c_int, [_vp, _vp, C.c_int64, _vp,
                                             C.c_int64, _P(Box), C.c_double,
                                             C.c_int, _P(Diagnostics), _vp]),
    "grhd_ccz4_compute_max_inverse_dt": (C.c_int, [_vp, _vp, C.c_int64,
                                                   _P(Box), _dp, _dp, _vp]),
    "grhd_ccz4_ssprk2_stage": (C.c_int, [_vp, C.c_int, _vp, C.c_int64, _vp,
                                         C.c_int64, _P(Box), _dp, C.c_double,
                                         _P(Diagnostics), _vp]),
    "grhd_ccz4_advance_ssprk2": (C.c_int, [_vp, _vp, C.c_int64, _P(Box), _dp,
                                           C.c_double, _P(Diagnostics), _vp]),
    "grhd_default_kitp_disk_config": (None, [_P(KitpDiskConfig)]),
    "grhd_kitp_advance_ssprk2": (C.c_int, [_vp, _vp, C.c_int64, _P(Box), _dp,
                                           _P(KitpConfig), C.c_double,
                                           C.c_double, _P(Diagnostics), _vp]),
    "grhd_kitp_disk_initial_data": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                              _P(KitpDiskConfig), C.c_double,
                                              _vp]),
    "grhd_region_copy": (C.c_int, [C.c_int, _vp, C.c_int64, _P(Box),
                                   _P(C.c_int), _P(C.c_int), _vp, _vp]),
    "grhd_region_copy_components": (C.c_int, [C.c_int, _vp, C.c_int64,
                                              _P(Box), _P(C.c_int),
                                              _P(C.c_int), C.c_int, _vp,
                                              _vp]),
    "grhd_level_exchange_components": (C.c_int, [_P(Box), _P(C.c_void_p),
                                                 _P(C.c_int64), C.c_int,
                                                 C.c_int, C.c_char_p, C.c_int,
                                                 _vp]),
    "grhd_checkpoint_write": (C.c_int, [C.c_char_p, _P(CheckpointHeader),
                                        C.c_char_p, _vp, C.c_int64, _P(Box),
                                        C.c_char_p, C.c_int, _vp]),
    "grhd_checkpoint_read": (C.c_int, [C.c_char_p, _P(CheckpointHeader),
                                       C.c_char_p, _vp, C.c_int64, _P(Box),
                                       C.c_char_p, C.c_int, _vp]),
    "grhd_default_kitp_config": (None, [_P(KitpConfig)]),
    "grhd_kitp_viscous_rhs": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_int64,
                                        _P(Box), _P(KitpConfig), C.c_double,
                                        _vp]),
    "grhd_kitp_sink_rhs": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_int64,
                                     _P(Box), _P(KitpConfig), C.c_double,
                                     _vp]),
    "grhd_kitp_sink_decay": (C.c_int, [_vp, _vp, C.c_int64, _P(Box),
                                       _P(KitpConfig), C.c_double, C.c_double,
                                       _vp]),
    "grhd_default_adjoint_torus": (None, [_P(AdjointTorus)]),
    "grhd_adjoint_unit_entropy": (C.c_int, [_P(Params), _P(AdjointTorus),
                                            _dp]),
    "grhd_adjoint_create": (C.c_int, [_P(Params), _P(Box), C.c_int, C.c_int,
                                      C.c_double, _P(_vp)]),
    "grhd_adjoint_destroy": (None, [_vp]),
    "grhd_adjoint_last_error": (C.c_int, [_vp, _P(Error)]),
    "grhd_adjoint_launch_count": (C.c_longlong, [_vp]),
    "grhd_adjoint_initial_data": (C.c_int, [_vp, _P(AdjointTorus), _vp,
                                            C.c_int64, _vp, C.c_int64, _vp]),
    "grhd_adjoint_forward": (C.c_int, [_vp, _P(AdjointTorus), _dp, _vp]),
    "grhd_adjoint_backward": (C.c_int, [_vp, _dp, _vp, C.c_int64, _vp]),
    "grhd_adjoint_tangent": (C.c_int, [_vp, _P(AdjointTorus), _dp, _dp, _dp,
                                       _vp]),
    "grhd_adjoint_rhs_vjp": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_int64,
                                       C.c_double, _vp, C.c_int64, _dp,
                                       _vp]),
    "grhd_adjoint_step_vjp": (C.c_int, [_vp, _vp, C.c_int64, _vp, C.c_int64,
                                        C.c_double, _vp, C.c_int64, _dp,
                                        _vp]),
}

_lib = None


class GRHDError(RuntimeError):
    """Raised for a non-OK status; mirrors the reference's exceptions."""

    def __init__(self, status: int, error: Error | None = None):
        self.status = status
        self.where = error.where if error is not None else 0
        self.cell = tuple(error.cell) if error is not None else (0, 0, 0)
        self.residual = error.residual if error is not None else 0.0
        msg = error.message.decode() if error is not None else ""
        super().__init__(msg or f"grhd status {status}")


class InvalidArgument(GRHDError, ValueError):
    """std::invalid_argument in the reference (cfl <= 0, dx <= 0)."""


def load():
    """Loads libgrhd_b200.so; raises if it is missing or incomplete."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.grhd_abi_version() != 1:
        raise RuntimeError("libgrhd_b200.so ABI version mismatch")
    _lib = lib
    return lib


def check(lib, ctx, status: int, last_error=None):
    if status == GRHD_OK:
        return
    err = Error()
    if ctx:
        (last_error or lib.grhd_last_error)(ctx, C.byref(err))
    if status == GRHD_ERR_INVALID_ARG:
        raise InvalidArgument(status, err)
    raise GRHDError(status, err)
