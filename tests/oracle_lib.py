"""ctypes binding of the CPU oracle (oracle/liborc_grhd.so).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use this module.  It restates nothing itself; it marshals numpy
arrays into the oracle's C entry points and replays the reference example
drivers' time loops (Examples/GRHDLevelDataKerrSchildDisk/
Main_GRHDLevelDataKerrSchildDisk.cpp:445-571 and Tests/
GRHDLevelDataMichelAccretion/GRHDLevelDataMichelAccretion.cpp:595-632).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_DIR = os.path.join(os.path.dirname(_HERE), "oracle")
_LIB_PATH = os.path.join(_ORACLE_DIR, "liborc_grhd.so")
# the same source built for timing (-O3, FMA contraction allowed)
_FAST_LIB_PATH = os.path.join(_ORACLE_DIR, "liborc_grhd_fast.so")

# GRDzhadzha's own operator (its headers compiled unmodified against
# oracle/shim, oracle/ref_capi.cpp): present where the reference tree was
# available to build it (make -C oracle ref)
REF_DIR = os.path.join(_ORACLE_DIR, "_ref")
_REF_LIB_PATH = os.path.join(REF_DIR, "libref_grhd.so")
_REF_FAST_LIB_PATH = os.path.join(REF_DIR, "libref_grhd_fast.so")

NCOMP = 11
D, S1, S2, S3, TAU, RHO, EPS, PRESS, V1, V2, V3 = range(11)
BG_KERR_SCHILD, BG_BINARY_PN = 0, 1


class Params(C.Structure):
    _fields_ = [
        ("background", C.c_int),
        ("ks_mass", C.c_double), ("ks_spin", C.c_double),
        ("pn_mass_1", C.c_double), ("pn_mass_2", C.c_double),
        ("pn_separation", C.c_double), ("pn_angular_velocity", C.c_double),
        ("pn_phase", C.c_double), ("pn_time", C.c_double),
        ("pn_softening_radius", C.c_double),
        ("gamma", C.c_double), ("dx", C.c_double),
        ("center", C.c_double * 3),
        ("atmo_rho_floor", C.c_double), ("atmo_pressure_floor", C.c_double),
        ("atmo_max_velocity_squared", C.c_double),
        ("atmo_metric_source_atmosphere_factor", C.c_double),
        ("rec_max_iterations", C.c_int),
        ("rec_tolerance", C.c_double), ("rec_pressure_floor", C.c_double),
        ("rec_max_velocity_squared", C.c_double),
        ("limiter_theta", C.c_double),
        ("use_reconstruction", C.c_int), ("use_static_metric_sources", C.c_int),
        ("use_metric_volume_time_sources", C.c_int),
        ("metric_time_derivative_step", C.c_double),
        ("excision_radius", C.c_double),
        ("accretion_radius", C.c_double),
    ]


class Box(C.Structure):
    _fields_ = [
        ("lo", C.c_int * 3), ("hi", C.c_int * 3),
        ("glo", C.c_int * 3), ("ghi", C.c_int * 3),
        ("dlo", C.c_int * 3), ("dhi", C.c_int * 3),
        ("comp_stride", C.c_int64),
    ]


class Diag(C.Structure):
    _fields_ = [("num_cells", C.c_longlong),
                ("num_failed_recoveries", C.c_longlong),
                ("num_floored_primitives", C.c_longlong),
                ("num_conserved_resets", C.c_longlong)]

    def as_tuple(self):
        return (self.num_cells, self.num_failed_recoveries,
                self.num_floored_primitives, self.num_conserved_resets)


class Error(C.Structure):
    _fields_ = [("code", C.c_int), ("where", C.c_int),
                ("cell", C.c_int * 3), ("residual", C.c_double)]


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
        "mass", "gamma", "sonic_radius", "sonic_density",
        "atmosphere_radius", "root_tolerance")]


class KitpDisk(C.Structure):
    _fields_ = [("mach", C.c_double), ("aspect_ratio", C.c_double),
                ("cavity_radius_factor", C.c_double),
                ("cavity_delta", C.c_double),
                ("outer_cutoff_radius", C.c_double),
                ("rho_peak", C.c_double),
                ("mode_amplitude", C.c_double * 4),
                ("mode_phase", C.c_double * 4)]


_lib = None


class KitpConfig(C.Structure):
    """orc_kitp_config: the binary-PN disk driver's source-term settings
    (Main_GRHDLevelDataBinaryPNKITPDisk.cpp SimulationConfig :63, :67-71)."""
    _fields_ = [(n, C.c_double) for n in (
        "alpha_viscosity", "viscosity_beta", "rho_floor", "sink_size",
        "sink_rate", "sink_shape")]


def kitp_config(**kw) -> KitpConfig:
    """The driver's defaults (:63, :67-71), overridden by kw."""
    k = KitpConfig(0.03, 0.0, 1.0e-10, 1.0, 1.0e4, 4.0)
    for name, v in kw.items():
        setattr(k, name, v)
    return k


def kitp_viscous_rhs(p, k, box, state, rhs, time=0.0):
    """rhs (flat, 5 x interior) -= the viscous stress divergence."""
    lib().orc_kitp_viscous_rhs(C.byref(p), C.byref(k), C.byref(box),
                               _dp(state), _dp(rhs), interior_cells(box),
                               time)


def kitp_sink_rhs(p, k, box, state, rhs, time=0.0):
    lib().orc_kitp_sink_rhs(C.byref(p), C.byref(k), C.byref(box), _dp(state),
                            _dp(rhs), interior_cells(box), time)


def kitp_sink_decay(p, k, box, state, time, dt):
    lib().orc_kitp_sink_decay(C.byref(p), C.byref(k), C.byref(box),
                              _dp(state), time, dt)


def build():
    subprocess.run(["make", "-s", "-C", _ORACLE_DIR], check=True)


def lib():
    """The parity build (no FMA contraction): the checker."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = _bind(C.CDLL(_LIB_PATH))
    return _lib


_fast_lib = None


def fast_lib():
    """The timing build of the same source (-O3, AVX2 + FMA): the CPU
    baseline, and the second correct evaluation of the reference's
    algorithm in tests/test_oracle_conditioning.py."""
    global _fast_lib
    if _fast_lib is None:
        if not os.path.exists(_FAST_LIB_PATH):
            build()
        _fast_lib = _bind(C.CDLL(_FAST_LIB_PATH))
    return _fast_lib


_ref_libs = {}


def have_ref() -> bool:
    """Whether the reference's own operator library was built."""
    return os.path.exists(_REF_LIB_PATH)


def ref_lib(fast=False):
    """The reference's own operator behind the oracle's C interface
    (`ref_` entry points): the parity build, or (fast) the -O3 build timed
    as the CPU baseline's reference implementation."""
    path = _REF_FAST_LIB_PATH if fast else _REF_LIB_PATH
    if path not in _ref_libs:
        L = C.CDLL(path)
        P, B = C.POINTER(Params), C.POINTER(Box)
        dp, i64 = C.POINTER(C.c_double), C.c_int64
        E, Dg = C.POINTER(Error), C.POINTER(Diag)
        L.ref_compute_rhs.argtypes = [P, B, dp, dp, i64, dp, C.c_double, E]
        L.ref_recover_primitives.argtypes = [P, B, dp, C.c_double, Dg]
        L.ref_compute_max_inverse_dt.argtypes = [P, B, dp, dp, C.c_double,
                                                 dp, E]
        L.ref_update_conserved.argtypes = [P, B, dp, dp, i64, C.c_double,
                                           C.c_double, C.c_int, Dg]
        L.ref_advance_ssprk2.argtypes = [P, B, dp, dp, C.c_double,
                                         C.c_double, Dg, E]
        L.ref_advance_rk4_cfl_ranks.argtypes = [
            P, B, dp, dp, C.c_double, C.c_double, C.c_double, C.c_int, dp,
            dp, Dg, E]
        L.ref_ccz4_compute_rhs.argtypes = [P, B, dp, dp, i64, dp, E]
        L.ref_ccz4_recover_primitives.argtypes = [P, B, dp, Dg]
        L.ref_ccz4_compute_max_inverse_dt.argtypes = [P, B, dp, dp, dp, E]
        _ref_libs[path] = L
    return _ref_libs[path]


def ref_kitp_lib():
    """The reference KITP disk driver's functions (oracle/ref_kitp.cpp)."""
    path = os.path.join(REF_DIR, "libref_kitp.so")
    if path not in _ref_libs:
        L = C.CDLL(path)
        P, B = C.POINTER(Params), C.POINTER(Box)
        dp, i64 = C.POINTER(C.c_double), C.c_int64
        KC, KD = C.POINTER(KitpConfig), C.POINTER(KitpDisk)
        L.ref_kitp_fill.argtypes = [P, KD, B, dp, C.c_double]
        L.ref_kitp_source_rhs.argtypes = [P, KC, B, dp, dp, i64, C.c_double,
                                          C.c_int]
        L.ref_kitp_sink_decay.argtypes = [P, KC, B, dp, C.c_double,
                                          C.c_double]
        L.ref_kitp_advance_ssprk2.argtypes = [P, KC, B, dp, C.c_double,
                                              C.c_double, C.POINTER(Error)]
        _ref_libs[path] = L
    return _ref_libs[path]


def ref_compute_rhs(p, box, state, time=0.0):
    n = interior_cells(box)
    rhs = np.zeros(5 * n, dtype=np.float64)
    inv = np.array([1.0 / p.dx] * 3)
    err = Error()
    st = ref_lib().ref_compute_rhs(C.byref(p), C.byref(box), _dp(state),
                                   _dp(rhs), n, _dp(inv), time,
                                   C.byref(err))
    if st:
        raise OracleError(st, err)
    return rhs


def ref_recover_primitives(p, box, state, time=0.0) -> Diag:
    d = Diag()
    st = ref_lib().ref_recover_primitives(C.byref(p), C.byref(box),
                                          _dp(state), time, C.byref(d))
    if st:
        raise OracleError(st)
    return d


def ref_max_inverse_dt(p, box, state, time=0.0):
    out = C.c_double()
    inv = np.array([1.0 / p.dx] * 3)
    err = Error()
    st = ref_lib().ref_compute_max_inverse_dt(C.byref(p), C.byref(box),
                                              _dp(state), _dp(inv), time,
                                              C.byref(out), C.byref(err))
    if st:
        raise OracleError(st, err)
    return out.value


def ref_advance_ssprk2(p, box, state, time, dt) -> None:
    d, err = Diag(), Error()
    inv = np.array([1.0 / p.dx] * 3)
    st = ref_lib().ref_advance_ssprk2(C.byref(p), C.byref(box), _dp(state),
                                      _dp(inv), time, dt, C.byref(d),
                                      C.byref(err))
    if st:
        raise OracleError(st, err)


def ref_advance_rk4_cfl(p, box, state, time, cfl, ranks=1, fast=False):
    """(dt, max inverse dt of the input, diag) of one CFL-limited RK4 step
    built from the reference operator's methods, one z slab per thread."""
    d, err = Diag(), Error()
    mi, dt = C.c_double(), C.c_double()
    inv = np.array([1.0 / p.dx] * 3)
    st = ref_lib(fast).ref_advance_rk4_cfl_ranks(
        C.byref(p), C.byref(box), _dp(state), _dp(inv), time, cfl, 0.0,
        ranks, C.byref(mi), C.byref(dt), C.byref(d), C.byref(err))
    if st:
        raise OracleError(st, err)
    return dt.value, mi.value, d


def _bind(L):
    """Declares the argument types of the oracle's entry points on L."""
    P, B = C.POINTER(Params), C.POINTER(Box)
    dp, i64 = C.POINTER(C.c_double), C.c_int64
    L.orc_default_params.argtypes = [P]
    L.orc_background_vars.argtypes = [P, C.c_double, C.c_double,
                                      C.c_double, C.c_double, dp]
    L.orc_compute_conserved.argtypes = [P, dp, dp, dp]
    L.orc_recover_primitive.argtypes = [P, dp, dp, dp,
                                        C.POINTER(C.c_int), dp]
    L.orc_muscl_hlle_flux.argtypes = [P, dp, dp, dp, dp, dp, dp,
                                      C.c_double, dp, C.c_int, dp]
    L.orc_compute_rhs.argtypes = [P, B, dp, dp, i64, dp, C.c_double,
                                  C.POINTER(Error)]
    L.orc_compute_rhs_mdot.argtypes = [P, B, dp, dp, i64, dp,
                                       C.c_double, dp, C.POINTER(Error)]
    L.orc_advance_ssprk2_mdot.argtypes = [P, B, dp, dp, C.c_double,
                                          C.c_double, C.POINTER(Diag),
                                          C.POINTER(Error), dp]
    L.orc_advance_rk4_mdot.argtypes = [P, B, dp, dp, C.c_double,
                                       C.c_double, C.POINTER(Diag),
                                       C.POINTER(Error), dp]
    L.orc_compute_rhs_slabs.argtypes = [P, B, dp, dp, i64, dp,
                                        C.c_double, C.c_int,
                                        C.POINTER(Error)]
    L.orc_recover_primitives.argtypes = [P, B, dp, C.c_double,
                                         C.POINTER(Diag)]
    L.orc_compute_max_inverse_dt.argtypes = [P, B, dp, dp, C.c_double,
                                             dp, C.POINTER(Error)]
    L.orc_compute_stable_dt.argtypes = [P, B, dp, dp, C.c_double,
                                        C.c_double, dp, C.POINTER(Error)]
    L.orc_update_conserved.argtypes = [P, B, dp, dp, i64, C.c_double,
                                       C.c_double, C.c_int,
                                       C.POINTER(Diag)]
    L.orc_advance_ssprk2.argtypes = [P, B, dp, dp, C.c_double,
                                     C.c_double, C.POINTER(Diag),
                                     C.POINTER(Error)]
    L.orc_advance_rk4.argtypes = [P, B, dp, dp, C.c_double, C.c_double,
                                  C.POINTER(Diag), C.POINTER(Error)]
    L.orc_default_torus_config.argtypes = [C.POINTER(TorusConfig)]
    L.orc_make_torus_parameters.argtypes = [P, C.POINTER(TorusConfig), B,
                                            C.c_double,
                                            C.POINTER(TorusParams)]
    L.orc_fill_torus.argtypes = [P, C.POINTER(TorusConfig),
                                 C.POINTER(TorusParams), B, dp,
                                 C.c_double]
    L.orc_michel_constants.argtypes = [C.POINTER(MichelConfig), dp]
    L.orc_michel_point.argtypes = [P, C.POINTER(MichelConfig), C.c_double,
                                   dp]
    L.orc_fill_michel.argtypes = [P, C.POINTER(MichelConfig), B, dp]
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_fill_conserved_from_primitives.argtypes = [P, B, dp,
                                                     C.c_double]
    L.orc_disk_diagnostics.argtypes = [P, B, C.c_int * 3, C.c_int * 3, dp,
                                       C.c_double, dp]
    K = C.POINTER(KitpConfig)
    L.orc_kitp_viscous_rhs.argtypes = [P, K, B, dp, dp, i64, C.c_double]
    L.orc_kitp_sink_rhs.argtypes = [P, K, B, dp, dp, i64, C.c_double]
    L.orc_kitp_sink_decay.argtypes = [P, K, B, dp, C.c_double,
                                      C.c_double]
    L.orc_fill_kitp_disk.argtypes = [P, C.POINTER(KitpDisk), B, dp,
                                     C.c_double]
    L.orc_fill_kitp_disk.restype = None
    L.orc_ccz4_compute_rhs.argtypes = [P, B, dp, dp, i64, dp,
                                       C.POINTER(Error)]
    L.orc_ccz4_recover_primitives.argtypes = [P, B, dp, C.POINTER(Diag)]
    L.orc_ccz4_recover_primitives.restype = None
    L.orc_ccz4_compute_max_inverse_dt.argtypes = [P, B, dp, dp, dp,
                                                  C.POINTER(Error)]
    L.orc_ccz4_fill_from_background.argtypes = [P, B, dp, C.c_double]
    L.orc_ccz4_fill_from_background.restype = None
    return L


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def default_params(**kw) -> Params:
    p = Params()
    lib().orc_default_params(C.byref(p))
    for k, v in kw.items():
        if k == "center":
            for i in range(3):
                p.center[i] = v[i]
        else:
            setattr(p, k, v)
    return p


def make_box(n, ghost=2, lo=(0, 0, 0)) -> Box:
    """A single box covering the whole (non-periodic) domain of n cells."""
    b = Box()
    for d in range(3):
        b.lo[d] = lo[d]
        b.hi[d] = lo[d] + n[d] - 1
        b.glo[d] = b.lo[d] - ghost
        b.ghi[d] = b.hi[d] + ghost
        b.dlo[d] = b.lo[d]
        b.dhi[d] = b.hi[d]
    b.comp_stride = int(np.prod([n[d] + 2 * ghost for d in range(3)]))
    return b


def new_state(box: Box) -> np.ndarray:
    return np.zeros(NCOMP * box.comp_stride, dtype=np.float64)


def interior_cells(box: Box) -> int:
    return int(np.prod([box.hi[d] - box.lo[d] + 1 for d in range(3)]))


def state_view(box: Box, state: np.ndarray) -> np.ndarray:
    """(comp, z, y, x) view over the ghosted box."""
    shape = tuple(box.ghi[d] - box.glo[d] + 1 for d in (2, 1, 0))
    return state.reshape(NCOMP, *shape)


def interior(box: Box, state: np.ndarray, comps=slice(0, 5)) -> np.ndarray:
    v = state_view(box, state)
    g = [box.lo[d] - box.glo[d] for d in range(3)]
    n = [box.hi[d] - box.lo[d] + 1 for d in range(3)]
    return v[comps, g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]


class OracleError(RuntimeError):
    def __init__(self, code, err: Error | None = None):
        self.code = code
        self.err = err
        msg = f"oracle status {code}"
        if err is not None:
            msg += (f" where={err.where} cell=({err.cell[0]},{err.cell[1]},"
                    f"{err.cell[2]}) residual={err.residual}")
        super().__init__(msg)


def compute_rhs(p, box, state, time=0.0, inv_dx=None):
    n = interior_cells(box)
    rhs = np.zeros(5 * n, dtype=np.float64)
    inv = np.array(inv_dx if inv_dx is not None else [1.0 / p.dx] * 3)
    err = Error()
    st = lib().orc_compute_rhs(C.byref(p), C.byref(box), _dp(state), _dp(rhs),
                               n, _dp(inv), time, C.byref(err))
    if st:
        raise OracleError(st, err)
    return rhs


def compute_rhs_mdot(p, box, state, time=0.0):
    """(rhs, Mdot through the voxelised sphere r < p.accretion_radius)."""
    n = interior_cells(box)
    rhs = np.zeros(5 * n, dtype=np.float64)
    inv = np.array([1.0 / p.dx] * 3)
    m = C.c_double()
    err = Error()
    st = lib().orc_compute_rhs_mdot(C.byref(p), C.byref(box), _dp(state),
                                    _dp(rhs), n, _dp(inv), time, C.byref(m),
                                    C.byref(err))
    if st:
        raise OracleError(st, err)
    return rhs, m.value


def advance_mdot(p, box, state, time, dt, method="rk4"):
    """One step; returns (diag, time integral of Mdot over the step)."""
    d, err, m = Diag(), Error(), C.c_double(0.0)
    inv = np.array([1.0 / p.dx] * 3)
    fn = (lib().orc_advance_rk4_mdot if method == "rk4"
          else lib().orc_advance_ssprk2_mdot)
    st = fn(C.byref(p), C.byref(box), _dp(state), _dp(inv), time, dt,
            C.byref(d), C.byref(err), C.byref(m))
    if st:
        raise OracleError(st, err)
    return d, m.value


def compute_rhs_slabs(p, box, state, num_slabs, time=0.0):
    n = interior_cells(box)
    rhs = np.zeros(5 * n, dtype=np.float64)
    inv = np.array([1.0 / p.dx] * 3)
    err = Error()
    st = lib().orc_compute_rhs_slabs(C.byref(p), C.byref(box), _dp(state),
                                     _dp(rhs), n, _dp(inv), time, num_slabs,
                                     C.byref(err))
    if st:
        raise OracleError(st, err)
    return rhs


def recover_primitives(p, box, state, time=0.0) -> Diag:
    d = Diag()
    lib().orc_recover_primitives(C.byref(p), C.byref(box), _dp(state), time,
                                 C.byref(d))
    return d


def max_inverse_dt(p, box, state, time=0.0):
    out = C.c_double()
    inv = np.array([1.0 / p.dx] * 3)
    err = Error()
    st = lib().orc_compute_max_inverse_dt(C.byref(p), C.byref(box),
                                          _dp(state), _dp(inv), time,
                                          C.byref(out), C.byref(err))
    if st:
        raise OracleError(st, err)
    return out.value


def stable_dt(p, box, state, cfl, time=0.0):
    out = C.c_double()
    inv = np.array([1.0 / p.dx] * 3)
    err = Error()
    st = lib().orc_compute_stable_dt(C.byref(p), C.byref(box), _dp(state),
                                     _dp(inv), cfl, time, C.byref(out),
                                     C.byref(err))
    if st:
        raise OracleError(st, err)
    return out.value


def update_conserved(p, box, state, rhs, dt, recovery_time=0.0, recover=True):
    d = Diag()
    lib().orc_update_conserved(C.byref(p), C.byref(box), _dp(state), _dp(rhs),
                               interior_cells(box), dt, recovery_time,
                               int(recover), C.byref(d))
    return d


def advance_ssprk2(p, box, state, time, dt) -> Diag:
    d, err = Diag(), Error()
    inv = np.array([1.0 / p.dx] * 3)
    st = lib().orc_advance_ssprk2(C.byref(p), C.byref(box), _dp(state),
                                  _dp(inv), time, dt, C.byref(d),
                                  C.byref(err))
    if st:
        raise OracleError(st, err)
    return d


def advance_rk4(p, box, state, time, dt, L=None) -> Diag:
    """One RK4 step of the oracle (L: the build, default the checker)."""
    d, err = Diag(), Error()
    inv = np.array([1.0 / p.dx] * 3)
    st = (L or lib()).orc_advance_rk4(C.byref(p), C.byref(box), _dp(state),
                                      _dp(inv), time, dt, C.byref(d),
                                      C.byref(err))
    if st:
        raise OracleError(st, err)
    return d


def background_vars(p, x, y, z, t=0.0) -> dict:
    out = np.zeros(64)
    lib().orc_background_vars(C.byref(p), t, x, y, z, _dp(out))
    return {
        "gamma": out[0:9].reshape(3, 3), "K_tensor": out[9:18].reshape(3, 3),
        "K": out[18], "lapse": out[19], "shift": out[20:23],
        "d1_gamma": out[23:50].reshape(3, 3, 3), "d1_lapse": out[50:53],
        "d1_shift": out[53:62].reshape(3, 3),
    }


def torus_config(**kw) -> TorusConfig:
    c = TorusConfig()
    lib().orc_default_torus_config(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def make_torus(p, cfg, box, time=0.0) -> TorusParams:
    t = TorusParams()
    st = lib().orc_make_torus_parameters(C.byref(p), C.byref(cfg),
                                         C.byref(box), time, C.byref(t))
    if st:
        raise OracleError(st)
    return t


def fill_torus(p, cfg, tp, box, state, time=0.0):
    st = lib().orc_fill_torus(C.byref(p), C.byref(cfg), C.byref(tp),
                              C.byref(box), _dp(state), time)
    if st:
        raise OracleError(st)


def michel_config(**kw) -> MichelConfig:
    c = MichelConfig(mass=1.0, gamma=5.0 / 3.0, sonic_radius=8.0,
                     sonic_density=1.0e-6, atmosphere_radius=4.0,
                     root_tolerance=1.0e-13)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def michel_constants(cfg) -> np.ndarray:
    out = np.zeros(5)
    lib().orc_michel_constants(C.byref(cfg), _dp(out))
    return out


def michel_point(p, cfg, radius) -> np.ndarray:
    out = np.zeros(5)
    st = lib().orc_michel_point(C.byref(p), C.byref(cfg), radius, _dp(out))
    if st:
        raise OracleError(st)
    return out


def fill_michel(p, cfg, box, state):
    st = lib().orc_fill_michel(C.byref(p), C.byref(cfg), C.byref(box),
                               _dp(state))
    if st:
        raise OracleError(st)


def set_threads(n: int):
    """Threads of the oracle's setup passes (initial data, recovery)."""
    lib().orc_set_threads(int(n))


def fill_conserved_from_primitives(p, box, state, time=0.0):
    lib().orc_fill_conserved_from_primitives(C.byref(p), C.byref(box),
                                             _dp(state), time)


def disk_diagnostics(p, box, lo, hi, state, time=0.0) -> np.ndarray:
    out = np.zeros(7)
    lib().orc_disk_diagnostics(C.byref(p), C.byref(box), (C.c_int * 3)(*lo),
                               (C.c_int * 3)(*hi), _dp(state), time, _dp(out))
    return out


def x_split_diagnostics(p, box, state, time=0.0) -> np.ndarray:
    """Diagnostics summed box by box over the reference's two-box x-split
    layout (make_x_split_layout) so the sum order matches its MPI_Allreduce
    of per-rank partial sums."""
    lo = [box.lo[d] for d in range(3)]
    hi = [box.hi[d] for d in range(3)]
    mid = (lo[0] + hi[0]) // 2
    a = disk_diagnostics(p, box, lo, [mid, hi[1], hi[2]], state, time)
    b = disk_diagnostics(p, box, [mid + 1, lo[1], lo[2]], hi, state, time)
    out = a.copy()
    out[:3] = a[:3] + b[:3]
    out[3:] = np.maximum(a[3:], b[3:])
    return out


def run_disk_example(background: int, steps_cap: int | None = None):
    """Replays Examples/GRHDLevelData{KerrSchild,BinaryPN}Disk main(): torus
    initial data, then SSPRK2 with CFL 0.18, max_dt 0.05 and output every 0.5
    to t = 2.  Returns (torus params, initial diag, final diag, steps)."""
    num_cells, num_z = 56, 9
    dx = 80.0 / num_cells
    center = (0.5 * num_cells * dx, 0.5 * num_cells * dx, 0.5 * num_z * dx)
    kw = dict(gamma=5.0 / 3.0, dx=dx, center=center, atmo_rho_floor=1e-10,
              atmo_pressure_floor=1e-12, atmo_max_velocity_squared=0.8,
              rec_max_iterations=80, rec_pressure_floor=1e-12,
              rec_max_velocity_squared=0.8, limiter_theta=1.4,
              metric_time_derivative_step=1e-3)
    if background == BG_KERR_SCHILD:
        p = default_params(background=BG_KERR_SCHILD, ks_mass=1.0, ks_spin=0.0,
                           use_metric_volume_time_sources=0, **kw)
        cfg = torus_config(total_mass=1.0, inner_radius=7.0,
                           pressure_max_radius=10.0, rho_peak=2e-5,
                           max_velocity_squared=0.8)
    else:
        p = default_params(background=BG_BINARY_PN, pn_mass_1=0.5,
                           pn_mass_2=0.5, pn_separation=8.0,
                           pn_angular_velocity=0.0, pn_phase=0.0, pn_time=0.0,
                           pn_softening_radius=1.0,
                           use_metric_volume_time_sources=1, **kw)
        cfg = torus_config(total_mass=1.0, inner_radius=14.0,
                           pressure_max_radius=18.0, rho_peak=2e-5,
                           max_velocity_squared=0.8)
    box = make_box((num_cells, num_cells, num_z))
    state = new_state(box)
    tp = make_torus(p, cfg, box, 0.0)
    time = 0.0
    fill_torus(p, cfg, tp, box, state, time)
    recover_primitives(p, box, state, time)
    init = x_split_diagnostics(p, box, state, time)
    final_time, output_interval, cfl, max_dt = 2.0, 0.5, 0.18, 0.05
    next_out = output_interval
    steps = 0
    while time < final_time - 1e-14:
        recover_primitives(p, box, state, time)
        sdt = stable_dt(p, box, state, cfl, time)
        dt = min(min(sdt, max_dt), final_time - time)
        if time + dt > next_out:
            dt = next_out - time
        if dt <= 1e-14:
            next_out += output_interval
            continue
        advance_ssprk2(p, box, state, time, dt)
        time += dt
        steps += 1
        recover_primitives(p, box, state, time)
        if time >= next_out - 1e-12 or time >= final_time - 1e-14:
            next_out += output_interval
        if steps_cap is not None and steps >= steps_cap:
            break
    final = x_split_diagnostics(p, box, state, time)
    return tp, init, final, steps


# ---- the operator on CCZ4-stored geometry ----
CCZ4_NUM_VARS = 36
CCZ4_GRHD = 25


def ccz4_state(p, box, grhd_state, time=0.0):
    """36-component state: the CCZ4 variables of the fixed background (the
    reference test's store_ccz4_background_vars), then the 11 GRHD
    components of `grhd_state`."""
    cs = box.comp_stride
    s = np.zeros(CCZ4_NUM_VARS * cs, dtype=np.float64)
    lib().orc_ccz4_fill_from_background(C.byref(p), C.byref(box), _dp(s),
                                        time)
    s[CCZ4_GRHD * cs:] = grhd_state
    return s


def ccz4_compute_rhs(p, box, state36):
    n = interior_cells(box)
    rhs = np.zeros(5 * n, dtype=np.float64)
    inv = np.array([1.0 / p.dx] * 3)
    err = Error()
    st = lib().orc_ccz4_compute_rhs(C.byref(p), C.byref(box), _dp(state36),
                                    _dp(rhs), n, _dp(inv), C.byref(err))
    if st:
        raise OracleError(st, err)
    return rhs


def ccz4_recover_primitives(p, box, state36) -> Diag:
    d = Diag()
    lib().orc_ccz4_recover_primitives(C.byref(p), C.byref(box), _dp(state36),
                                      C.byref(d))
    return d


def ccz4_max_inverse_dt(p, box, state36):
    out = C.c_double()
    inv = np.array([1.0 / p.dx] * 3)
    err = Error()
    st = lib().orc_ccz4_compute_max_inverse_dt(
        C.byref(p), C.byref(box), _dp(state36), _dp(inv), C.byref(out),
        C.byref(err))
    if st:
        raise OracleError(st, err)
    return out.value


def kitp_disk(**kw) -> KitpDisk:
    """The disk drivers' SimulationConfig disk defaults (:56-61), no modes,
    with overrides."""
    k = KitpDisk(10.0, 0.1, 2.5, 1e-5, 1e10, 4e-5)
    for name, v in kw.items():
        if name in ("mode_amplitude", "mode_phase"):
            arr = getattr(k, name)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(k, name, v)
    return k


def fill_kitp_disk(p, k, box, state, t=0.0):
    lib().orc_fill_kitp_disk(C.byref(p), C.byref(k), C.byref(box), _dp(state),
                             t)
