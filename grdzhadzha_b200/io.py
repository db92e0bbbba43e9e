"""On-disk formats of the reference's example drivers.

* KITPCHK1 checkpoints (Examples/GRHDLevelDataBinaryPNKITPDisk/
  Main_GRHDLevelDataBinaryPNKITPDisk.cpp:1191-1590) written from and read
  into a device LevelBox through grhd_checkpoint_write / _read, so that a
  GPU run restarts from a reference run's checkpoint and the other way
  round;
* the driver's configuration signature (config_signature, :1203-1223)
  that a checkpoint must match;
* the diagnostics CSV row (append_diagnostics,
  Main_GRHDLevelDataKerrSchildDisk.cpp:330-341).
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from .operator import LevelBox, _ptr, _stream

# The KITP driver's SimulationConfig fields in config_signature's order
# (:1205-1222) with their defaults (:36-71).
SIGNATURE_FIELDS = (
    ("num_cells", 192), ("num_z_cells", 25), ("num_ghosts", 2),
    ("domain_length", 96.0), ("output_interval", 0.5), ("cfl", 0.14),
    ("max_dt", 0.02), ("mass_1", 0.5), ("mass_2", 0.5),
    ("separation", 8.0), ("binary_phase", 0.0), ("binary_time", 0.0),
    ("binary_angular_velocity", 0.0), ("softening_radius", 0.5),
    ("metric_time_derivative_step", 1.0e-3), ("mach", 10.0),
    ("aspect_ratio", 0.1), ("cavity_radius_factor", 2.5),
    ("cavity_delta", 1.0e-5), ("outer_cutoff_radius", 1.0e10),
    ("rho_peak", 4.0e-5), ("rho_floor", 1.0e-10),
    ("pressure_floor", 8.0e-14), ("max_velocity_squared", 0.72),
    ("limiter_theta", 1.3), ("use_reconstruction", True),
    ("use_static_metric_sources", True),
    ("use_metric_volume_time_sources", True), ("alpha_viscosity", 0.03),
    ("viscosity_beta", 0.0), ("sink_size", 1.0), ("sink_rate", 1.0e4),
    ("sink_shape", 4.0))


def _fmt(v) -> str:
    """A value as std::ostream with setprecision(17) prints it."""
    if isinstance(v, bool):
        return "1" if v else "0"
    if isinstance(v, int):
        return str(v)
    s = format(float(v), ".17g")
    if "e" in s:
        mant, exp = s.split("e")
        sign = exp[0] if exp[0] in "+-" else "+"
        digits = exp.lstrip("+-")
        s = f"{mant}e{sign}{digits.zfill(2)}"
    return s


def config_signature(**config) -> str:
    """config_signature (:1203-1223) of a driver configuration (defaults
    for fields not given)."""
    values = dict(SIGNATURE_FIELDS)
    for k, v in config.items():
        if k not in values:
            raise KeyError(k)
        values[k] = v
    return " ".join(_fmt(values[k]) for k, _ in SIGNATURE_FIELDS)


def diagnostics_row(step: int, time: float, diagnostics, counts) -> str:
    """append_diagnostics (Main_GRHDLevelDataKerrSchildDisk.cpp:330-341):
    step, time, mass, disk_mass, tau, max_rho, max_pressure, max_velocity,
    max_lorentz_factor, failed_recoveries, floored_primitives,
    conserved_resets."""
    fields = [str(int(step)), _fmt(float(time))]
    fields += [_fmt(float(x)) for x in diagnostics]
    fields += [str(int(c)) for c in counts]
    return ",".join(fields) + "\n"


class CheckpointError(RuntimeError):
    """The reference's std::runtime_error of a checkpoint read/write."""


def write_checkpoint(path: str, level: LevelBox, header: L.CheckpointHeader,
                     signature: str):
    lib = L.load()
    err = C.create_string_buffer(256)
    b = level.c_box()
    st = lib.grhd_checkpoint_write(path.encode(), C.byref(header),
                                   signature.encode(), _ptr(level.state),
                                   level.comp_stride(), C.byref(b), err, 256,
                                   _stream())
    if st != L.GRHD_OK:
        raise CheckpointError(err.value.decode())


def read_checkpoint(path: str, level: LevelBox | None = None,
                    expected_signature: str | None = None
                    ) -> L.CheckpointHeader:
    """The header; with `level`, the GRHD state into it."""
    lib = L.load()
    err = C.create_string_buffer(256)
    h = L.CheckpointHeader()
    b = level.c_box() if level is not None else None
    st = lib.grhd_checkpoint_read(
        path.encode(), C.byref(h),
        expected_signature.encode() if expected_signature else None,
        _ptr(level.state) if level is not None else None,
        level.comp_stride() if level is not None else 0,
        C.byref(b) if b is not None else None, err, 256, _stream())
    if st != L.GRHD_OK:
        raise CheckpointError(err.value.decode())
    return h
