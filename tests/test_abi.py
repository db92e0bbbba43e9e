"""The C-ABI library loads without a GPU and exports every symbol that
include/grhd_b200.h declares (no compute calls)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "grhd_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(grhd_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = header_functions()
    for required in ("grhd_create", "grhd_destroy", "grhd_compute_rhs",
                     "grhd_recover_primitives", "grhd_update_conserved",
                     "grhd_compute_max_inverse_dt", "grhd_compute_stable_dt",
                     "grhd_advance_ssprk2", "grhd_advance_rk4"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from grdzhadzha_b200 import _lib as L
    if not os.path.exists(L.LIB_PATH):
        pytest.fail(f"{L.LIB_PATH} not built")
    lib = C.CDLL(L.LIB_PATH)
    for name in header_functions():
        assert hasattr(lib, name), name
        assert name in L.SIGNATURES, f"{name} has no ctypes signature"


def test_params_layout_matches_header_defaults():
    """grhd_default_params fills the reference defaults through the ABI
    (pure host code, no device needed)."""
    from grdzhadzha_b200 import _lib as L
    lib = L.load()
    p = L.Params()
    lib.grhd_default_params(C.byref(p))
    assert p.adiabatic_index == pytest.approx(5.0 / 3.0)
    assert p.recovery_max_iterations == 50
    assert p.recovery_tolerance == 1e-12
    assert p.limiter_theta == 1.5
    assert p.metric_time_derivative_step == 1e-3
    assert p.excision_radius == 0.0
    assert lib.grhd_status_string(1) == b"primitive recovery failed"
