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


# C struct of the header -> its ctypes mirror in grdzhadzha_b200._lib
STRUCTS = {
    "grhd_params": "Params", "grhd_box": "Box",
    "grhd_diagnostics": "Diagnostics", "grhd_error": "Error",
    "grhd_torus_config": "TorusConfig", "grhd_torus_params": "TorusParams",
    "grhd_michel_config": "MichelConfig", "grhd_kitp_config": "KitpConfig",
    "grhd_kitp_disk_config": "KitpDiskConfig",
    "grhd_checkpoint_header": "CheckpointHeader",
    "grhd_ensemble_member": "EnsembleMember",
    "grhd_ensemble_tuning": "EnsembleTuning",
    "grhd_adjoint_torus": "AdjointTorus",
}


def test_header_is_plain_c_and_ctypes_layouts_match(tmp_path):
    """The header compiles as C99 and as C++, and every struct the ABI
    passes has the same size and field offsets in C as in its ctypes
    mirror (a mismatch would pass garbage across the boundary)."""
    import shutil
    import subprocess
    from grdzhadzha_b200 import _lib as L
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    inc = os.path.join(ROOT, "include")
    lines = ['#include <stdio.h>', '#include <stddef.h>',
             '#include "grhd_b200.h"', 'int main(void) {']
    for cname, pyname in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in getattr(L, pyname)._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", '
                         f'offsetof({cname}, {fname}));')
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-I", inc,
                    str(src), "-o", str(exe)], check=True)
    gxx = shutil.which("g++")
    if gxx is not None:
        cpp = tmp_path / "layout.cpp"
        cpp.write_text('#include "grhd_b200.h"\nint main() { return 0; }\n')
        subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall",
                        "-Werror", "-I", inc, str(cpp)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True,
                         text=True).stdout.split("\n")
    for line in filter(None, out):
        cname, what, value = line.split()
        cls = getattr(L, STRUCTS[cname])
        if what == "size":
            assert C.sizeof(cls) == int(value), cname
        else:
            assert getattr(cls, what).offset == int(value), (cname, what)


def test_cxx_dropin_compiles_and_links(tmp_path):
    """tests/cxx_dropin.cpp -- the C++ drop-in operator class a maintainer
    writes over the header -- compiles warning-free with g++ and links
    against the built library (run on a GPU by
    tests/test_gpu_cxx_dropin.py)."""
    import shutil
    import cases
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    from grdzhadzha_b200 import _lib as L
    if not os.path.exists(L.LIB_PATH):
        pytest.fail(f"{L.LIB_PATH} not built")
    assert os.path.exists(cases.build_cxx_dropin(tmp_path))
