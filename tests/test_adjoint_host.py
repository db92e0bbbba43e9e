"""The reverse-mode pointwise functions of the discrete adjoint
(grdzhadzha_b200/csrc/grhd_adjoint.cuh) agree with central finite
differences of the forward functions they reverse: p2c, floors,
characteristic speeds, the MUSCL-HLLE face flux (replayed limiter
branches), con2prim by the implicit function theorem and the static-metric
sources, plus the spin derivative of the face geometry and of the sources
through the dual-number metric.  Built as a host program with nvcc and run
on the CPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    return None


def test_reverse_functions_match_finite_differences(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    exe = tmp_path / "adjoint_host_check"
    subprocess.run(
        [nvcc, "-std=c++17", "-O2", "-Xcompiler", "-ffp-contract=off",
         "-Wno-deprecated-gpu-targets",
         "-I", os.path.join(ROOT, "grdzhadzha_b200", "csrc"),
         "-I", os.path.join(ROOT, "include"), "-x", "cu",
         os.path.join(ROOT, "tests", "adjoint_host_check.cu"),
         "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASSED" in r.stdout


def test_rhs_and_step_adjoint_match_oracle_differences(tmp_path):
    """The adjoint's work items (limiter bits, face / shell / cell reverse,
    the taped RK4 stage, the reverse of the recovery) run in host loops give
    the vector-Jacobian products of one RHS evaluation (with its accretion
    rate) and of one RK4 step (with its accretion integral) that central
    differences of the oracle give, at spin 0 and 0.7, with atmosphere
    floors, velocity caps, excision and physical boundaries."""
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")],
                   check=True)
    exe = tmp_path / "adjoint_rhs_check"
    odir = os.path.join(ROOT, "oracle")
    subprocess.run(
        [nvcc, "-std=c++17", "-O2", "-Xcompiler", "-ffp-contract=off",
         "-Wno-deprecated-gpu-targets",
         "-I", os.path.join(ROOT, "grdzhadzha_b200", "csrc"),
         "-I", os.path.join(ROOT, "include"), "-I", odir, "-x", "cu",
         os.path.join(ROOT, "tests", "adjoint_rhs_check.cu"),
         "-o", str(exe), "-L", odir, "-lorc_grhd",
         "-Xlinker", "-rpath=" + odir], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASSED" in r.stdout
