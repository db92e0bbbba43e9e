"""The C ABI from compiled C++: tests/cxx_dropin.cpp holds the drop-in
class for FixedBGLevelDataFiniteVolumeOperator (Source/Matter/GRHD/
FixedBGFArrayBoxFiniteVolume.hpp:446-614) with the reference's method
names and exception types; this test builds it with g++ against
include/grhd_b200.h and libgrhd_b200.so, runs compute_rhs,
compute_stable_dt and advance_ssprk2 on a reference test fixture and
checks them against the oracle: RHS <= 1e-12 of each component's scale
(as the Python parity tests), the stable dt to 1e-13, one SSPRK2 step's
change of the conserved state <= 1e-11 of its scale and its recovery
counts exactly; and that cfl = 0
throws std::invalid_argument, as the reference's compute_stable_dt does
(:549-550)."""
import os
import subprocess

import numpy as np
import pytest

import cases
import oracle_lib as O

pytestmark = pytest.mark.gpu

_NAMES = {"gamma": "adiabatic_index", "atmo_rho_floor": "rho_floor",
          "atmo_pressure_floor": "pressure_floor",
          "atmo_max_velocity_squared": "max_velocity_squared",
          "atmo_metric_source_atmosphere_factor":
              "metric_source_atmosphere_factor",
          "rec_max_iterations": "recovery_max_iterations",
          "rec_tolerance": "recovery_tolerance",
          "rec_pressure_floor": "recovery_pressure_floor",
          "rec_max_velocity_squared": "recovery_max_velocity_squared"}


@pytest.mark.parametrize("name", ["fixedbg", "ksdisk"])
def test_cxx_dropin_matches_oracle(name, tmp_path):
    p, box, s, t = cases.CASES[name]()
    assert p.background == O.BG_KERR_SCHILD and p.excision_radius <= 0.0
    exe = cases.build_cxx_dropin(tmp_path)
    dt = 0.5 * O.stable_dt(p, box, s.copy(), 0.25, t)
    lines = []
    for field, _ in O.Params._fields_:
        v = getattr(p, field)
        v = " ".join(repr(float(x)) for x in v) if field == "center" \
            else repr(float(v))
        lines.append(f"{_NAMES.get(field, field)} {v}")
    lines += [f"lo {box.lo[0]} {box.lo[1]} {box.lo[2]}",
              f"hi {box.hi[0]} {box.hi[1]} {box.hi[2]}",
              f"ghost {box.lo[0] - box.glo[0]}",
              f"domain_lo {box.dlo[0]} {box.dlo[1]} {box.dlo[2]}",
              f"domain_hi {box.dhi[0]} {box.dhi[1]} {box.dhi[2]}",
              f"dt {dt!r}", "cfl 0.25"]
    (tmp_path / "params.txt").write_text("\n".join(lines) + "\n")
    s.tofile(str(tmp_path / "state.bin"))
    out = subprocess.run([exe, str(tmp_path / "params.txt"),
                          str(tmp_path / "state.bin"), str(tmp_path)],
                         capture_output=True, text=True, timeout=300)
    print(out.stdout, out.stderr)
    assert out.returncode == 0, out.stderr
    assert "invalid_argument ok" in out.stdout

    rhs = np.fromfile(str(tmp_path / "rhs.bin")).reshape(5, -1)
    ref = O.compute_rhs(p, box, s.copy(), t).reshape(5, -1)
    err = cases.rel_err(rhs, ref)
    assert np.all(err <= 1e-12), err

    got_dt = float((tmp_path / "stable_dt.txt").read_text())
    want_dt = O.stable_dt(p, box, s.copy(), 0.25, t)
    assert abs(got_dt - want_dt) <= 1e-13 * want_dt, (got_dt, want_dt)

    after = np.fromfile(str(tmp_path / "ssprk2.bin"))
    ref_state = s.copy()
    diag = O.advance_ssprk2(p, box, ref_state, t, dt)
    line = [x for x in out.stdout.splitlines()
            if x.startswith("ssprk2_diag")][0]
    assert [int(x) for x in line.split()[1:]] == [
        diag.num_cells, diag.num_failed_recoveries,
        diag.num_floored_primitives, diag.num_conserved_resets], line
    start = O.interior(box, s)
    err = cases.rel_err(O.interior(box, after) - start,
                        O.interior(box, ref_state) - start)
    assert np.all(err <= 1e-11), err
    assert os.path.getsize(tmp_path / "ssprk2.bin") == s.nbytes
