"""The oracle pinned to GRDzhadzha itself.

oracle/_ref holds the reference's own code: its GRHD headers and its test
and example drivers compiled unmodified against oracle/shim (the Chombo and
GRChombo names they use, one process), by `make -C oracle ref` where the
reference tree is available.  These tests check

* the shim: the reference's own test mains pass, and its LevelData drivers
  reproduce the diagnostics its progress log records
  (GRHD_PROGRESS.md:396-409, :423-428; the recorded runs used two MPI
  ranks, so sums over the boxes may differ in the last digits);
* the restatement: oracle/grhd_oracle.c equals the reference operator bit
  for bit (compute_rhs with its ghost fill, recover_primitives with its
  counters, compute_max_inverse_dt, advance_ssprk2, the error record of a
  failed recovery, the CCZ4-geometry operator) on the parity fixtures;
* the reference RK4 the CPU baseline times (built from the operator's
  compute_rhs and update_conserved, one z slab per thread with the slab
  ghosts exchanged): independent of the slab count bit for bit, and equal
  to the oracle's RK4 up to the order of its stage sums.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import cases
import oracle_lib as O

pytestmark = pytest.mark.skipif(
    not O.have_ref(), reason="reference build absent (make -C oracle ref)")


def _run(name, *args, cwd=None, timeout=600):
    exe = os.path.join(O.REF_DIR, name)
    r = subprocess.run([exe, *args], cwd=cwd, capture_output=True,
                       text=True, timeout=timeout)
    return r.returncode, r.stdout + r.stderr


@pytest.mark.parametrize("name", ["GRHDFixedBGTest", "GRHDBinaryPNTest",
                                  "GRHDMichelAccretion",
                                  "GRHDFixedBGAMRHookTest"])
def test_reference_own_tests_pass(name, tmp_path):
    rc, out = _run(name, cwd=tmp_path)
    print(out)
    assert rc == 0 and "passed" in out, out


def _value(out, label):
    m = re.search(re.escape(label) + r"\s*([-+0-9.eE]+)", out)
    assert m, (label, out)
    return float(m.group(1))


def test_reference_leveldata_michel_reproduces_its_record(tmp_path):
    """Tests/GRHDLevelDataMichelAccretion as recorded at
    GRHD_PROGRESS.md:423-428 (printed to 6 digits)."""
    rc, out = _run("GRHDLevelDataMichelAccretion", cwd=tmp_path)
    print(out)
    assert rc == 0 and "passed" in out
    want = {"initial mass:": 0.00172117, "final mass:": 0.00172335,
            "relative mass change:": 0.00126778, "max rho:": 2.06653e-06,
            "max pressure:": 1.75256e-07, "max speed squared:": 0.0357728}
    for label, v in want.items():
        assert _value(out, label) == pytest.approx(v, rel=6e-6), label


def _summary(path):
    out = {}
    for line in open(path):
        parts = line.split()
        if len(parts) == 2:
            try:
                out[parts[0]] = float(parts[1])
            except ValueError:
                pass
    return out


def test_reference_leveldata_disks_reproduce_their_record():
    """The two LevelData disk drivers (56^2 x 9 cells, two boxes, 40 SSPRK2
    steps to t = 2) against the 17-digit diagnostics of
    GRHD_PROGRESS.md:378-388 (binary PN) and :396-409 (Kerr-Schild).
    The torus construction matches to the last digit; the evolved masses
    and maxima to 2e-13 (measured: masses 7e-16 / 2.5e-15, maxima 2e-16 ..
    9.8e-14 for the maximum pressure: the recorded runs were another
    compilation, summing over two MPI ranks)."""
    runs = {}
    with tempfile.TemporaryDirectory() as tmp:
        procs = {}
        for name in ("GRHDLevelDataKerrSchildDisk",
                     "GRHDLevelDataBinaryPNDisk"):
            d = os.path.join(tmp, name)
            os.makedirs(d)
            procs[name] = subprocess.Popen(
                [os.path.join(O.REF_DIR, name)], cwd=d,
                stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        for name, pr in procs.items():
            out, _ = pr.communicate(timeout=900)
            assert pr.returncode == 0 and "passed" in out, out
            d = os.path.join(tmp, name, "output")
            summ = [f for f in os.listdir(d) if f.endswith("_summary.txt")]
            runs[name] = _summary(os.path.join(d, summ[0]))
    ks = runs["GRHDLevelDataKerrSchildDisk"]
    for key, v in {"torus_specific_angular_momentum": 3.952846210518592,
                   "torus_surface_potential": -0.038999967542758737,
                   "torus_max_enthalpy": 1.0058220833394507,
                   "torus_polytropic_constant": 3.1607131163777216}.items():
        assert ks[key] == v, key
    for key, v in {"initial_disk_mass": 0.028799123650408626,
                   "final_disk_mass": 0.028801497749415979,
                   "max_rho": 1.9556944512350192e-05,
                   "max_pressure": 4.5283557131844508e-08,
                   "max_velocity": 0.51157954453700194,
                   "max_lorentz_factor": 1.1638247126610648}.items():
        assert ks[key] == pytest.approx(v, rel=2e-13, abs=0), key
    pn = runs["GRHDLevelDataBinaryPNDisk"]
    for key, v in {"initial_disk_mass": 0.019469376019477229,
                   "final_disk_mass": 0.019469695978953892,
                   "max_rho": 1.9894710361761495e-05,
                   "max_pressure": 1.162435841077777e-08,
                   "max_velocity": 0.28737021599042162}.items():
        assert pn[key] == pytest.approx(v, rel=2e-13, abs=0), key
    assert ks["conserved_resets"] == 0 and pn["conserved_resets"] == 0


def _cases():
    """The parity fixtures; the reference has no excision, so the two cases
    that use it run here without it (their cells stay clear of the
    singularities: the centre lies between cell centres)."""
    for name in ("fixedbg", "ksdisk", "pndisk", "michel18", "torus_a09",
                 "michel_c1"):
        p, box, s, t = cases.CASES[name]()
        p.excision_radius = 0.0
        p.accretion_radius = 0.0
        yield name, p, box, s, t


@pytest.mark.parametrize("name,p,box,s,t", list(_cases()),
                         ids=lambda v: v if isinstance(v, str) else "")
def test_restatement_equals_reference_bit_for_bit(name, p, box, s, t):
    # compute_rhs, with the physical ghost fill it writes into the state
    s_o, s_r = s.copy(), s.copy()
    try:
        r_o = O.compute_rhs(p, box, s_o, t)
    except O.OracleError as e_o:
        with pytest.raises(O.OracleError) as e_r:
            O.ref_compute_rhs(p, box, s_r, t)
        a, b = e_o.err, e_r.value.err
        assert (a.where, list(a.cell), a.residual) == \
            (b.where, list(b.cell), b.residual)
        return
    r_r = O.ref_compute_rhs(p, box, s_r, t)
    assert np.array_equal(r_o, r_r), np.abs(r_o - r_r).max()
    assert np.array_equal(s_o, s_r, equal_nan=True)
    # recover_primitives and its counters
    s_o, s_r = s.copy(), s.copy()
    d_o = O.recover_primitives(p, box, s_o, t)
    d_r = O.ref_recover_primitives(p, box, s_r, t)
    assert np.array_equal(s_o, s_r, equal_nan=True)
    assert (d_o.num_cells, d_o.num_failed_recoveries,
            d_o.num_floored_primitives, d_o.num_conserved_resets) == \
        (d_r.num_cells, d_r.num_failed_recoveries,
         d_r.num_floored_primitives, d_r.num_conserved_resets)
    # compute_max_inverse_dt
    mi = O.max_inverse_dt(p, box, s.copy(), t)
    assert mi == O.ref_max_inverse_dt(p, box, s.copy(), t)
    # advance_ssprk2 with the CFL 0.25 step
    s_o, s_r = s.copy(), s.copy()
    O.advance_ssprk2(p, box, s_o, t, 0.25 / mi)
    O.ref_advance_ssprk2(p, box, s_r, t, 0.25 / mi)
    for c in (slice(0, 5), slice(5, 11)):
        assert np.array_equal(O.interior(box, s_o, c),
                              O.interior(box, s_r, c))


def test_recovery_failure_record_equals_reference():
    """A cell with D < 0 inside the box: the same exception (where, cell,
    residual) from both."""
    p, box, s, t = cases.CASES["fixedbg"]()
    V = O.state_view(box, s)
    g = [box.lo[d] - box.glo[d] for d in range(3)]
    V[O.D, g[2] + 1, g[1] + 2, g[0] + 1] = -1.0
    with pytest.raises(O.OracleError) as e_o:
        O.compute_rhs(p, box, s.copy(), t)
    with pytest.raises(O.OracleError) as e_r:
        O.ref_compute_rhs(p, box, s.copy(), t)
    a, b = e_o.value.err, e_r.value.err
    print("oracle", a.where, list(a.cell), a.residual, "reference", b.where,
          list(b.cell), b.residual)
    assert (a.where, list(a.cell), a.residual) == \
        (b.where, list(b.cell), b.residual)


def test_ccz4_operator_equals_reference_bit_for_bit():
    """LevelDataFiniteVolumeOperator (FArrayBoxFiniteVolume.hpp:1215-1364)
    on the Kerr-Schild disk's state with the CCZ4 variables of its
    background."""
    p, box, s, t = cases.CASES["ksdisk"]()
    s36 = O.ccz4_state(p, box, s)
    a, b = s36.copy(), s36.copy()
    r_o = O.ccz4_compute_rhs(p, box, a)
    n = O.interior_cells(box)
    r_r = np.zeros(5 * n)
    err = O.Error()
    inv = np.array([1.0 / p.dx] * 3)
    L = O.ref_lib()
    st = L.ref_ccz4_compute_rhs(O.C.byref(p), O.C.byref(box), O._dp(b),
                                O._dp(r_r), n, O._dp(inv), O.C.byref(err))
    assert st == 0
    assert np.array_equal(r_o, r_r), np.abs(r_o - r_r).max()
    a, b = s36.copy(), s36.copy()
    O.ccz4_recover_primitives(p, box, a)
    d = O.Diag()
    L.ref_ccz4_recover_primitives(O.C.byref(p), O.C.byref(box), O._dp(b),
                                  O.C.byref(d))
    assert np.array_equal(a, b, equal_nan=True)
    out = O.C.c_double()
    L.ref_ccz4_compute_max_inverse_dt(O.C.byref(p), O.C.byref(box),
                                      O._dp(s36.copy()), O._dp(inv),
                                      O.C.byref(out), O.C.byref(err))
    assert out.value == O.ccz4_max_inverse_dt(p, box, s36.copy())


def test_reference_rk4_ranks_and_oracle_rk4():
    """The CPU baseline's reference step: 1, 2, 3 and 4 slab threads give
    the same state bit for bit (each slab's stencil sees the exchanged
    ghosts; slabs are at least the ghost layer thick, since the reference
    fills a ghost outside the domain from its own box's edge plane);
    against the oracle's RK4 (stage sums in another order) the conserved
    state agrees to 1e-14 of its scale."""
    p, box, s, t = cases.CASES["ksdisk"]()
    outs = []
    for ranks in (1, 2, 3, 4):
        a = s.copy()
        dt, mi, d = O.ref_advance_rk4_cfl(p, box, a, t, 0.25, ranks=ranks)
        outs.append(a)
    assert mi == O.max_inverse_dt(p, box, s.copy(), t)
    for a in outs[1:]:
        assert np.array_equal(O.interior(box, a, slice(0, 11)),
                              O.interior(box, outs[0], slice(0, 11)))
    with pytest.raises(O.OracleError):
        O.ref_advance_rk4_cfl(p, box, s.copy(), t, 0.25, ranks=5)
    b = s.copy()
    O.advance_rk4(p, box, b, t, dt)
    err = cases.rel_err(O.interior(box, outs[0]).reshape(5, -1),
                        O.interior(box, b).reshape(5, -1))
    print("reference RK4 vs oracle RK4:", err)
    assert np.all(err <= 1e-14), err
