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
  failed recovery, the CCZ4-geometry operator) on the parity fixtures and
  on stressed states (torus cells drained until their recovery fails; the
  atmosphere of the torus and of the binary-PN disk dipped under its
  floors; torus cells sped up past the atmosphere's velocity cap);
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


def _torus_floors():
    """The a = 0.9 torus with a seeded twentieth of its cells (ghosts
    included) drained towards vacuum: all five conserved variables scaled
    by one factor in 1e-6..1e-2 (the ideal-gas recovery is homogeneous of
    degree one, so the velocity is kept and density and pressure fall).
    Where the pressure would fall below the recovery floor the recovery
    fails: the RHS and the CFL bound raise the reference's error (its first
    failing cell), and the post-update recovery resets 114 cells to the
    atmosphere."""
    p, box, s, t = cases.CASES["torus_a09"]()
    v = O.state_view(box, s)
    rng = np.random.default_rng(20261204)
    mask = rng.random(v.shape[1:]) < 0.05
    k = 10.0 ** rng.uniform(-6.0, -2.0, v.shape[1:])
    for c in range(5):
        v[c] = np.where(mask, v[c] * k, v[c])
    return p, box, s, t


def _atmosphere_dip(name):
    """A parity fixture with every atmosphere cell (rho at most twice the
    density floor) scaled by 0.99 in all five conserved variables: their
    recovery converges at the pressure floor and the floors raise rho
    back, so the floored-primitive resets run (the a = 0.9 torus: 2304
    interior cells; the binary-PN disk, with its volume-time source:
    27084) while the RHS, CFL bound and SSPRK2 step go through."""
    p, box, s, t = cases.CASES[name]()
    v = O.state_view(box, s)
    atm = v[O.RHO] <= 2.0 * p.atmo_rho_floor
    for c in range(5):
        v[c] = np.where(atm, v[c] * 0.99, v[c])
    return p, box, s, t


def _torus_fast():
    """The a = 0.9 torus with the recovery's velocity cap at 0.9 and a
    seeded fifth of its torus cells (rho > 1e-6) sped up to v^2 in
    0.81..0.88 (v scaled, conserved variables rebuilt from the primitives;
    v^2 = 1 - (rho / D)^2), above the atmosphere cap 0.8: the floors
    rescale their velocities (6021 floored resets) and the face states
    around them, and the RHS, CFL bound and SSPRK2 step go through."""
    p, box, s, t = cases.CASES["torus_a09"]()
    p.rec_max_velocity_squared = 0.9
    v = O.state_view(box, s)
    rng = np.random.default_rng(7)
    v2 = 1.0 - (v[O.RHO] / v[O.D]) ** 2
    sel = (v[O.RHO] > 1e-6) & (v2 > 1e-4) & (rng.random(v.shape[1:]) < 0.2)
    target = rng.uniform(0.81, 0.88, v.shape[1:])
    f = np.sqrt(np.where(sel, target / np.maximum(v2, 1e-300), 1.0))
    for c in (O.V1, O.V2, O.V3):
        v[c] = v[c] * f
    O.fill_conserved_from_primitives(p, box, s, t)
    return p, box, s, t


def _cases():
    """The parity fixtures; the reference has no excision, so the cases
    that use it run here without it (their cells stay clear of the
    singularities: the centre lies between cell centres)."""
    named = [(name, cases.CASES[name]) for name in
             ("fixedbg", "ksdisk", "pndisk", "michel18", "torus_a09",
              "michel_c1")]
    for name, make in named + [("torus_floors", _torus_floors),
                               ("torus_atmosphere_dip",
                                lambda: _atmosphere_dip("torus_a09")),
                               ("pndisk_atmosphere_dip",
                                lambda: _atmosphere_dip("pndisk")),
                               ("torus_fast", _torus_fast)]:
        p, box, s, t = make()
        p.excision_radius = 0.0
        p.accretion_radius = 0.0
        yield name, p, box, s, t


def _both(run_oracle, run_reference):
    """Both results, or None once both raised the same error record (the
    failing cell, where-code and residual)."""
    try:
        a = run_oracle()
    except O.OracleError as e_o:
        with pytest.raises(O.OracleError) as e_r:
            run_reference()
        x, y = e_o.err, e_r.value.err
        assert (x.where, list(x.cell), x.residual) == \
            (y.where, list(y.cell), y.residual)
        return None
    return a, run_reference()


@pytest.mark.parametrize("name,p,box,s,t", list(_cases()),
                         ids=lambda v: v if isinstance(v, str) else "")
def test_restatement_equals_reference_bit_for_bit(name, p, box, s, t):
    # compute_rhs, with the physical ghost fill it writes into the state
    s_o, s_r = s.copy(), s.copy()
    r = _both(lambda: O.compute_rhs(p, box, s_o, t),
              lambda: O.ref_compute_rhs(p, box, s_r, t))
    if r is not None:
        assert np.array_equal(r[0], r[1]), np.abs(r[0] - r[1]).max()
        assert np.array_equal(s_o, s_r, equal_nan=True)
    # recover_primitives and its counters (failures reset to the
    # atmosphere: it does not raise)
    s_o, s_r = s.copy(), s.copy()
    d_o = O.recover_primitives(p, box, s_o, t)
    d_r = O.ref_recover_primitives(p, box, s_r, t)
    assert np.array_equal(s_o, s_r, equal_nan=True)
    assert (d_o.num_cells, d_o.num_failed_recoveries,
            d_o.num_floored_primitives, d_o.num_conserved_resets) == \
        (d_r.num_cells, d_r.num_failed_recoveries,
         d_r.num_floored_primitives, d_r.num_conserved_resets)
    # compute_max_inverse_dt
    m = _both(lambda: O.max_inverse_dt(p, box, s.copy(), t),
              lambda: O.ref_max_inverse_dt(p, box, s.copy(), t))
    if m is None:
        return
    assert m[0] == m[1]
    # advance_ssprk2 with the CFL 0.25 step
    s_o, s_r = s.copy(), s.copy()
    r = _both(lambda: O.advance_ssprk2(p, box, s_o, t, 0.25 / m[0]),
              lambda: O.ref_advance_ssprk2(p, box, s_r, t, 0.25 / m[0]))
    if r is not None:
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


@pytest.mark.parametrize("name", ["ksdisk", "ksdisk_atmosphere_dip",
                                  "torus_fast"])
def test_ccz4_operator_equals_reference_bit_for_bit(name):
    """LevelDataFiniteVolumeOperator (FArrayBoxFiniteVolume.hpp:1215-1364)
    on a state with the CCZ4 variables of its background: the Kerr-Schild
    disk, the same with its atmosphere dipped under the floors, and the
    torus with cells past the atmosphere's velocity cap."""
    make = {"ksdisk": cases.CASES["ksdisk"],
            "ksdisk_atmosphere_dip": lambda: _atmosphere_dip("ksdisk"),
            "torus_fast": _torus_fast}[name]
    p, box, s, t = make()
    p.excision_radius = 0.0
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
    d_o = O.ccz4_recover_primitives(p, box, a)
    d = O.Diag()
    L.ref_ccz4_recover_primitives(O.C.byref(p), O.C.byref(box), O._dp(b),
                                  O.C.byref(d))
    assert np.array_equal(a, b, equal_nan=True)
    counts = (d.num_cells, d.num_failed_recoveries,
              d.num_floored_primitives, d.num_conserved_resets)
    assert counts == (d_o.num_cells, d_o.num_failed_recoveries,
                      d_o.num_floored_primitives, d_o.num_conserved_resets)
    print(name, "recovery counts", counts)
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


# ---- the KITP disk driver (Examples/GRHDLevelDataBinaryPNKITPDisk) ----

KITP_DRIVER = "GRHDLevelDataBinaryPNKITPDisk"
KITP_N, KITP_NZ, KITP_L = 24, 8, 36.0


def kitp_driver_params():
    """The driver's operator on its 24^2 x 8 grid over 36 M
    (make_center, make_background_params, make_atmosphere_options,
    make_recovery_options, :298-346; IdealGasEOS 5/3, :1686)."""
    dx = KITP_L / KITP_N
    return O.default_params(
        background=O.BG_BINARY_PN, pn_mass_1=0.5, pn_mass_2=0.5,
        pn_separation=8.0, pn_softening_radius=0.5, gamma=5 / 3, dx=dx,
        center=(0.5 * KITP_N * dx, 0.5 * KITP_N * dx, 0.5 * KITP_NZ * dx),
        atmo_rho_floor=1e-10, atmo_pressure_floor=8e-14,
        atmo_max_velocity_squared=0.72, rec_max_velocity_squared=0.75,
        rec_max_iterations=80, rec_pressure_floor=8e-14, limiter_theta=1.3,
        use_metric_volume_time_sources=1)


def kitp_driver_disk():
    return O.kitp_disk(mach=10.0, aspect_ratio=0.1, cavity_radius_factor=2.5,
                       cavity_delta=1e-5, outer_cutoff_radius=1e10,
                       rho_peak=4e-5)


def run_kitp_driver(out_dir):
    """The reference driver to t = 0.06 with checkpoints every 0.02 (three
    steps of dt = 0.02, checkpoints after steps 1 and 2)."""
    rc, out = _run(KITP_DRIVER, "0.06", "--num-cells", str(KITP_N),
                   "--num-z-cells", str(KITP_NZ), "--domain-length",
                   str(KITP_L), "--no-frames", "--output-dir", str(out_dir),
                   "--checkpoint-interval", "0.02", cwd=out_dir)
    assert rc == 0, out
    return [os.path.join(out_dir, "checkpoints",
                         f"checkpoint_step_{n:08d}.bin") for n in (1, 2)]


def test_kitp_pieces_equal_reference_driver():
    """kitp_primitive's disk fill (:398-565), the alpha-viscosity RHS
    (:676-806), the sink RHS (:567-610, sinks 20 M wide so that they reach
    the disk) and the sink decay (:612-662): the oracle's restatements
    equal the driver's own functions bit for bit."""
    C = O.C
    L = O.ref_kitp_lib()
    p = kitp_driver_params()
    box = O.make_box((KITP_N, KITP_N, KITP_NZ))
    disk = kitp_driver_disk()
    k = O.kitp_config(sink_size=20.0, sink_rate=1.0, viscosity_beta=0.2)
    n = O.interior_cells(box)
    for t in (0.0, 0.37):
        a, b = O.new_state(box), O.new_state(box)
        O.fill_kitp_disk(p, disk, box, a, t)
        assert L.ref_kitp_fill(C.byref(p), C.byref(disk), C.byref(box),
                               O._dp(b), t) == 0
        assert np.array_equal(O.interior(box, a, slice(0, 11)),
                              O.interior(box, b, slice(0, 11)))
        O.recover_primitives(p, box, a, t)
        for which, fn in ((0, O.kitp_viscous_rhs), (1, O.kitp_sink_rhs)):
            r_o, r_r = np.zeros(5 * n), np.zeros(5 * n)
            fn(p, k, box, a, r_o, t)
            L.ref_kitp_source_rhs(C.byref(p), C.byref(k), C.byref(box),
                                  O._dp(a.copy()), O._dp(r_r), n, t, which)
            assert np.abs(r_r).max() > 0
            assert np.array_equal(r_o, r_r), (which, np.abs(r_o - r_r).max())
        s_o, s_r = a.copy(), a.copy()
        O.kitp_sink_decay(p, k, box, s_o, t, 0.01)
        L.ref_kitp_sink_decay(C.byref(p), C.byref(k), C.byref(box),
                              O._dp(s_r), t, 0.01)
        assert np.array_equal(O.interior(box, s_o, slice(0, 11)),
                              O.interior(box, s_r, slice(0, 11)))


def kitp_oracle_step(p, k, box, s, t, dt):
    """advance_kitp_ssprk2 (:842-876) from the oracle's pieces."""
    old, stage = s.copy(), s.copy()
    r0 = O.compute_rhs(p, box, s, t)
    O.kitp_viscous_rhs(p, k, box, s, r0, t)
    O.update_conserved(p, box, stage, r0, dt, t + dt, True)
    r1 = O.compute_rhs(p, box, stage, t + dt)
    O.kitp_viscous_rhs(p, k, box, stage, r1, t + dt)
    cur = O.interior(box, s)
    cur[...] = 0.5 * (O.interior(box, old) + O.interior(box, stage)
                      + dt * r1.reshape(cur.shape))
    O.kitp_sink_decay(p, k, box, s, t + 0.5 * dt, dt)
    O.recover_primitives(p, box, s, t + dt)


def test_kitp_driver_run_equals_oracle_replay(tmp_path):
    """The driver's run (:1735-1905: initial fill and recovery; per step a
    recovery, the stable dt, advance_kitp_ssprk2, a recovery) replayed by
    the oracle: the GRHD components of both checkpoints equal it bit for
    bit, and the product's config_signature is the driver's."""
    import kitp_checkpoint as KC
    from grdzhadzha_b200 import io
    paths = run_kitp_driver(tmp_path)
    p = kitp_driver_params()
    k = O.kitp_config()
    box = O.make_box((KITP_N, KITP_N, KITP_NZ))
    s = O.new_state(box)
    O.fill_kitp_disk(p, kitp_driver_disk(), box, s, 0.0)
    O.recover_primitives(p, box, s, 0.0)
    t, next_ckpt = 0.0, 0.02
    for n, path in enumerate(paths, start=1):
        O.recover_primitives(p, box, s, t)
        stable = 0.14 / max(O.max_inverse_dt(p, box, s, t), 1e-14)
        dt = min(stable, 0.02, 0.06 - t, 0.5 - t, next_ckpt - t)
        kitp_oracle_step(p, k, box, s, t, dt)
        t += dt
        next_ckpt += 0.02
        O.recover_primitives(p, box, s, t)
        h, sig, v = KC.read(path)
        assert (h["steps"], h["time"]) == (n, t)
        want = np.moveaxis(v[2:-2, 2:-2, 2:-2, 25:36], -1, 0)
        assert np.array_equal(O.interior(box, s, slice(0, 11)), want), n
        assert sig == io.config_signature(
            num_cells=KITP_N, num_z_cells=KITP_NZ, domain_length=KITP_L)
