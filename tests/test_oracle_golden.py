"""Pins the CPU oracle against the reference's recorded outputs.

Golden values are the ones the reference's own drivers printed and logged
(GRHD_PROGRESS.md:396-409 Kerr-Schild disk, :378-388 binary-PN disk,
:423-428 LevelData Michel, :180-186 Michel profile); the thresholds are the
reference tests' own where it has them.
"""
import numpy as np
import pytest

import oracle_lib as O


def rel(a, b):
    return abs(a - b) / abs(b)


def test_kerr_schild_disk_golden():
    """Examples/GRHDLevelDataKerrSchildDisk: 56^2 x 9, 40 SSPRK2 steps."""
    tp, init, final, steps = O.run_disk_example(O.BG_KERR_SCHILD)
    assert steps == 40
    assert rel(tp.ell, 3.952846210518592) < 1e-14
    assert rel(tp.surface_potential, -0.038999967542758737) < 1e-14
    assert rel(tp.max_enthalpy, 1.0058220833394507) < 1e-15
    assert rel(tp.polytropic_constant, 3.1607131163777216) < 1e-14
    assert rel(init[1], 0.028799123650408626) < 1e-13
    assert rel(final[1], 0.028801497749415979) < 1e-13
    assert rel(final[3], 1.9556944512350192e-05) < 1e-13
    assert rel(final[4], 4.5283557131844508e-08) < 1e-13
    assert rel(final[5], 0.51157954453700194) < 1e-13
    assert rel(final[6], 1.1638247126610648) < 1e-13


def test_binary_pn_disk_golden():
    """Examples/GRHDLevelDataBinaryPNDisk: time-dependent metric with the
    metric volume-time source, 40 SSPRK2 steps."""
    tp, init, final, steps = O.run_disk_example(O.BG_BINARY_PN)
    assert steps == 40
    assert rel(tp.ell, 4.9353189499884671) < 1e-14
    assert rel(tp.surface_potential, -0.023380221245975233) < 1e-14
    assert rel(tp.max_enthalpy, 1.0014653367693895) < 1e-15
    assert rel(tp.polytropic_constant, 0.79550718821504551) < 1e-14
    assert rel(init[1], 0.019469376019477229) < 1e-13
    assert rel(final[1], 0.019469695978953892) < 1e-13
    assert rel(final[3], 1.9894710361761495e-05) < 1e-13
    assert rel(final[4], 1.162435841077777e-08) < 1e-13
    assert rel(final[5], 0.28737021599042162) < 1e-13


def michel_leveldata_setup():
    n, dx = 18, 2.0
    c = 0.5 * n * dx
    p = O.default_params(
        background=O.BG_KERR_SCHILD, ks_mass=1.0, ks_spin=0.0, gamma=5 / 3,
        dx=dx, center=(c, c, c), atmo_rho_floor=1e-12,
        atmo_pressure_floor=1e-16, atmo_max_velocity_squared=0.8,
        rec_max_iterations=100, rec_pressure_floor=1e-16,
        rec_max_velocity_squared=0.8, limiter_theta=1.2)
    box = O.make_box((n, n, n))
    s = O.new_state(box)
    O.fill_michel(p, O.michel_config(), box, s)
    return p, box, s


def test_michel_leveldata_golden():
    """Tests/GRHDLevelDataMichelAccretion: 18^3, 5 SSPRK2 steps to t=0.1."""
    p, box, s = michel_leveldata_setup()
    d = O.recover_primitives(p, box, s)
    assert d.num_failed_recoveries == 0 and d.num_conserved_resets == 0
    m0 = O.interior(box, s)[0].sum()
    t, steps = 0.0, 0
    while t < 0.1 - 1e-14:
        dt = min(min(O.stable_dt(p, box, s, 0.2), 0.02), 0.1 - t)
        O.advance_ssprk2(p, box, s, t, dt)
        t += dt
        steps += 1
    I = O.interior(box, s, slice(0, 11))
    m1 = I[0].sum()
    assert steps == 5
    assert round(m0, 8) == 0.00172117
    assert round(m1, 8) == 0.00172335
    assert abs((m1 - m0) / m0 - 0.00126778) < 5e-9
    assert abs(I[5].max() - 2.06653e-06) < 5e-12
    assert abs(I[7].max() - 1.75256e-07) < 5e-13


def test_michel_profile():
    """Tests/GRHDMichelAccretion: 512 radii in [4,40]; mass flux, Bernoulli
    and con2prim round trip on the Kerr-Schild metric (thresholds :396-399)."""
    cfg = O.michel_config()
    k = O.michel_constants(cfg)
    assert abs(k[4] - 1.0 / 13.0) < 1e-14
    assert abs(k[3] ** 2 - 1.0 / 16.0) < 1e-14
    p = O.default_params(gamma=5 / 3, rec_max_iterations=200,
                         rec_tolerance=1e-14, rec_pressure_floor=1e-16)
    mf, be, rc = 0.0, 0.0, 0.0
    for i in range(512):
        r = 4.0 + 36.0 * (i + 0.5) / 512
        rho, pres, eps, ur, vr = O.michel_point(p, cfg, r)
        f = 1 - 2 / r
        h = 1 + cfg.gamma * pres / ((cfg.gamma - 1) * rho)
        mf = max(mf, abs(r * r * rho * ur - k[1]) / abs(k[1]))
        be = max(be, abs(h * np.sqrt(f + ur * ur) - k[2]) / abs(k[2]))
        v = O.background_vars(p, r, 0.0, 0.0)
        gLL = v["gamma"]
        gUU = np.linalg.inv(gLL)
        prim = np.array([rho, eps, pres, vr, 0.0, 0.0])
        cons = np.zeros(5)
        O.lib().orc_compute_conserved(O.C.byref(p), O._dp(prim),
                                      O._dp(np.ascontiguousarray(gLL.ravel())),
                                      O._dp(cons))
        out = np.zeros(6)
        it = O.C.c_int()
        res = O.C.c_double()
        ok = O.lib().orc_recover_primitive(
            O.C.byref(p), O._dp(cons),
            O._dp(np.ascontiguousarray(gUU.ravel())), O._dp(out),
            O.C.byref(it), O.C.byref(res))
        assert ok
        rc = max(rc, abs(out[0] - rho) / rho, abs(out[2] - pres) / pres,
                 abs(out[3] - vr) / abs(vr))
    assert mf < 1e-9 and be < 1e-9 and rc < 2e-6


def test_fixed_bg_point_identities():
    """Tests/GRHDFixedBGTest.cpp:569-690: KS M=1 a=0.3, dx=0.25, cell
    (24,15,10): gamma gamma^-1 = delta, nonzero K_ij, p2c -> con2prim."""
    p = O.default_params(ks_mass=1.0, ks_spin=0.3, dx=0.25, gamma=5 / 3)
    x, y, z = [(i + 0.5) * 0.25 for i in (24, 15, 10)]
    v = O.background_vars(p, x, y, z)
    g = v["gamma"]
    gUU = np.linalg.inv(g)
    assert np.abs(g @ gUU - np.eye(3)).max() < 1e-11
    assert np.abs(v["K_tensor"]).max() > 1e-14
    prim = np.array([1.1, 0.2, (5 / 3 - 1) * 1.1 * 0.2, 0.01, -0.015, 0.005])
    cons = np.zeros(5)
    O.lib().orc_compute_conserved(O.C.byref(p), O._dp(prim),
                                  O._dp(np.ascontiguousarray(g.ravel())),
                                  O._dp(cons))
    out = np.zeros(6)
    it, res = O.C.c_int(), O.C.c_double()
    assert O.lib().orc_recover_primitive(
        O.C.byref(p), O._dp(cons), O._dp(np.ascontiguousarray(gUU.ravel())),
        O._dp(out), O.C.byref(it), O.C.byref(res))
    assert np.abs(out - prim).max() < 1e-10


def test_slab_boxes_match_single_box():
    """The multi-box CPU baseline (one z-slab box per thread, as one MPI
    rank per box would) gives the single-box RHS."""
    p, box, s = michel_leveldata_setup()
    O.recover_primitives(p, box, s)
    r1 = O.compute_rhs(p, box, s.copy())
    r2 = O.compute_rhs_slabs(p, box, s.copy(), 4)
    assert np.array_equal(r1, r2)
