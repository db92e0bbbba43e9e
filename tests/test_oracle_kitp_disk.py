"""The oracle's restatement of the binary disk drivers' Keplerian disk
(kitp_primitive, Examples/GRHDLevelDataBinaryPNKITPDisk/
Main_GRHDLevelDataBinaryPNKITPDisk.cpp:398-520), checked against the
physics its formulas encode (the reference records no outputs of this
fill, so the restatement is not pinned to reference numbers):

* far outside the binary the gas orbits at the Keplerian rate reduced by
  the pressure support, Omega = sqrt(M / r^3 (1 - 1/Mach^2)) (:429-442);
* the disk is a vertical Gaussian of scale height H = (H/R) r (:478-482);
* the sound speed follows the binary's potential, c_s^2 = -Phi / Mach^2,
  and p = rho c_s^2 / Gamma (:487-494);
* the cavity inside cavity_radius_factor x separation is emptied to
  cavity_delta of the peak (:408-418);
* an m = 1 mode of amplitude A modulates the midplane density by
  1 + A cos(phi + phase) (the benchmark's binary-disk modes, new).
"""
import math

import numpy as np

import oracle_lib as O


def _setup(n=48, L=60.0, **disk):
    dx = 2 * L / n
    c = 0.5 * n * dx
    p = O.default_params(background=O.BG_BINARY_PN, pn_mass_1=0.5,
                         pn_mass_2=0.5, pn_separation=10.0,
                         pn_softening_radius=0.5, gamma=5 / 3, dx=dx,
                         center=(c, c, c), atmo_rho_floor=1e-10,
                         atmo_pressure_floor=8e-14,
                         atmo_max_velocity_squared=0.72)
    box = O.make_box((n, n, n))
    s = O.new_state(box)
    k = O.kitp_disk(mach=10.0, aspect_ratio=0.1, cavity_radius_factor=2.0,
                    outer_cutoff_radius=50.0, **disk)
    O.fill_kitp_disk(p, k, box, s)
    V = O.state_view(box, s)
    g = 2
    idx = np.arange(-g, n + g)
    pos = (idx + 0.5) * dx - c
    return p, k, V, pos


def test_disk_is_keplerian_with_pressure_support():
    p, k, V, pos = _setup()
    z0 = np.argmin(np.abs(pos))
    for r_want in (30.0, 40.0):
        i = np.argmin(np.abs(pos - r_want))
        x, y = pos[i], pos[z0]
        r = math.hypot(x, y)
        # v^y at (x, ~0): the orbital speed (lapse and shift are ~1 and ~0
        # there at the 1e-2 level; compare the ratio of two radii instead)
        vy = V[O.V2, z0, z0, i]
        omega = math.sqrt(1.0 / r ** 3 * (1 - 1 / 100.0))
        assert abs(vy / (omega * r) - 1.0) < 0.05, (r, vy, omega * r)
    i1, i2 = np.argmin(np.abs(pos - 30.0)), np.argmin(np.abs(pos - 45.0))
    r1, r2 = pos[i1], pos[i2]
    ratio = V[O.V2, z0, z0, i1] / V[O.V2, z0, z0, i2]
    assert abs(ratio / math.sqrt(r2 / r1) - 1.0) < 1e-2


def test_disk_vertical_profile_and_sound_speed():
    p, k, V, pos = _setup(n=96)
    j = np.argmin(np.abs(pos))
    i = np.argmin(np.abs(pos - 35.0))
    r = math.hypot(pos[i], pos[j])
    H = 0.1 * r
    zs = [np.argmin(np.abs(pos - z)) for z in (pos[j], H)]
    rho0 = V[O.RHO, zs[0], j, i]
    z1 = pos[zs[1]]
    rho1 = V[O.RHO, zs[1], j, i]
    want = math.exp(-0.5 * (z1 / H) ** 2) / math.exp(-0.5 * (pos[zs[0]] / H) ** 2)
    assert abs(rho1 / rho0 - want) < 1e-3 * want + 1e-6
    cs2 = V[O.PRESS, zs[0], j, i] * p.gamma / rho0
    z = pos[zs[0]]
    pot = -0.5 / math.sqrt((pos[i] - 5.0) ** 2 + pos[j] ** 2 + z * z + 0.25) \
        - 0.5 / math.sqrt((pos[i] + 5.0) ** 2 + pos[j] ** 2 + z * z + 0.25)
    assert abs(cs2 / (-pot / 100.0) - 1.0) < 1e-12


def test_cavity_and_mode():
    p, k, V, pos = _setup()
    j = np.argmin(np.abs(pos))
    inner = [np.argmin(np.abs(pos - r)) for r in (6.0,)]
    for i in inner:
        assert V[O.RHO, j, j, i] < 1e-5 * 4e-5 + 1e-9
    amp, ph = 1e-3, 0.7
    _, _, Vm, _ = _setup(mode_amplitude=[amp, 0, 0, 0],
                         mode_phase=[ph, 0, 0, 0])
    i = np.argmin(np.abs(pos - 35.0))
    for (a, b) in ((i, j), (j, i)):
        x, y = pos[a], pos[b]
        phi = math.atan2(y, x)
        rel = Vm[O.RHO, j, b, a] / V[O.RHO, j, b, a] - 1.0
        assert abs(rel - amp * math.cos(phi + ph)) < 1e-6, (rel, phi)
