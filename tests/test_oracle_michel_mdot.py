"""The rest-mass accretion rate pinned to the analytic Michel flux.

For steady Michel inflow onto a Schwarzschild hole (Kerr-Schild, a = 0)
the rest-mass flux through every sphere is the same: 4 pi r^2 rho u^r =
4 pi mass_flux with mass_flux = r_s^2 rho_s u_s, u_s = -sqrt(M / (2 r_s))
(Tests/GRHDMichelAccretion/GRHDMichelAccretion.cpp:109-132), so the
accretion rate Mdot = -(outward flux) = -4 pi mass_flux > 0, whatever the
radius R.  The diagnostic sums sqrt(gamma) F_D dA over the faces of the
voxelised sphere r < R (F_D the MUSCL-HLLE face flux of D = rho W, so
sqrt(gamma) F_D = sqrt(-g) rho u^i); on the analytic state its error is the
scheme's truncation error and falls at second order with dx, and its
spread over R with it.  Measured (oracle, one RHS of the noise-free state,
Gamma = 4/3, r_s = 8, rho_s = 1e-6, on [-16, 16]^3):

  R     n = 32     n = 64     n = 128
  4    -1.7e-2    -3.9e-3    -1.0e-3
  6    -7.0e-3    -1.7e-3    -4.3e-4
  8    -9.7e-3    -1.9e-3    +2.6e-4
  12   -3.2e-3    -8.9e-4    -2.4e-4

This test runs n = 32 and 64 on the oracle; tests/test_gpu_michel_mdot.py
runs the GPU path from 32^3 to 256^3."""
import os

import numpy as np

import cases
import oracle_lib as O

RADII = (4.0, 6.0, 8.0, 12.0)


def michel_exact(mass=1.0, sonic_radius=8.0, sonic_density=1e-6):
    """-4 pi r_s^2 rho_s u_s with u_s = -sqrt(M / (2 r_s))."""
    u_s = -np.sqrt(mass / (2.0 * sonic_radius))
    return -4.0 * np.pi * sonic_radius ** 2 * sonic_density * u_s


def michel_params(n, L=16.0):
    dx = 2.0 * L / n
    c = 0.5 * n * dx
    return O.default_params(background=O.BG_KERR_SCHILD, ks_mass=1.0,
                            ks_spin=0.0, gamma=4 / 3, dx=dx,
                            center=(c, c, c), atmo_rho_floor=1e-12,
                            atmo_pressure_floor=1e-16,
                            atmo_max_velocity_squared=0.8,
                            rec_max_iterations=100, rec_pressure_floor=1e-16,
                            rec_max_velocity_squared=0.9, limiter_theta=2.0,
                            excision_radius=1.5)


def test_oracle_michel_constants_are_the_reference_formula():
    cfg = O.michel_config(gamma=4 / 3, sonic_radius=8.0,
                          atmosphere_radius=2.5)
    k = O.michel_constants(cfg)
    assert k[3] == -np.sqrt(1.0 / 16.0)                 # sonic u^r
    assert abs(-4 * np.pi * k[1] - michel_exact()) <= 1e-15 * michel_exact()


def test_oracle_mdot_converges_to_the_michel_flux():
    O.set_threads(max(1, min(32, os.cpu_count() or 1)))
    cfg = O.michel_config(gamma=4 / 3, sonic_radius=8.0,
                          atmosphere_radius=2.5)
    exact = michel_exact()
    err = {}
    for n in (32, 64):
        p = michel_params(n)
        box = O.make_box((n, n, n))
        s = O.new_state(box)
        O.fill_michel(p, cfg, box, s)
        O.recover_primitives(p, box, s)
        for R in RADII:
            p.accretion_radius = R
            _, m = O.compute_rhs_mdot(p, box, s.copy())
            err[n, R] = m / exact - 1.0
    O.set_threads(1)
    print("oracle Mdot / exact - 1:", {k: f"{v:.2e}" for k, v in err.items()})
    for R in RADII:
        assert abs(err[64, R]) <= 4e-3, (R, err[64, R])
        # second order: the error falls by >= 2^1.5 from n = 32 to 64
        assert abs(err[64, R]) <= abs(err[32, R]) / 2.8, (R, err)
    spread = {n: max(err[n, R] for R in RADII) - min(err[n, R] for R in RADII)
              for n in (32, 64)}
    assert spread[64] <= spread[32] / 2.8, spread
