"""Seeded synthetic workloads built on the device: Kerr-Schild tori and
Michel inflows, singly or as the batched ensemble of many of them.

Setups follow the reference's torus and Michel initial data
(Source/InitialConditions/FixedBGTorus.hpp:291-409,
Tests/GRHDLevelDataMichelAccretion/GRHDLevelDataMichelAccretion.cpp:
312-372); sizes, seeds and parameter ranges are this package's choices,
stated in each function."""
from __future__ import annotations

import numpy as np

from .operator import (AtmosphereOptions, CircularBinaryPN, IdealGasEOS,
                       KerrSchild, LevelBox,
                       RecoveryOptions,
                       TimeDependentFixedBGLevelDataFiniteVolumeOperator)

SEED = 20261203


def kerr_schild_torus(n, spin=0.9, half_width=40.0, gamma=5.0 / 3.0,
                      inner_radius=6.0, pressure_max_radius=12.0,
                      rho_peak=1.0, perturbation=1e-3, seed=SEED + 1,
                      accretion_radius=0.0, precision="fp64",
                      device="cuda"):
    """Constant-angular-momentum torus around a Kerr-Schild hole (M = 1)
    on an n^3 grid over [-half_width, half_width]^3: atmosphere 1e-10 /
    1e-12 / v^2 cap 0.8, recovery v^2 cap 0.9, MUSCL-MC (theta 2) + HLLE,
    excision r < 1.5, density times (1 + perturbation U(-1, 1)).  Returns
    (operator, level).

    The recovery cap sits above the atmosphere cap: the floors rescale a
    fast cell's velocity to exactly the atmosphere cap (Atmosphere.hpp:
    36-40), and with equal caps the next con2prim of that reset state
    fails whenever rounding puts v^2 on or above the cap."""
    nn = (n, n, n) if isinstance(n, int) else tuple(n)
    dx = 2.0 * half_width / nn[0]
    c = tuple(0.5 * nn[d] * dx for d in range(3))
    op = TimeDependentFixedBGLevelDataFiniteVolumeOperator(
        IdealGasEOS(gamma), KerrSchild(mass=1.0, spin=spin, dx=dx), dx, c,
        AtmosphereOptions(1e-10, 1e-12, 0.8), 2.0, True,
        RecoveryOptions(80, 1e-12, 1e-12, 0.9), True, False, 1e-3, 1.5,
        accretion_radius, precision)
    lv = LevelBox.cube(nn, device=device)
    op.fill_torus(lv, inner_radius=inner_radius,
                  pressure_max_radius=pressure_max_radius, rho_peak=rho_peak,
                  max_velocity_squared=0.8)
    if perturbation:
        op.perturb_density(lv, perturbation, seed)
    op.recover_primitives(lv)
    return op, lv


def binary_pn_disk(n, half_width=40.0, gamma=5.0 / 3.0, inner_radius=14.0,
                   pressure_max_radius=18.0, rho_peak=2e-5, separation=8.0,
                   softening_radius=1.0, precision="fp64", device="cuda"):
    """Circumbinary torus around the circular PN binary (masses 0.5 + 0.5,
    separation 8, softening 1; the binary disk drivers' setting) on an n^3
    grid over [-half_width, half_width]^3: atmosphere 1e-10 / 1e-12 / v^2
    cap 0.8, MUSCL-MC (theta 1.4) + HLLE, volume-time source on.  Returns
    (operator, level)."""
    nn = (n, n, n) if isinstance(n, int) else tuple(n)
    dx = 2.0 * half_width / nn[0]
    c = tuple(0.5 * nn[d] * dx for d in range(3))
    op = TimeDependentFixedBGLevelDataFiniteVolumeOperator(
        IdealGasEOS(gamma),
        CircularBinaryPN(mass_1=0.5, mass_2=0.5, separation=separation,
                         softening_radius=softening_radius, dx=dx),
        dx, c, AtmosphereOptions(1e-10, 1e-12, 0.8), 1.4, True,
        RecoveryOptions(80, 1e-12, 1e-12, 0.8), True, True, 1e-3, 0.0, 0.0,
        precision)
    lv = LevelBox.cube(nn, device=device)
    op.fill_torus(lv, inner_radius=inner_radius,
                  pressure_max_radius=pressure_max_radius, rho_peak=rho_peak,
                  max_velocity_squared=0.8)
    op.recover_primitives(lv)
    return op, lv


def binary_disk(n=320, half_width=60.0, gamma=5.0 / 3.0, inner_radius=20.0,
                outer_radius=50.0, aspect_ratio=0.1, mode_amplitude=1e-3,
                seed=SEED + 2, precision="mixed", device="cuda"):
    """The binary-disk configuration: circular PN binary (0.5 + 0.5,
    separation 10, softening 0.5, Newtonian orbital frequency) with the disk
    drivers' Keplerian disk (kitp_primitive) between inner_radius (the
    cavity edge, 2 separations) and outer_radius (the logistic cut-off),
    H/R = aspect_ratio (Mach 1 / aspect_ratio), and azimuthal density
    modes m = 1..4 of amplitude mode_amplitude with phases U[0, 2 pi)
    (numpy, seeded); n^3 over [-half_width, half_width]^3, atmosphere
    1e-10 / 8e-14 / v^2 cap 0.72 and recovery floor 8e-14 / v^2 cap 0.75
    (the driver's, make_recovery_options, :339-346), MUSCL-MC (theta 1.3) +
    HLLE, volume-time source on.  Returns (operator, level)."""
    nn = (n, n, n) if isinstance(n, int) else tuple(n)
    dx = 2.0 * half_width / nn[0]
    c = tuple(0.5 * nn[d] * dx for d in range(3))
    sep = 10.0
    op = TimeDependentFixedBGLevelDataFiniteVolumeOperator(
        IdealGasEOS(gamma),
        CircularBinaryPN(mass_1=0.5, mass_2=0.5, separation=sep,
                         softening_radius=0.5, dx=dx),
        dx, c, AtmosphereOptions(1e-10, 8e-14, 0.72), 1.3, True,
        RecoveryOptions(80, 1e-12, 8e-14, 0.75), True, True, 1e-3, 0.0, 0.0,
        precision)
    rng = np.random.default_rng(seed)
    lv = LevelBox.cube(nn, device=device)
    op.fill_kitp_disk(lv, mach=1.0 / aspect_ratio, aspect_ratio=aspect_ratio,
                      cavity_radius_factor=inner_radius / sep,
                      outer_cutoff_radius=outer_radius,
                      mode_amplitude=[mode_amplitude] * 4,
                      mode_phase=list(rng.uniform(0.0, 2.0 * np.pi, 4)))
    return op, lv


def michel(n, sonic_radius=8.0, half_width=16.0, gamma=4.0 / 3.0,
           noise=1e-6, seed=SEED, accretion_radius=0.0, precision="fp64",
           device="cuda"):
    """Michel inflow onto a Schwarzschild hole (M = 1) in Kerr-Schild
    coordinates on an n^3 grid over [-half_width, half_width]^3: sonic
    density 1e-6, atmosphere inside r = 2.5 and floors 1e-12 / 1e-16,
    v^2 caps 0.8 (atmosphere) / 0.9 (recovery), MUSCL-MC (theta 2) + HLLE,
    excision r < 1.5, density times (1 + noise U(-1, 1)).  Returns
    (operator, level)."""
    nn = (n, n, n) if isinstance(n, int) else tuple(n)
    dx = 2.0 * half_width / nn[0]
    c = tuple(0.5 * nn[d] * dx for d in range(3))
    op = TimeDependentFixedBGLevelDataFiniteVolumeOperator(
        IdealGasEOS(gamma), KerrSchild(mass=1.0, spin=0.0, dx=dx), dx, c,
        AtmosphereOptions(1e-12, 1e-16, 0.8), 2.0, True,
        RecoveryOptions(100, 1e-12, 1e-16, 0.9), True, False, 1e-3, 1.5,
        accretion_radius, precision)
    lv = LevelBox.cube(nn, device=device)
    op.fill_michel(lv, sonic_radius=sonic_radius, sonic_density=1e-6,
                   atmosphere_radius=2.5)
    if noise:
        op.perturb_density(lv, noise, seed)
    op.recover_primitives(lv)
    return op, lv


def batched_ensemble(count=96, sizes=(32, 48, 64, 96, 128), seed=SEED + 3,
                     precision="mixed", device="cuda", max_cells=None):
    """The batched ensemble: `count` independent members with n drawn
    uniformly from `sizes`; the first half Michel inflows (sonic radius
    U[5, 12], half width 2 r_s, Gamma 4/3, accretion sphere r = 4), the
    second half Kerr-Schild tori (spin U[0, 0.99], inner edge U[6, 10],
    pressure maximum inner + 6, half width 40, Gamma 4/3 or 5/3, accretion
    sphere r = 2.5); numpy seeded.  `max_cells` (optional) caps the total
    cell count by dropping the largest sizes.  Returns (members, specs)."""
    rng = np.random.default_rng(seed)
    members, specs = [], []
    total = 0
    for i in range(count):
        n = int(rng.choice(sizes))
        if max_cells is not None:
            while n ** 3 + total > max_cells and n > min(sizes):
                n = max(s for s in sizes if s < n)
        total += n ** 3
        if i < count // 2:
            rs = float(rng.uniform(5.0, 12.0))
            spec = {"kind": "michel", "n": n, "sonic_radius": rs,
                    "half_width": 2.0 * rs, "gamma": 4.0 / 3.0,
                    "seed": int(seed + i)}
            op, lv = michel(n, sonic_radius=rs, half_width=2.0 * rs,
                            seed=spec["seed"], accretion_radius=4.0,
                            precision=precision, device=device)
        else:
            a = float(rng.uniform(0.0, 0.99))
            rin = float(rng.uniform(6.0, 10.0))
            g = float(rng.choice([4.0 / 3.0, 5.0 / 3.0]))
            spec = {"kind": "torus", "n": n, "spin": a, "inner_radius": rin,
                    "pressure_max_radius": rin + 6.0, "gamma": g,
                    "seed": int(seed + i)}
            op, lv = kerr_schild_torus(n, spin=a, gamma=g, inner_radius=rin,
                                       pressure_max_radius=rin + 6.0,
                                       seed=spec["seed"],
                                       accretion_radius=2.5,
                                       precision=precision, device=device)
        members.append((op, lv))
        specs.append(spec)
    return members, specs


def adjoint_torus(n=128, half_width=20.0, steps=400, checkpoint_every=25,
                  spin=0.7, gamma=5.0 / 3.0, inner_radius=3.5,
                  pressure_max_radius=6.0, accretion_radius=2.5, cfl=0.25,
                  device="cuda"):
    """The adjoint workload: a constant-angular-momentum torus around a
    Kerr-Schild hole (M = 1, spin 0.7) on an n^3 grid over
    [-half_width, half_width]^3, inner edge 3.5, pressure maximum 6 (close
    enough that its inner edge spills through r = 2.5 within the run),
    Gamma 5/3, density 1 at the pressure maximum, five azimuthal density
    modes of amplitudes 1e-2 .. 2e-3 with fixed phases, atmosphere
    1e-10 / 1e-12 / v^2 cap 0.8, recovery v^2 cap 0.9, MUSCL-MC + HLLE,
    excision r < 1.5; J = integral of the accretion rate through r = 2.5
    over `steps` RK4 steps of the fixed size cfl / (max inverse dt of the
    initial state).  Returns (operator, adjoint)."""
    from .adjoint import TorusAccretionAdjoint, default_torus
    nn = (n, n, n) if isinstance(n, int) else tuple(n)
    dx = 2.0 * half_width / nn[0]
    c = tuple(0.5 * nn[d] * dx for d in range(3))
    op = TimeDependentFixedBGLevelDataFiniteVolumeOperator(
        IdealGasEOS(gamma), KerrSchild(mass=1.0, spin=spin, dx=dx), dx, c,
        AtmosphereOptions(1e-10, 1e-12, 0.8), 2.0, True,
        RecoveryOptions(80, 1e-12, 1e-12, 0.9), True, False, 1e-3, 1.5,
        accretion_radius, "fp64")
    lv = LevelBox.cube(nn, device=device)
    torus = default_torus(spin=spin, inner_radius=inner_radius,
                          pressure_max_radius=pressure_max_radius)
    # the step size: CFL of the initial state, computed by a one-step
    # adjoint object (no tape beyond one step)
    probe = TorusAccretionAdjoint(op, lv, 1, 1, 1.0, torus)
    probe.initial_state(level=lv)
    dt = cfl / op.compute_max_inverse_dt(lv)
    del probe
    adj = TorusAccretionAdjoint(op, lv, steps, checkpoint_every, dt, torus)
    return op, adj
