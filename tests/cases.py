"""Seeded parity cases shared by the GPU tests, smoke() and bench.py's CPU leg.

Each case builds the same level state twice: through the oracle (numpy) and
as the input of the product operator.  Configurations follow the reference
tests and examples:

  fixedbg   Tests/GRHDFixedBGTest.cpp:84-95, 354-432 (KS M=1 a=0.3, dx=0.25,
            box [20,22]x[15,17]x[10,12], synthetic primitive field)
  ksdisk    Examples/GRHDLevelDataKerrSchildDisk (56^2 x 9 torus, a=0)
  pndisk    Examples/GRHDLevelDataBinaryPNDisk (56^2 x 9 torus, binary PN)
  michel18  Tests/GRHDLevelDataMichelAccretion (18^3, dx=2)
  torus_a09 a reduced-size Kerr-Schild torus with spin 0.9 (the 256^3
            workload's physics at 32^3) with a seeded 1e-3 density
            perturbation and the 1e-10 atmosphere
  michel_c1 Michel onto M=1 in KS, Gamma=4/3, r_s=8, on [-16,16]^3 with
            seeded 1e-6 density noise (the 64^3 workload at 24^3),
            excision r < 1.5
"""
from __future__ import annotations

import numpy as np

import oracle_lib as O

SEED = 20261203


def _fixedbg():
    p = O.default_params(ks_mass=1.0, ks_spin=0.3, dx=0.25, gamma=5 / 3,
                         rec_max_iterations=80, limiter_theta=1.5)
    box = O.make_box((3, 3, 3), lo=(20, 15, 10))
    s = O.new_state(box)
    V = O.state_view(box, s)
    for kk in range(box.ghi[2] - box.glo[2] + 1):
        for jj in range(box.ghi[1] - box.glo[1] + 1):
            for ii in range(box.ghi[0] - box.glo[0] + 1):
                i, j, k = box.glo[0] + ii, box.glo[1] + jj, box.glo[2] + kk
                rho = 0.7 + 1.0e-3 * (i + 2 * j + 3 * k)
                eps = 0.12 + 1.0e-4 * (2 * i + j + k)
                V[O.RHO, kk, jj, ii] = rho
                V[O.EPS, kk, jj, ii] = eps
                V[O.PRESS, kk, jj, ii] = (5 / 3 - 1) * rho * eps
                V[O.V1, kk, jj, ii] = 1.0e-3 * (1.0 + i)
                V[O.V2, kk, jj, ii] = -7.5e-4 * (1.0 + j)
                V[O.V3, kk, jj, ii] = 5.0e-4 * (1.0 + k)
    O.fill_conserved_from_primitives(p, box, s)
    return p, box, s, 0.0


def _disk(background):
    num_cells, num_z = 56, 9
    dx = 80.0 / num_cells
    center = (0.5 * num_cells * dx, 0.5 * num_cells * dx, 0.5 * num_z * dx)
    kw = dict(gamma=5.0 / 3.0, dx=dx, center=center, atmo_rho_floor=1e-10,
              atmo_pressure_floor=1e-12, atmo_max_velocity_squared=0.8,
              rec_max_iterations=80, rec_pressure_floor=1e-12,
              rec_max_velocity_squared=0.8, limiter_theta=1.4,
              metric_time_derivative_step=1e-3)
    if background == O.BG_KERR_SCHILD:
        p = O.default_params(background=O.BG_KERR_SCHILD, ks_mass=1.0,
                             ks_spin=0.0, use_metric_volume_time_sources=0,
                             **kw)
        cfg = O.torus_config(total_mass=1.0, inner_radius=7.0,
                             pressure_max_radius=10.0, rho_peak=2e-5,
                             max_velocity_squared=0.8)
    else:
        p = O.default_params(background=O.BG_BINARY_PN, pn_mass_1=0.5,
                             pn_mass_2=0.5, pn_separation=8.0,
                             pn_softening_radius=1.0,
                             use_metric_volume_time_sources=1, **kw)
        cfg = O.torus_config(total_mass=1.0, inner_radius=14.0,
                             pressure_max_radius=18.0, rho_peak=2e-5,
                             max_velocity_squared=0.8)
    box = O.make_box((num_cells, num_cells, num_z))
    s = O.new_state(box)
    tp = O.make_torus(p, cfg, box, 0.0)
    O.fill_torus(p, cfg, tp, box, s, 0.0)
    O.recover_primitives(p, box, s, 0.0)
    return p, box, s, 0.0


def _michel18():
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
    O.recover_primitives(p, box, s)
    return p, box, s, 0.0


def perturb_density(p, box, s, amplitude, seed, time=0.0):
    """rho *= 1 + amplitude * U(-1, 1) over the ghosted box, pressure and
    velocity kept, eps and the conserved variables recomputed."""
    rng = np.random.default_rng(seed)
    V = O.state_view(box, s)
    V[O.RHO] *= 1.0 + amplitude * rng.uniform(-1.0, 1.0, V[O.RHO].shape)
    V[O.EPS] = V[O.PRESS] / ((p.gamma - 1.0) * V[O.RHO])
    O.fill_conserved_from_primitives(p, box, s, time)


def torus_a09(n=32, L=40.0, seed=SEED + 1):
    dx = 2.0 * L / n
    c = 0.5 * n * dx
    p = O.default_params(background=O.BG_KERR_SCHILD, ks_mass=1.0,
                         ks_spin=0.9, gamma=5 / 3, dx=dx, center=(c, c, c),
                         atmo_rho_floor=1e-10, atmo_pressure_floor=1e-12,
                         atmo_max_velocity_squared=0.8, rec_max_iterations=80,
                         rec_max_velocity_squared=0.8, limiter_theta=2.0,
                         excision_radius=1.5)
    cfg = O.torus_config(total_mass=1.0, inner_radius=6.0,
                         pressure_max_radius=12.0, rho_peak=1.0,
                         max_velocity_squared=0.8)
    box = O.make_box((n, n, n))
    s = O.new_state(box)
    tp = O.make_torus(p, cfg, box, 0.0)
    O.fill_torus(p, cfg, tp, box, s, 0.0)
    perturb_density(p, box, s, 1e-3, seed)
    O.recover_primitives(p, box, s)
    return p, box, s, 0.0


def michel_c1(n=24, seed=SEED + 0):
    L = 16.0
    dx = 2.0 * L / n
    c = 0.5 * n * dx
    p = O.default_params(background=O.BG_KERR_SCHILD, ks_mass=1.0,
                         ks_spin=0.0, gamma=4 / 3, dx=dx, center=(c, c, c),
                         atmo_rho_floor=1e-12, atmo_pressure_floor=1e-16,
                         atmo_max_velocity_squared=0.8,
                         rec_max_iterations=100, rec_pressure_floor=1e-16,
                         rec_max_velocity_squared=0.8, limiter_theta=2.0,
                         excision_radius=1.5)
    cfg = O.michel_config(gamma=4 / 3, sonic_radius=8.0,
                          atmosphere_radius=2.5)
    box = O.make_box((n, n, n))
    s = O.new_state(box)
    O.fill_michel(p, cfg, box, s)
    perturb_density(p, box, s, 1e-6, seed)
    O.recover_primitives(p, box, s)
    return p, box, s, 0.0


CASES = {
    "fixedbg": _fixedbg,
    "ksdisk": lambda: _disk(O.BG_KERR_SCHILD),
    "pndisk": lambda: _disk(O.BG_BINARY_PN),
    "michel18": _michel18,
    "torus_a09": torus_a09,
    "michel_c1": michel_c1,
}


def gpu_operator(p, precision="fp64"):
    """The product operator with the oracle case's settings."""
    import grdzhadzha_b200 as G
    eos = G.IdealGasEOS(p.gamma)
    atmo = G.AtmosphereOptions(p.atmo_rho_floor, p.atmo_pressure_floor,
                               p.atmo_max_velocity_squared,
                               p.atmo_metric_source_atmosphere_factor)
    rec = G.RecoveryOptions(p.rec_max_iterations, p.rec_tolerance,
                            p.rec_pressure_floor, p.rec_max_velocity_squared)
    center = tuple(p.center[d] for d in range(3))
    if p.background == O.BG_KERR_SCHILD:
        bg = G.KerrSchild(mass=p.ks_mass, spin=p.ks_spin, dx=p.dx)
        return G.TimeDependentFixedBGLevelDataFiniteVolumeOperator(
            eos, bg, p.dx, center, atmo, p.limiter_theta,
            bool(p.use_reconstruction), rec,
            bool(p.use_static_metric_sources), False,
            p.metric_time_derivative_step, p.excision_radius,
            p.accretion_radius, precision)
    bg = G.CircularBinaryPN(mass_1=p.pn_mass_1, mass_2=p.pn_mass_2,
                            separation=p.pn_separation,
                            angular_velocity=p.pn_angular_velocity,
                            phase=p.pn_phase, time=p.pn_time,
                            softening_radius=p.pn_softening_radius, dx=p.dx)
    return G.TimeDependentFixedBGLevelDataFiniteVolumeOperator(
        eos, bg, p.dx, center, atmo, p.limiter_theta,
        bool(p.use_reconstruction), rec, bool(p.use_static_metric_sources),
        bool(p.use_metric_volume_time_sources),
        p.metric_time_derivative_step, p.excision_radius, p.accretion_radius,
        precision)


def gpu_level(box, state_np, device="cuda"):
    import torch
    import grdzhadzha_b200 as G
    lv = G.LevelBox(lo=tuple(box.lo), hi=tuple(box.hi),
                    ghost=box.lo[0] - box.glo[0],
                    domain_lo=tuple(box.dlo), domain_hi=tuple(box.dhi),
                    state=torch.empty(0), device=device)
    shape = O.state_view(box, state_np).shape
    lv.state = torch.from_numpy(state_np.reshape(shape).copy()).to(device)
    return lv


def rel_err(got: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Per-component max|got - ref| / scale (components on axis 0).

    The scale of a scalar component is its own max|ref|; the three
    components of a vector (S_i in the conserved set, v^i in the
    primitives) share the max over the vector, since an axis-dependent
    normalisation would turn a component that is a small residual of
    cancelling terms (e.g. S_z of a disk in vertical balance) into a large
    relative error of ordinary rounding."""
    g = got.reshape(got.shape[0], -1)
    r = ref.reshape(ref.shape[0], -1)
    scale = np.maximum(np.abs(r).max(axis=1), 1e-300)
    groups = {5: [(1, 4)], 11: [(1, 4), (8, 11)]}.get(got.shape[0], [])
    for a, b in groups:
        scale[a:b] = scale[a:b].max()
    return np.abs(g - r).max(axis=1) / scale


def oracle_params_of(op) -> O.Params:
    """The oracle's parameters for a product operator (any background),
    field by field from the operator's own parameter block."""
    q = op.params
    names = {"gamma": "adiabatic_index", "atmo_rho_floor": "rho_floor",
             "atmo_pressure_floor": "pressure_floor",
             "atmo_max_velocity_squared": "max_velocity_squared",
             "atmo_metric_source_atmosphere_factor":
                 "metric_source_atmosphere_factor",
             "rec_max_iterations": "recovery_max_iterations",
             "rec_tolerance": "recovery_tolerance",
             "rec_pressure_floor": "recovery_pressure_floor",
             "rec_max_velocity_squared": "recovery_max_velocity_squared"}
    p = O.default_params()
    for field, _ in O.Params._fields_:
        v = getattr(q, names.get(field, field))
        if field == "center":
            v = tuple(v)
        setattr(p, field, v)
    return p


def dilate_cross(mask: np.ndarray, r: int = 2) -> np.ndarray:
    """Cells within r cells of a marked cell along one axis (the reach of
    a cell's primitives into the MUSCL-HLLE RHS: the slopes of the two
    neighbours on each side read it); no wrap-around."""
    out = mask.copy()
    for ax in range(mask.ndim):
        for s in range(1, r + 1):
            a = [slice(None)] * mask.ndim
            b = [slice(None)] * mask.ndim
            a[ax], b[ax] = slice(s, None), slice(None, -s)
            out[tuple(a)] |= mask[tuple(b)]
            out[tuple(b)] |= mask[tuple(a)]
    return out


def rhs_parity_by_con2prim(got, ref, p_gpu, p_orc, tol):
    """Split an RHS comparison by the con2prim root solves behind it.

    The reference's con2prim (Valencia.hpp:116-228) stops Newton at the
    first iterate with |f(p)| < tol, an absolute tolerance on a residual of
    size tau + D.  Two correct evaluations whose rounding differs (another
    compiler's contraction of the reference itself, or another closed form
    of gamma^ij) accept different iterates where |f| lands within rounding
    of tol; there the pressures differ by about tol / f'(p) (< tol, since
    f' > 1 / (Gamma - 1) >= 1.5), where elsewhere they agree to rounding
    (~1e-16 (tau + D)).  Cells whose recovered pressures differ by more
    than 1e-2 tol are such flips; every RHS cell within two cells of one
    along an axis reads its primitives.

    got, ref: (5, ncell) RHS; p_gpu, p_orc: recovered pressures (n, n, n).
    Returns (flip count, per-component max error outside the flips'
    reach relative to the component's scale as rel_err, per-component
    max absolute difference inside their reach)."""
    flips = np.abs(p_gpu - p_orc) > 1e-2 * tol
    reach = dilate_cross(flips).reshape(-1)
    g = got.reshape(5, -1)
    r = ref.reshape(5, -1)
    scale = np.abs(r).max(axis=1)
    scale[1:4] = scale[1:4].max()
    out = np.abs(g[:, ~reach] - r[:, ~reach]).max(axis=1) / scale
    inside = (np.abs(g[:, reach] - r[:, reach]).max(axis=1) if reach.any()
              else np.zeros(5))
    return int(flips.sum()), out, inside


def build_cxx_dropin(out_dir) -> str:
    """Compiles tests/cxx_dropin.cpp (the C++ drop-in operator class over
    include/grhd_b200.h) with g++ and links it to libgrhd_b200.so and the
    CUDA runtime; returns the executable's path."""
    import os
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    libdir = os.path.join(root, "grdzhadzha_b200")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = os.path.join(str(out_dir), "cxx_dropin")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra",
                    "-Werror", "-I", os.path.join(root, "include"),
                    "-I", os.path.join(cuda, "include"),
                    os.path.join(here, "cxx_dropin.cpp"), "-L", libdir,
                    "-lgrhd_b200", "-L", os.path.join(cuda, "lib64"),
                    "-lcudart", f"-Wl,-rpath,{libdir}", "-o", exe],
                   check=True)
    return exe
