"""The benchmark configurations at their full sizes (the binary disk's are
in test_gpu_kitp.py, the ensemble's in test_gpu_ensemble.py, the
adjoint's in test_gpu_adjoint.py).

* Config 1, Michel inflow 64^3 on [-16, 16]^3 (FP64): one RHS and two RK4
  steps against the oracle on the same input (RHS <= 1e-12 of each
  component's scale; the steps' change <= 1e-11 of its scale, as the
  smaller parity tests), then 100 RK4 steps on the GPU: finite, and the
  rest mass changes by less than 10 % (the reference's own bar for its
  LevelData Michel run, Tests/GRHDLevelDataMichelAccretion/
  GRHDLevelDataMichelAccretion.cpp:649-682).
* Config 2, Kerr-Schild torus a = 0.9, 256^3 on [-40, 40]^3: the FP64 RHS
  of the GPU-generated initial state against the oracle's multi-box RHS of
  the same state, and two RK4 steps of the mixed path against FP64 with
  the same dt.  The RHS bound is the one that does not depend on the
  grid: the RHS difference times a CFL step (CFL 0.25) <= 1e-12 of each
  conserved component's scale.  (Relative to the RHS itself the 32^3
  torus meets 1e-12, but on the fine grid the equilibrium torus's RHS is a
  small residual, max |RHS| 0.03 against |U| ~ 1, while the differences
  stay at the ~1e-12 absolute level of the con2prim solves stopping at
  neighbouring iterates; measured 1.4e-12 to 4.0e-12.)  The mixed path
  differs from FP64 by up to 1.5e-4 of the scale after two steps
  (measured; at the torus's surface, where the density falls to the
  atmosphere and the FP32 reconstruction and floors act differently),
  bound 3e-4.
"""
import os

import numpy as np
import pytest

import cases
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _threads():
    return max(1, min(32, os.cpu_count() or 1))


def test_config1_michel_64():
    p, box, s, t = cases.michel_c1(n=64)
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, s)
    rhs = lv.new_rhs()
    op.compute_rhs(rhs, lv, time=t)
    ref = O.compute_rhs(p, box, s.copy(), t)
    err = cases.rel_err(rhs.cpu().numpy().reshape(5, -1), ref.reshape(5, -1))
    assert np.all(err <= 1e-12), err
    lv = cases.gpu_level(box, s)
    state = s.copy()
    for _ in range(2):
        dt = O.stable_dt(p, box, state, 0.25, t)
        op.advance_rk4(lv, time=t, dt=dt)
        O.advance_rk4(p, box, state, t, dt)
        t += dt
    got = lv.interior(slice(0, 5)).cpu().numpy()
    want = O.interior(box, state)
    start = O.interior(box, s)
    err = cases.rel_err(got - start, want - start)
    assert np.all(err <= 1e-11), err
    mass0 = float(lv.interior(slice(0, 1)).sum())
    tn, mi, _ = op.advance_rk4_cfl_steps(lv, 0.25, 100, time=t)
    assert torch.isfinite(lv.state).all()
    mass1 = float(lv.interior(slice(0, 1)).sum())
    print(f"Michel 64^3: 102 steps to t = {tn:.3f}, mass change "
          f"{mass1 / mass0 - 1:.3e}")
    assert abs(mass1 / mass0 - 1.0) < 0.1


def _where(got, want, op, n):
    """Cell and coordinate radius of each component's largest difference
    (printed with the failing case)."""
    out = []
    dx, c = op.params.dx, op.params.center
    for q in range(5):
        d = np.abs(got[q] - want[q])
        f = int(np.argmax(d))
        k, j, i = np.unravel_index(f, (n, n, n))
        x, y, z = ((i + 0.5) * dx - c[0], (j + 0.5) * dx - c[1],
                   (k + 0.5) * dx - c[2])
        out.append((q, (i, j, k), round(float(np.sqrt(x * x + y * y + z * z)),
                                        3), float(d.max()),
                    float(np.abs(want[q]).max())))
    return out


def _oracle_params_of_torus(op):
    """The oracle's parameters for grdzhadzha_b200.workloads.
    kerr_schild_torus (Kerr-Schild, excision, no volume-time source)."""
    q = op.params
    return O.default_params(
        background=O.BG_KERR_SCHILD, ks_mass=q.ks_mass, ks_spin=q.ks_spin,
        gamma=q.adiabatic_index, dx=q.dx, center=tuple(q.center),
        atmo_rho_floor=q.rho_floor, atmo_pressure_floor=q.pressure_floor,
        atmo_max_velocity_squared=q.max_velocity_squared,
        atmo_metric_source_atmosphere_factor=q.metric_source_atmosphere_factor,
        rec_max_iterations=q.recovery_max_iterations,
        rec_tolerance=q.recovery_tolerance,
        rec_pressure_floor=q.recovery_pressure_floor,
        rec_max_velocity_squared=q.recovery_max_velocity_squared,
        limiter_theta=q.limiter_theta,
        use_reconstruction=q.use_reconstruction,
        use_static_metric_sources=q.use_static_metric_sources,
        use_metric_volume_time_sources=0,
        excision_radius=q.excision_radius)


def test_config2_torus_256_rhs_matches_oracle():
    from grdzhadzha_b200 import workloads as W
    n = 256
    op, lv = W.kerr_schild_torus(n)
    s = lv.state.cpu().numpy().reshape(-1).copy()
    rhs = lv.new_rhs()
    op.compute_rhs(rhs, lv)
    p = _oracle_params_of_torus(op)
    box = O.make_box((n, n, n))
    ref = O.compute_rhs_slabs(p, box, s, _threads())
    got = rhs.cpu().numpy().reshape(5, -1)
    dt = op.compute_stable_dt(cases.gpu_level(box, s), cfl=0.25)
    u = O.interior(box, s).reshape(5, -1)
    scale = np.abs(u).max(axis=1)
    scale[1:4] = scale[1:4].max()
    err = np.abs(got - ref.reshape(5, -1)).max(axis=1) * dt / scale
    print("torus 256^3 RHS err x dt / |U|", err,
          _where(got, ref.reshape(5, -1), op, n))
    assert np.all(err <= 1e-12), err


def test_config2_torus_256_mixed_against_fp64():
    from grdzhadzha_b200 import workloads as W
    op64, a = W.kerr_schild_torus(256, precision="fp64")
    opm, b = W.kerr_schild_torus(256, precision="mixed")
    assert torch.equal(a.state, b.state)
    dt = op64.compute_stable_dt(a, cfl=0.25)
    t = 0.0
    for _ in range(2):
        op64.advance_rk4(a, time=t, dt=dt)
        opm.advance_rk4(b, time=t, dt=dt)
        t += dt
    got = b.interior(slice(0, 5)).cpu().numpy().reshape(5, -1)
    want = a.interior(slice(0, 5)).cpu().numpy().reshape(5, -1)
    err = cases.rel_err(got, want)
    print("torus 256^3 mixed vs FP64 after 2 steps:", err,
          _where(got, want, op64, 256))
    assert np.all(err <= 3e-4), err
