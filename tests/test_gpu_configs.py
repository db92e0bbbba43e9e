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


def _recovered_pressure(op, box, s, n, time=0.0):
    """Pressures of the same state recovered by the GPU and by the oracle
    (interior, (n, n, n))."""
    lv = cases.gpu_level(box, s)
    op.recover_primitives(lv, time=time)
    pg = lv.interior(slice(O.PRESS, O.PRESS + 1)).cpu().numpy()
    so = s.copy()
    O.recover_primitives(cases.oracle_params_of(op), box, so, time)
    po = O.interior(box, so, slice(O.PRESS, O.PRESS + 1))
    return pg.reshape(n, n, n), po.reshape(n, n, n)


def _full_size_rhs_parity(op, lv, n, time=0.0):
    """The FP64 RHS of the GPU-generated state against the oracle's
    multi-box RHS of the same state, split by con2prim iterate flips
    (cases.rhs_parity_by_con2prim)."""
    O.set_threads(_threads())
    s = lv.state.cpu().numpy().reshape(-1).copy()
    rhs = lv.new_rhs()
    op.compute_rhs(rhs, lv, time=time)
    got = rhs.cpu().numpy().reshape(5, -1)
    del rhs
    p = cases.oracle_params_of(op)
    box = O.make_box((n, n, n))
    ref = O.compute_rhs_slabs(p, box, s.copy(), _threads(), time)
    ref = ref.reshape(5, -1)
    pg, po = _recovered_pressure(op, box, s, n, time)
    tol = op.params.recovery_tolerance
    flips, out, inside = cases.rhs_parity_by_con2prim(got, ref, pg, po, tol)
    return (flips, out, inside, cases.rel_err(got, ref),
            _where(got, ref, op, n), tol / op.params.dx)


def test_config2_torus_256_rhs_matches_oracle():
    """Config 2's FP64 RHS against the oracle at 256^3, per component
    relative to max|RHS_oracle|.

    Every cell outside the reach of a con2prim iterate flip: <= 1e-12
    (measured on B200: 6e-14 to 3e-13).  A flip is a cell where the two
    root solves accepted different Newton iterates (|dp| ~ tol / f', up to
    6.5e-13, against rounding-level ~1e-16 elsewhere); it happens between
    any two correct evaluations that round differently, the reference's
    own algorithm included (the oracle built with and without FMA
    contraction flips 3 cells of 2.1M on a 128^3 torus, tests/
    test_oracle_conditioning.py).  Inside a flip's reach the RHS differs by
    the flux of that pressure difference over one cell: bound 4 tol / dx
    (measured 1.2 tol / dx); flips at most 1e-3 of the cells."""
    from grdzhadzha_b200 import workloads as W
    n = 256
    op, lv = W.kerr_schild_torus(n)
    flips, out, inside, allc, where, tol_dx = _full_size_rhs_parity(op, lv, n)
    print(f"torus 256^3: {flips} con2prim flips; outside their reach "
          f"{out}; inside max|d| {inside} (tol/dx {tol_dx:.2e}); all "
          f"cells {allc}; {where}")
    assert np.all(out <= 1e-12), out
    assert np.all(inside <= 4.0 * tol_dx), inside
    assert flips <= 1e-3 * n ** 3, flips


def _oracle_spread(p, box, s, threads, time=0.0):
    """rel_err between the oracle's timing build (-O3, FMA) and its parity
    build on the same input: how far two correct compilations of the
    reference's algorithm are apart on this state."""
    import ctypes as C
    out = []
    for L in (O.lib(), O.fast_lib()):
        L.orc_set_threads(threads)
        n = O.interior_cells(box)
        rhs = np.zeros(5 * n)
        inv = np.array([1.0 / p.dx] * 3)
        err = O.Error()
        assert L.orc_compute_rhs_slabs(C.byref(p), C.byref(box),
                                       O._dp(s.copy()), O._dp(rhs), n,
                                       O._dp(inv), time, threads,
                                       C.byref(err)) == 0
        out.append(rhs.reshape(5, -1))
    return cases.rel_err(out[1], out[0])


def test_config3_binary_disk_320_fp64_rhs_matches_oracle():
    """Config 3 (the circumbinary disk on the time-dependent PN metric) at
    its full 320^3, FP64 RHS against the oracle's, in two parts.

    The thin disk (H/R = 0.1) is near equilibrium: its RHS is a residual
    ~1e-3 of the flux and source terms that cancel in it, so rounding at
    the level of those terms is ~1e-11 of max|RHS| -- for two builds of the
    reference's own algorithm as much as for GPU against oracle.

    * The operator without the volume-time source: per component, the GPU
      is within max(1e-12, 2 x spread) of the oracle, spread = the oracle's
      FMA build against its no-FMA build on the same state, measured here
      (on B200: GPU 1.1e-12 to 3.0e-11; no con2prim flips).
    * The volume-time source -q d_t ln sqrt(gamma) (FixedBGFArrayBoxFinite
      Volume.hpp:616-675), a central difference in time with step h =
      1e-3: ln sqrt(gamma) = log(det gamma) / 2 comes from CUDA's log
      (within 1 ulp) on the GPU and from libm's on the host, and the
      difference quotient carries that ulp times 1/(2h).  Per cell
      |term_GPU - term_oracle| <= |q| (2 ulp(4) / 2) / (2h) = |q| 4.4e-13
      (log det < 4 on this grid; measured: at most |q| 5.55e-14, one ulp
      of log det in [1, 2), in 22 % of the cells)."""
    from grdzhadzha_b200 import workloads as W
    n = 320
    th = _threads()
    op0, lv = W.binary_disk(n, precision="fp64")
    s = lv.state.cpu().numpy().reshape(-1).copy()
    del lv
    box = O.make_box((n, n, n))
    O.set_threads(th)
    got, ref = {}, {}
    for vol in (0, 1):
        p = cases.oracle_params_of(op0)
        p.use_metric_volume_time_sources = vol
        op = cases.gpu_operator(p)
        lv = cases.gpu_level(box, s)
        rhs = lv.new_rhs()
        op.compute_rhs(rhs, lv, time=0.0)
        got[vol] = rhs.cpu().numpy().reshape(5, -1)
        del rhs, lv, op
        ref[vol] = O.compute_rhs_slabs(p, box, s.copy(), th).reshape(5, -1)
        if vol == 0:
            spread = _oracle_spread(p, box, s, th)
            pg, po = _recovered_pressure(cases.gpu_operator(p), box, s, n)
            flips = int((np.abs(pg - po) > 1e-2 * p.rec_tolerance).sum())
    torch.cuda.empty_cache()
    err0 = cases.rel_err(got[0], ref[0])
    print(f"binary disk 320^3 without the volume source: GPU vs oracle "
          f"{err0}, oracle FMA vs no-FMA {spread}, {flips} flips")
    assert flips <= 1e-3 * n ** 3, flips
    assert np.all(err0 <= np.maximum(1e-12, 2.0 * spread)), (err0, spread)
    q = O.interior(box, s).reshape(5, -1)
    h = op0.params.metric_time_derivative_step
    dterm = np.abs((got[1] - got[0]) - (ref[1] - ref[0]))
    ratio = dterm / np.maximum(np.abs(q), 1e-300)
    bound = (2.0 * np.spacing(4.0) / 2.0) / (2.0 * h)
    print(f"volume-time source: max |d| / |q| {ratio.max(axis=1)} "
          f"(bound {bound:.2e}); cells differing "
          f"{(dterm[0] > 0).mean():.3f}")
    assert np.all(dterm <= bound * np.abs(q) + 1e-300), ratio.max(axis=1)


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


@pytest.mark.parametrize("name", ["michel_c1", "torus_a09"])
def test_fp64_drift_against_oracle_100_steps(name):
    """Drift of the FP64 GPU state from the oracle's over N RK4 steps with
    the same dt, on 64^3 grids: config 1 (Michel inflow, a = 0, excision)
    and the config-2 torus (a = 0.9) at 64^3.  Each step's RHS agrees to
    rounding except where a con2prim root solve accepts a different Newton
    iterate (see test_config2_torus_256_rhs_matches_oracle); the drift is
    how far those differences carry.  Per conserved component, max|U_gpu -
    U_oracle| relative to the component's scale (rel_err), after 10 and 100
    steps, against the spread of two correct compilations of the
    reference's algorithm on the same steps: the oracle's FMA build against
    its no-FMA build, run beside it here.  Bounds max(5e-12, 2 x spread)
    after 10 steps and max(1e-9, 2 x spread) after 100, the spread taken
    over the components.  Measured on B200: Michel 7.5e-16 / 8.6e-16
    (smooth inflow, no flips); torus 1.1e-12 / 1.3e-9 against an oracle
    spread of 1.0e-12 / 2.9e-9."""
    n = 64
    p, box, s, t = cases.CASES[name](n=n)
    # the benchmark torus's recovery cap above the atmosphere cap
    # (grdzhadzha_b200.workloads.kerr_schild_torus)
    p.rec_max_velocity_squared = 0.9
    O.set_threads(_threads())
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, s)
    dt = O.stable_dt(p, box, s.copy(), 0.25, t)
    state = s.copy()
    fma_state = s.copy()
    fast = O.fast_lib()
    drift, spread = {}, {}
    for step in range(1, 101):
        op.advance_rk4(lv, time=t, dt=dt)
        O.advance_rk4(p, box, state, t, dt)
        O.advance_rk4(p, box, fma_state, t, dt, L=fast)
        t += dt
        if step in (10, 100):
            got = lv.interior(slice(0, 5)).cpu().numpy()
            want = O.interior(box, state)
            drift[step] = cases.rel_err(got, want)
            spread[step] = float(cases.rel_err(
                O.interior(box, fma_state), want).max())
    print(f"{name} 64^3 FP64 drift vs oracle: after 10 steps {drift[10]}, "
          f"after 100 steps {drift[100]}; oracle FMA vs no-FMA {spread}")
    assert np.all(drift[10] <= max(5e-12, 2.0 * spread[10])), (drift, spread)
    assert np.all(drift[100] <= max(1e-9, 2.0 * spread[100])), (drift, spread)
