"""The oracle's restatement of the operator on CCZ4-stored geometry
(LevelDataFiniteVolumeOperator, Source/Matter/GRHD/FArrayBoxFiniteVolume.hpp:
681-1364), pinned against the fixed-background operator the way the
reference pins it.

* The reference's own check (Tests/GRHDFixedBGTest/GRHDFixedBGTest.cpp:
  195-237): with the CCZ4 variables filled from the Kerr-Schild background
  (store_ccz4_background_vars, :97-134) and the test primitive field of
  :84-95 on the box [20..22]x[15..17]x[10..12] with 2 ghosts and the
  problem domain equal to the ghosted box, the CCZ4-geometry flux RHS equals
  the fixed-background flux RHS to 1e-10 (the reference's tolerance).
* The sources: their finite-difference metric derivatives converge to the
  analytic ones at second order (error ratio near 4 when dx halves with the
  cell at the same place).
* Recovery and the CFL bound on the same state agree with the fixed-
  background operator to 1e-12 (only the geometry's rounding differs).
"""
import numpy as np

import cases
import oracle_lib as O


def _reference_box(n=3, lo=(20, 15, 10)):
    """The reference test's box: domain = ghosted box (no physical ghost)."""
    box = O.make_box((n, n, n), lo=lo)
    for d in range(3):
        box.dlo[d], box.dhi[d] = box.glo[d], box.ghi[d]
    return box


def _test_state(p, box):
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
                V[O.PRESS, kk, jj, ii] = (p.gamma - 1) * rho * eps
                V[O.V1, kk, jj, ii] = 1.0e-3 * (1.0 + i)
                V[O.V2, kk, jj, ii] = -7.5e-4 * (1.0 + j)
                V[O.V3, kk, jj, ii] = 5.0e-4 * (1.0 + k)
    O.fill_conserved_from_primitives(p, box, s)
    return s


def _params(**kw):
    base = dict(ks_mass=1.0, ks_spin=0.3, dx=0.25, gamma=5 / 3,
                rec_max_iterations=80, limiter_theta=1.5)
    base.update(kw)
    return O.default_params(**base)


def test_ccz4_flux_rhs_equals_fixed_background():
    p = _params(use_static_metric_sources=0)
    box = _reference_box()
    s = _test_state(p, box)
    fixed = O.compute_rhs(p, box, s.copy()).reshape(5, -1)
    ccz4 = O.ccz4_compute_rhs(p, box, O.ccz4_state(p, box, s)).reshape(5, -1)
    err = cases.rel_err(ccz4, fixed)
    print("flux RHS, CCZ4 vs fixed background:", err)
    assert np.all(err <= 1e-10), err


def _source_error(dx):
    """max |CCZ4 source - analytic source| at the middle cell (21,16,11)
    placed at the same point for every dx."""
    X = (5.375, 4.125, 2.875)
    centre = tuple((m + 0.5) * dx - X[d] for d, m in enumerate((21, 16, 11)))
    out = []
    for src in (1, 0):
        p = _params(dx=dx, center=centre, use_static_metric_sources=src)
        box = _reference_box()
        s = _test_state(p, box)
        f = O.compute_rhs(p, box, s.copy()).reshape(5, 3, 3, 3)[:, 1, 1, 1]
        c = O.ccz4_compute_rhs(p, box, O.ccz4_state(p, box, s)).reshape(
            5, 3, 3, 3)[:, 1, 1, 1]
        out.append((f, c))
    (f1, c1), (f0, c0) = out
    return np.max(np.abs((c1 - c0) - (f1 - f0)))


def test_ccz4_sources_converge_at_second_order():
    e1, e2 = _source_error(0.25), _source_error(0.125)
    print("source error at dx, dx/2:", e1, e2, "ratio", e1 / e2)
    assert e1 > 0.0 and 3.0 < e1 / e2 < 5.0


def test_ccz4_recovery_and_cfl_match_fixed_background():
    p = _params()
    box = O.make_box((6, 5, 4), lo=(18, 14, 9))
    s = _test_state(p, box)
    V = O.state_view(box, s)
    rng = np.random.default_rng(cases.SEED)
    V[O.TAU] *= 1.0 + 1e-3 * rng.uniform(-1, 1, V[O.TAU].shape)
    V[O.D] *= 1.0 + 1e-3 * rng.uniform(-1, 1, V[O.D].shape)
    s36 = O.ccz4_state(p, box, s)
    inv_f = O.max_inverse_dt(p, box, s.copy())
    inv_c = O.ccz4_max_inverse_dt(p, box, s36)
    assert abs(inv_c - inv_f) <= 1e-12 * inv_f
    ref = s.copy()
    d_f = O.recover_primitives(p, box, ref)
    d_c = O.ccz4_recover_primitives(p, box, s36)
    assert d_c.as_tuple() == d_f.as_tuple()
    got = s36[O.CCZ4_GRHD * box.comp_stride:]
    err = cases.rel_err(got.reshape(11, -1), ref.reshape(11, -1))
    assert np.all(err <= 1e-12), err
