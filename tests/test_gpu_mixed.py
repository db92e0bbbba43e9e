"""Error of the mixed FP32/FP64 path against FP64 (new; no reference
counterpart: the reference is FP64 throughout).

The mixed path evaluates reconstruction, HLLE, metric and sources in FP32;
con2prim, the near-horizon metric, the volume-time source and the RK
accumulation stay FP64.  The bounds below are the stated error of each
result:
  * one RHS: per-component max|mixed - FP64| / max|FP64| <= 1e-4 (FP32
    face fluxes; the flux difference F(i+1/2) - F(i-1/2) and the
    flux/source balance of an equilibrium torus amplify FP32 rounding;
    measured on B200: D, S_i 1e-7 to 6e-6, tau up to 4.3e-5, where the
    tau RHS is a small residual of flux and source);
  * the rest-mass accretion rate through r = 6M of the Michel inflow after
    20 RK4 steps, and its time integral: <= 1e-6 relative (the target the
    mixed path is held to; measured 1e-9 and 3e-8);
  * the conserved state after 20 RK4 steps: <= 1e-6 of its scale.
"""
import numpy as np
import pytest

import cases
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["michel_c1", "torus_a09", "ksdisk",
                                  "pndisk", "fixedbg"])
def test_mixed_rhs_error(name):
    p, box, s, t = cases.CASES[name]()
    op = cases.gpu_operator(p, precision="mixed")
    lv = cases.gpu_level(box, s)
    rhs = lv.new_rhs()
    op.compute_rhs(rhs, lv, time=t)
    ref = O.compute_rhs(p, box, s.copy(), t)
    err = cases.rel_err(rhs.cpu().numpy().reshape(5, -1), ref.reshape(5, -1))
    print(f"mixed RHS error {name}: {err}")
    assert np.all(err <= 1e-4), err


def _run(p, box, s, precision, steps, R):
    p.accretion_radius = R
    op = cases.gpu_operator(p, precision=precision)
    lv = cases.gpu_level(box, s)
    op.accretion(reset=True)
    t, mi = 0.0, 0.0
    for _ in range(steps):
        dt, mi, _d = op.advance_rk4_cfl(lv, 0.25, time=t, max_inverse_dt=mi)
        t += dt
    mdot, integral = op.accretion()
    return lv.interior(slice(0, 5)).cpu().numpy(), mdot, integral, t


def test_mixed_accretion_rate_error():
    p, box, s, _ = cases.michel_c1(n=32)
    u64, m64, i64, t64 = _run(p, box, s, "fp64", 20, 6.0)
    p, box, s, _ = cases.michel_c1(n=32)
    u32, m32, i32, t32 = _run(p, box, s, "mixed", 20, 6.0)
    assert abs(t32 - t64) <= 1e-6 * t64
    em = abs(m32 - m64) / abs(m64)
    ei = abs(i32 - i64) / abs(i64)
    eu = cases.rel_err(u32 - O.interior(box, s), u64 - O.interior(box, s))
    print(f"mixed vs FP64 after 20 RK4 steps: Mdot {em:.2e}, "
          f"integral {ei:.2e}, state increment {eu}")
    assert em <= 1e-6 and ei <= 1e-6
    assert np.all(cases.rel_err(u32, u64) <= 1e-6)
