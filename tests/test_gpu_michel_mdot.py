"""The GPU's rest-mass accretion rate against the analytic Michel flux
(the pin of tests/test_oracle_michel_mdot.py, here on the product path:
GPU initial data from grhd_michel_initial_data, one grhd_compute_rhs of
the noise-free state per sphere, grhd_accretion).  Spheres R = 4, 6, 8, 12
on [-16, 16]^3 at n = 32, 64, 128, 256: Mdot -> -4 pi r_s^2 rho_s u_s at
second order in dx for every R (least-squares order of |error| against dx
over the four grids >= 1.7), and at 256^3 every R agrees with the analytic
rate to 4e-4."""
import numpy as np
import pytest

import cases
from test_oracle_michel_mdot import RADII, michel_exact

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_gpu_mdot_converges_to_the_michel_flux():
    from grdzhadzha_b200 import workloads as W
    exact = michel_exact()
    err = {}
    for n in (32, 64, 128, 256):
        op0, lv = W.michel(n, noise=0.0)
        for R in RADII:
            p = cases.oracle_params_of(op0)
            p.accretion_radius = R
            op = cases.gpu_operator(p)
            op.compute_rhs(lv.new_rhs(), lv)
            m, _ = op.accretion(reset=True)
            err[n, R] = m / exact - 1.0
            del op
        del lv, op0
        torch.cuda.empty_cache()
    print("GPU Mdot / exact - 1:", {k: f"{v:.2e}" for k, v in err.items()})
    ns = (32, 64, 128, 256)
    for R in RADII:
        # slope of log|error| against log dx
        order = np.polyfit(np.log([1.0 / n for n in ns]),
                           np.log([abs(err[n, R]) for n in ns]), 1)[0]
        print(f"R = {R}: order {order:.2f}")
        assert order >= 1.7, (R, order, err)
        assert abs(err[256, R]) <= 4e-4, (R, err[256, R])
