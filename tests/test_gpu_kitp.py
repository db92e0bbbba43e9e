"""Source terms of the binary-PN disk production driver
(Examples/GRHDLevelDataBinaryPNKITPDisk/Main_GRHDLevelDataBinaryPNKITPDisk.cpp)
on the GPU against the oracle's restatement: the alpha-viscosity stress
divergence (:676-806), the sink right-hand side (:567-610) and the sink
decay (:612-662), on the binary-PN disk of Examples/GRHDLevelDataBinaryPNDisk
(56^2 x 9).  Per component, max|GPU - oracle| <= 1e-12 of max|oracle|
(the device's exp / pow / division round differently from libm's)."""
import numpy as np
import pytest

import cases
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

# sinks 20 M^-1 wide so that they reach the disk (the driver's default
# width keeps them at the bodies, inside the disk's cavity)
CFG = dict(alpha_viscosity=0.03, viscosity_beta=0.2, rho_floor=1e-10,
           sink_size=20.0, sink_rate=1.0, sink_shape=4.0)


def _setup(time=0.7):
    from grdzhadzha_b200.operator import kitp_config
    p, box, s, _ = cases.CASES["pndisk"]()
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, s)
    return p, box, s, op, lv, kitp_config(**CFG), O.kitp_config(**CFG), time


def test_viscous_rhs_matches_oracle():
    p, box, s, op, lv, cfg, ocfg, t = _setup()
    rhs = lv.new_rhs()
    rhs.fill_(0.5)
    op.kitp_viscous_rhs(rhs, lv, cfg, time=t)
    ref = np.full(5 * O.interior_cells(box), 0.5)
    O.kitp_viscous_rhs(p, ocfg, box, s, ref, t)
    got = rhs.cpu().numpy().reshape(5, -1) - 0.5
    want = ref.reshape(5, -1) - 0.5
    assert np.abs(want[1:3]).max() > 0.0 and np.abs(want[4]).max() > 0.0
    err = cases.rel_err(got, want)
    assert np.all(err[1:] <= 1e-12), err


def test_sink_rhs_and_decay_match_oracle():
    p, box, s, op, lv, cfg, ocfg, t = _setup()
    rhs = lv.new_rhs()
    op.kitp_sink_rhs(rhs, lv, cfg, time=t)
    ref = np.zeros(5 * O.interior_cells(box))
    O.kitp_sink_rhs(p, ocfg, box, s, ref, t)
    assert np.abs(ref).max() > 0.0
    err = cases.rel_err(rhs.cpu().numpy().reshape(5, -1), ref.reshape(5, -1))
    assert np.all(err <= 1e-12), err
    dt = 0.05
    op.kitp_sink_decay(lv, t + 0.5 * dt, dt, cfg)
    ref_state = s.copy()
    O.kitp_sink_decay(p, ocfg, box, ref_state, t + 0.5 * dt, dt)
    got = O.interior(box, lv.state.cpu().numpy().reshape(-1))
    want = O.interior(box, ref_state)
    assert not np.array_equal(want, O.interior(box, s))
    err = cases.rel_err(got, want)
    assert np.all(err <= 1e-12), err


def test_requires_binary_background():
    from grdzhadzha_b200 import InvalidArgument
    p, box, s, t = cases.CASES["fixedbg"]()
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, s)
    with pytest.raises(InvalidArgument):
        op.kitp_sink_decay(lv, 0.0, 0.1)
