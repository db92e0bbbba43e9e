"""The sm_100a operator (through the C ABI) against GRDzhadzha's own
operator: the reference's headers compiled unmodified against oracle/shim
(oracle/_ref/libref_grhd.so, built where the reference tree is available
and shipped with the other built libraries).  The same tolerances as the
oracle parity tests (the restatement equals the reference bit for bit,
tests/test_oracle_reference.py): one RHS evaluation per conserved component
max|gpu - ref| / max|ref| <= 1e-12 (Tests/GRHDFixedBGTest/
GRHDFixedBGTest.cpp:419-421), the physical ghost fill to 1e-13, one SSPRK2
step's increment to 1e-11 and its conserved state to 1e-13 of scale.  The
reference has no excision; the fixtures that use it run without it.

Also the KITP disk driver itself (oracle/_ref/GRHDLevelDataBinaryPNKITPDisk,
run here): the product reads its KITPCHK1 checkpoint and writes the same
bytes back, and the device's driver step from its first checkpoint meets
its second."""
import os

import numpy as np
import pytest

import cases
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.have_ref(),
                                 reason="reference build absent")]


def _case(name):
    p, box, s, t = cases.CASES[name]()
    p.excision_radius = 0.0
    p.accretion_radius = 0.0
    return p, box, s, t


@pytest.mark.parametrize("name", ["fixedbg", "ksdisk", "pndisk", "michel18",
                                  "torus_a09"])
def test_compute_rhs_matches_reference(name):
    p, box, s, t = _case(name)
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, s)
    rhs = lv.new_rhs()
    op.compute_rhs(rhs, lv, time=t)
    ref_state = s.copy()
    ref = O.ref_compute_rhs(p, box, ref_state, t)
    err = cases.rel_err(rhs.cpu().numpy().reshape(5, -1), ref.reshape(5, -1))
    print(f"{name}: GPU vs reference RHS {err}")
    assert np.all(err <= 1e-12), err
    g = cases.rel_err(lv.state.cpu().numpy().reshape(11, -1)[:5],
                      ref_state.reshape(11, -1)[:5])
    assert np.all(g <= 1e-13), g


@pytest.mark.parametrize("name", ["ksdisk", "pndisk", "michel18"])
def test_ssprk2_step_matches_reference(name):
    p, box, s, t = _case(name)
    dt = 0.5 * 0.25 / O.ref_max_inverse_dt(p, box, s.copy(), t)
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, s)
    assert op.compute_max_inverse_dt(lv, time=t) == pytest.approx(
        O.ref_max_inverse_dt(p, box, s.copy(), t), rel=1e-13)
    op.advance_ssprk2(lv, time=t, dt=dt)
    ref = s.copy()
    O.ref_advance_ssprk2(p, box, ref, t, dt)
    got = lv.interior().cpu().numpy()
    want = O.interior(box, ref, slice(0, 11))
    inc = cases.rel_err(got[:5] - O.interior(box, s),
                        want[:5] - O.interior(box, s))
    full = cases.rel_err(got[:5], want[:5])
    print(f"{name}: SSPRK2 increment {inc}, state {full}")
    assert np.all(inc <= 1e-11), inc
    assert np.all(full <= 1e-13), full


# ---- the KITP disk driver's own run on the device ----

def _kitp_case(tmp_path):
    import test_oracle_reference as TR
    if not os.path.exists(os.path.join(O.REF_DIR, TR.KITP_DRIVER)):
        pytest.skip("reference KITP driver not built")
    paths = TR.run_kitp_driver(tmp_path)
    p = TR.kitp_driver_params()
    box = O.make_box((TR.KITP_N, TR.KITP_N, TR.KITP_NZ))
    return TR, paths, p, box


def test_reference_checkpoint_round_trips_through_the_device(tmp_path):
    """The product reads the checkpoint the reference driver wrote (header,
    signature and the GRHD components of every stored cell, bit for bit)
    and writes the same state back as the same bytes."""
    import kitp_checkpoint as KC
    from grdzhadzha_b200 import io
    TR, paths, p, box = _kitp_case(tmp_path)
    h, sig, v = KC.read(paths[1])
    lv = cases.gpu_level(box, O.new_state(box))
    hdr = io.read_checkpoint(paths[1], lv, expected_signature=sig)
    assert (hdr.steps, hdr.time, list(hdr.recovery_totals)) == \
        (h["steps"], h["time"], h["recovery_totals"])
    assert np.array_equal(np.moveaxis(lv.state.cpu().numpy(), 0, -1),
                          v[..., 25:36])
    out = str(tmp_path / "rewritten.bin")
    io.write_checkpoint(out, lv, hdr, sig)
    assert open(out, "rb").read() == open(paths[1], "rb").read()


def test_kitp_driver_step_on_the_device_matches_the_reference(tmp_path):
    """From the reference driver's first checkpoint, the driver's next step
    on the device (recovery, stable dt, grhd_kitp_advance_ssprk2, recovery)
    against its second checkpoint: the step's change of the conserved
    state within 1e-11 of its scale and the state within 1e-13 (the
    tolerance of the operator's own step parity tests)."""
    import kitp_checkpoint as KC
    from grdzhadzha_b200 import io
    from grdzhadzha_b200.operator import kitp_config
    TR, paths, p, box = _kitp_case(tmp_path)
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, O.new_state(box))
    h1 = io.read_checkpoint(paths[0], lv)
    start = lv.interior(slice(0, 5)).cpu().numpy()
    t = h1.time
    op.recover_primitives(lv, time=t)
    stable = 0.14 / op.compute_max_inverse_dt(lv, time=t)
    dt = min(stable, 0.02, 0.06 - t, 0.5 - t, h1.next_checkpoint_time - t)
    op.kitp_advance_ssprk2(lv, t, dt, kitp_config())
    op.recover_primitives(lv, time=t + dt)
    h2, sig, v = KC.read(paths[1])
    assert t + dt == h2["time"]
    want = np.moveaxis(v[2:-2, 2:-2, 2:-2, 25:30], -1, 0)
    got = lv.interior(slice(0, 5)).cpu().numpy()
    inc = cases.rel_err((got - start).reshape(5, -1),
                        (want - start).reshape(5, -1))
    full = cases.rel_err(got.reshape(5, -1), want.reshape(5, -1))
    print("KITP driver step, device vs reference: increment", inc,
          "state", full)
    assert np.all(inc <= 1e-11), inc
    assert np.all(full <= 1e-13), full
