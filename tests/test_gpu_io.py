"""Diagnostics and KITPCHK1 checkpoints through the C ABI on the GPU.

* grhd_disk_diagnostics equals the oracle's compute_diagnostics
  restatement on the Kerr-Schild disk (sums to 1e-13 relative: another
  summation order; maxima exactly);
* a checkpoint written from the device state has the reference's byte
  layout (read back by an independent implementation of that layout:
  header fields, signature, the 11 GRHD components last in each cell's
  record of NUM_VARS values, the CCZ4 slots zero);
* a checkpoint in that layout restores the device state exactly, and a
  wrong signature or grid is refused with the reference's message."""
import numpy as np
import pytest

import cases
import kitp_checkpoint as K
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_disk_diagnostics_match_oracle():
    p, box, s, t = cases.CASES["ksdisk"]()
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, s)
    got = np.array(op.disk_diagnostics(lv, time=t))
    want = O.disk_diagnostics(p, box, list(box.lo), list(box.hi), s, t)
    assert np.all(np.abs(got[:3] - want[:3]) <= 1e-13 * np.abs(want[:3]))
    assert np.array_equal(got[3:], want[3:])


def _header(n, nz, g, ncomp=36):
    from grdzhadzha_b200 import _lib as L
    h = L.CheckpointHeader()
    h.num_components, h.num_cells, h.num_z_cells, h.num_ghosts = ncomp, n, nz, g
    h.steps, h.frame_index = 40, 4
    h.time, h.next_output_time, h.next_checkpoint_time = 2.0, 2.5, 50.0
    for q in range(4):
        h.recovery_totals[q] = 100 + q
    for q in range(7):
        h.diagnostics[q] = 0.1 * (q + 1)
    for q in range(3):
        h.diagnostic_counts[q] = q
    return h


def test_checkpoint_write_has_reference_layout(tmp_path):
    from grdzhadzha_b200 import io
    p, box, s, t = cases.CASES["pndisk"]()
    lv = cases.gpu_level(box, s)
    nx = box.hi[0] - box.lo[0] + 1
    nz = box.hi[2] - box.lo[2] + 1
    sig = io.config_signature(num_cells=nx, num_z_cells=nz)
    path = str(tmp_path / "checkpoint_step_00000040.bin")
    io.write_checkpoint(path, lv, _header(nx, nz, 2), sig)
    h, fsig, vals = K.read(path)
    assert fsig == sig
    assert (h["num_components"], h["num_cells"], h["num_z_cells"],
            h["num_ghosts"], h["steps"], h["frame_index"]) == (36, nx, nz, 2,
                                                              40, 4)
    assert h["recovery_totals"] == [100, 101, 102, 103]
    assert h["diagnostic_counts"] == [0, 1, 2]
    state = lv.state.cpu().numpy()  # (11, z, y, x)
    assert np.array_equal(vals[..., 25:], np.moveaxis(state, 0, -1))
    assert not vals[..., :25].any()


def test_checkpoint_read_restores_state(tmp_path):
    from grdzhadzha_b200 import io
    p, box, s, t = cases.CASES["pndisk"]()
    lv = cases.gpu_level(box, s)
    nx = box.hi[0] - box.lo[0] + 1
    nz = box.hi[2] - box.lo[2] + 1
    g = 2
    state = lv.state.cpu().numpy()
    vals = np.zeros(state.shape[1:] + (36,))
    vals[..., 25:] = np.moveaxis(state, 0, -1) * 1.5
    vals[..., :25] = 7.0  # CCZ4 slots: ignored
    hdr = {"num_components": 36, "num_cells": nx, "num_z_cells": nz,
           "num_ghosts": g, "steps": 9, "frame_index": 1, "time": 0.75,
           "next_output_time": 1.0, "next_checkpoint_time": 50.0,
           "recovery_totals": [1, 2, 3, 4], "diagnostics": [0.5] * 7,
           "diagnostic_counts": [7, 8, 9]}
    sig = io.config_signature(num_cells=nx, num_z_cells=nz)
    path = str(tmp_path / "ref.bin")
    K.write(path, hdr, sig, vals)
    out = cases.gpu_level(box, np.zeros_like(s))
    h = io.read_checkpoint(path, out, expected_signature=sig)
    assert (h.steps, h.time, h.recovery_totals[3]) == (9, 0.75, 4)
    assert np.array_equal(out.state.cpu().numpy(), state * 1.5)
    with pytest.raises(io.CheckpointError, match="configuration does not"):
        io.read_checkpoint(path, out, expected_signature=sig + " 1")
    small = cases.gpu_level(*cases.CASES["michel18"]()[1:3:1])
    with pytest.raises(io.CheckpointError, match="grid does not match"):
        io.read_checkpoint(path, small, expected_signature=sig)
