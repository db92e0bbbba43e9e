"""The example drivers' on-disk formats, host side (no GPU): the
configuration signature and diagnostics CSV row as the reference's
std::ostream (setprecision 17) prints them, and the independent KITPCHK1
layout implementation the GPU checkpoint tests use."""
import numpy as np

import kitp_checkpoint as K
from grdzhadzha_b200 import io


def test_signature_formats_like_ostream():
    sig = io.config_signature(num_cells=64, num_z_cells=9,
                              use_reconstruction=False)
    f = sig.split(" ")
    assert len(f) == len(io.SIGNATURE_FIELDS) == 33
    assert f[:3] == ["64", "9", "2"]          # ints as ints
    assert f[3] == "96"                       # 96.0 prints without a point
    assert f[5] == "0.14000000000000001"     # 17 significant digits
    assert f[18] == "1.0000000000000001e-05"  # two-digit exponent
    assert f[19] == "10000000000"             # 1e10 below 17 digits: fixed
    assert f[25:28] == ["0", "1", "1"]        # bools as 0 / 1


def test_diagnostics_row_columns():
    row = io.diagnostics_row(7, 0.5, [1.0, 0.25, 3.0, 1e-5, 2e-8, 0.3,
                                      1.05], [1, 2, 3])
    assert row == ("7,0.5,1,0.25,3,1.0000000000000001e-05,2e-08,"
                   "0.29999999999999999,1.05,1,2,3\n")


def test_checkpoint_layout_round_trip(tmp_path):
    h = {"num_components": 36, "num_cells": 6, "num_z_cells": 3,
         "num_ghosts": 2, "steps": 12, "frame_index": 3, "time": 1.25,
         "next_output_time": 1.5, "next_checkpoint_time": 2.0,
         "recovery_totals": [10, 1, 2, 3], "diagnostics": [1.0] * 7,
         "diagnostic_counts": [4, 5, 6]}
    vals = np.random.default_rng(1).random((7, 10, 10, 36))
    path = tmp_path / "c.bin"
    K.write(path, h, io.config_signature(), vals)
    h2, sig, v2 = K.read(path)
    assert h2 == h and sig == io.config_signature()
    assert np.array_equal(v2, vals)
