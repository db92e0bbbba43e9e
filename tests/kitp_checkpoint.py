"""An independent numpy implementation of the KITPCHK1 checkpoint layout of
Examples/GRHDLevelDataBinaryPNKITPDisk/Main_GRHDLevelDataBinaryPNKITPDisk.cpp
(write_checkpoint :1385-1505, read_checkpoint_header :1289-1345,
checkpoint_value_index :1347-1356), used by the tests to check the
library's reader and writer against the reference's byte layout."""
from __future__ import annotations

import struct

import numpy as np

HEADER_FMT = "<8sIiiiiiiddd4Q7d3Q"


def write(path, header: dict, signature: str, values: np.ndarray):
    """values: (nz+2g, ny+2g, nx+2g, ncomp) float64, the interleaved
    state over the storage box."""
    h = header
    head = struct.pack(
        HEADER_FMT, b"KITPCHK1", 1, h["num_components"], h["num_cells"],
        h["num_z_cells"], h["num_ghosts"], h["steps"], h["frame_index"],
        h["time"], h["next_output_time"], h["next_checkpoint_time"],
        *h["recovery_totals"], *h["diagnostics"], *h["diagnostic_counts"])
    sig = signature.encode()
    with open(path, "wb") as f:
        f.write(head)
        f.write(struct.pack("<Q", len(sig)))
        f.write(sig)
        f.write(struct.pack("<Q", values.size))
        f.write(np.ascontiguousarray(values, dtype="<f8").tobytes())


def read(path):
    """(header dict, signature, values (nz+2g, ny+2g, nx+2g, ncomp))."""
    data = open(path, "rb").read()
    n = struct.calcsize(HEADER_FMT)
    f = struct.unpack(HEADER_FMT, data[:n])
    assert f[0] == b"KITPCHK1" and f[1] == 1
    h = {"num_components": f[2], "num_cells": f[3], "num_z_cells": f[4],
         "num_ghosts": f[5], "steps": f[6], "frame_index": f[7],
         "time": f[8], "next_output_time": f[9],
         "next_checkpoint_time": f[10], "recovery_totals": list(f[11:15]),
         "diagnostics": list(f[15:22]), "diagnostic_counts": list(f[22:25])}
    (slen,) = struct.unpack("<Q", data[n:n + 8])
    sig = data[n + 8:n + 8 + slen].decode()
    off = n + 8 + slen
    (count,) = struct.unpack("<Q", data[off:off + 8])
    vals = np.frombuffer(data[off + 8:off + 8 + 8 * count], dtype="<f8")
    g = h["num_ghosts"]
    shape = (h["num_z_cells"] + 2 * g, h["num_cells"] + 2 * g,
             h["num_cells"] + 2 * g, h["num_components"])
    assert vals.size == np.prod(shape)
    return h, sig, vals.reshape(shape)
