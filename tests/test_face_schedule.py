"""The face pass's z-march length (grhd_face_zchunk, host only) against an
independent list-scheduling simulation: every block of the launch, in
launch order (the full z blocks of every 15 x 15-cell tile, then the short
last z row), starts on the resident slot that frees first and costs its
planes plus its two lead-in planes; the chosen length is the candidate of
32, 16, 8, 6, 4 planes whose launch finishes first (ties keep the longer
march).  Pinned beside it: the choices the measurements were taken with on
a B200 (148 SMs, two FP64 / three FP32 face blocks per SM)."""
import ctypes as C
import heapq

import numpy as np
import pytest

TILE = 15
CANDIDATES = (32, 16, 8, 6, 4)


def makespan(nx, ny, nz, z, slots):
    tiles = -(-nx // TILE) * -(-ny // TILE)
    costs = [z + 2] * (tiles * (nz // z))
    if nz % z:
        costs += [nz % z + 2] * tiles
    free = [0] * min(slots, max(len(costs), 1))
    heapq.heapify(free)
    end = 0
    for c in costs:
        t = heapq.heappop(free) + c
        end = max(end, t)
        heapq.heappush(free, t)
    return end


def choice(nx, ny, nz, slots):
    best, cost = None, None
    for z in CANDIDATES:
        m = makespan(nx, ny, nz, z, slots)
        if cost is None or m < cost:
            best, cost = z, m
    return best


@pytest.fixture(scope="module")
def lib():
    from grdzhadzha_b200 import _lib as L
    return L.load()


def zchunk(lib, nx, ny, nz, slots):
    out = C.c_int(0)
    assert lib.grhd_face_zchunk(nx, ny, nz, slots, C.byref(out)) == 0
    return out.value


def test_measured_choices(lib):
    fp64, fp32 = 2 * 148, 3 * 148
    # 256^3: 32-plane blocks (16 gave 5.24 ms per FP64 launch, 64 gave 5.66,
    # against 5.22)
    assert zchunk(lib, 256, 256, 256, fp64) == 32
    # 128^3: 32 planes would leave a 28-block second wave; a shorter march
    # removes that tail
    assert zchunk(lib, 128, 128, 128, fp64) == 6
    assert zchunk(lib, 128, 128, 128, fp32) == 8
    # the host-buffer wavefront's 11-plane chunks of a 256^3 grid
    assert zchunk(lib, 256, 256, 11, fp64) == 8


def test_matches_list_scheduling(lib):
    rng = np.random.default_rng(20261204)
    for _ in range(300):
        nx, ny = (int(v) for v in rng.integers(1, 300, 2))
        nz = int(rng.integers(1, 300))
        slots = int(rng.choice([1, 7, 148, 296, 444, 1000]))
        assert zchunk(lib, nx, ny, nz, slots) == choice(nx, ny, nz, slots), \
            (nx, ny, nz, slots)


def test_rejects_empty_boxes_and_no_slots(lib):
    out = C.c_int(0)
    for args in ((0, 8, 8, 296), (8, 8, 0, 296), (8, 8, 8, 0)):
        assert lib.grhd_face_zchunk(*args, C.byref(out)) != 0
