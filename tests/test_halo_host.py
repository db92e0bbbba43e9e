"""Host logic of a level split over ranks (grdzhadzha_b200.halo), on CPU.

The reference's multi-rank runs (2 MPI ranks over an x-split layout,
Tests/GRHDLevelDataMichelAccretion/GRHDLevelDataMichelAccretion.cpp:
375-401) check the exchange by poisoning the internal ghosts
(Tests/GRHDLevelDataBinaryPNSmoke/GRHDLevelDataBinaryPNSmoke.cpp:204-235).
Here:
  * the halo plan of every rank, for slab and pencil cuts (slabs thinner
    than the ghost width included), receives every in-domain ghost cell
    exactly once and from its owner, and p's send to q is q's receive
    from p;
  * world-size 2 and 3 gloo process groups run HaloExchange over
    TorchTransport: ghosts poisoned with NaN, interiors holding a known
    function of (component, cell); after the exchange every in-domain
    ghost holds its owner's value and the outflow ghosts are untouched;
    the MAX and SUM reductions give the level's values.
The device pack / unpack (grhd_region_copy) is replaced by a host
restatement of the same buffer layout ([component][k][j][i]), since there
is no GPU here; the GPU tests drive the device one.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from grdzhadzha_b200 import halo as H  # noqa: E402

DOMAIN_LO, DOMAIN_HI = (0, 0, 0), (9, 7, 12)


def _ghost_cells(lo, hi, g=2):
    return {(i, j, k)
            for k in range(lo[2] - g, hi[2] + g + 1)
            for j in range(lo[1] - g, hi[1] + g + 1)
            for i in range(lo[0] - g, hi[0] + g + 1)
            if not (lo[0] <= i <= hi[0] and lo[1] <= j <= hi[1]
                    and lo[2] <= k <= hi[2])}


def _cells(lo, hi):
    return {(i, j, k) for k in range(lo[2], hi[2] + 1)
            for j in range(lo[1], hi[1] + 1)
            for i in range(lo[0], hi[0] + 1)}


def _in_domain(c):
    return all(DOMAIN_LO[d] <= c[d] <= DOMAIN_HI[d] for d in range(3))


LAYOUTS = {
    "slabs2": H.slab_boxes(DOMAIN_LO, DOMAIN_HI, 2),
    "slabs3": H.slab_boxes(DOMAIN_LO, DOMAIN_HI, 3),
    # 13 cells into 12 slabs: one-cell slabs, ghosts from two ranks away
    "thin_slabs": H.slab_boxes(DOMAIN_LO, DOMAIN_HI, 12),
    "pencils2x2": H.pencil_boxes(DOMAIN_LO, DOMAIN_HI, 2, 2),
    "pencils3x2": H.pencil_boxes(DOMAIN_LO, DOMAIN_HI, 3, 2),
}


@pytest.mark.parametrize("name", list(LAYOUTS))
def test_halo_plan_receives_every_ghost_once(name):
    boxes = LAYOUTS[name]
    owned = set()
    for lo, hi in boxes:
        c = _cells(lo, hi)
        assert not (owned & c), "boxes overlap"
        owned |= c
    assert owned == _cells(DOMAIN_LO, DOMAIN_HI)
    plans = [H.halo_plan(boxes, r, DOMAIN_LO, DOMAIN_HI)
             for r in range(len(boxes))]
    for r, (lo, hi) in enumerate(boxes):
        sends, recvs = plans[r]
        got = {}
        for peer, rlo, rhi in recvs:
            for c in _cells(rlo, rhi):
                assert c not in got, f"ghost {c} received twice"
                got[c] = peer
        want = {c for c in _ghost_cells(lo, hi) if _in_domain(c)}
        assert set(got) == want
        for c, peer in got.items():
            plo, phi = boxes[peer]
            assert all(plo[d] <= c[d] <= phi[d] for d in range(3))
        for peer, slo, shi in sends:
            back = [x for x in plans[peer][1] if x[0] == r]
            assert back == [(r, slo, shi)]


def test_split_rejects_too_many_parts():
    with pytest.raises(ValueError):
        H.slab_boxes(DOMAIN_LO, DOMAIN_HI, 14)


class HostRegions:
    """pack / unpack over a CPU state tensor in the device layout."""

    @staticmethod
    def _view(level, lo, hi):
        g = level.ghost
        sl = tuple(slice(lo[d] - (level.lo[d] - g), hi[d] + 1 - (level.lo[d] - g))
                   for d in (2, 1, 0))
        return level.state[(slice(None),) + sl]

    def pack(self, level, lo, hi, buf):
        buf.copy_(self._view(level, lo, hi).reshape(-1))

    def unpack(self, level, lo, hi, buf):
        v = self._view(level, lo, hi)
        v.copy_(buf.view(v.shape))


def _value(c, i, j, k):
    return 1.0e6 * c + i + 100.0 * j + 10000.0 * k


def _worker(rank, world, port, layout, result_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(
                                seconds=60))
    try:
        from grdzhadzha_b200 import halo as Hw
        from grdzhadzha_b200.operator import LevelBox
        boxes = LAYOUTS[layout]
        lo, hi = boxes[rank]
        lv = LevelBox(lo=lo, hi=hi, ghost=2, domain_lo=DOMAIN_LO,
                      domain_hi=DOMAIN_HI, device="cpu")
        lv.state.fill_(float("nan"))
        g = 2
        for (i, j, k) in _cells(lo, hi):
            for c in range(11):
                lv.state[c, k - lo[2] + g, j - lo[1] + g, i - lo[0] + g] = \
                    _value(c, i, j, k)
        ex = Hw.HaloExchange(boxes, rank, DOMAIN_LO, DOMAIN_HI,
                             Hw.TorchTransport(), HostRegions())
        ex.exchange(lv)
        ex.exchange(lv)  # buffers are reused on the second exchange
        bad = []
        for (i, j, k) in _ghost_cells(lo, hi):
            got = lv.state[:, k - lo[2] + g, j - lo[1] + g, i - lo[0] + g]
            if _in_domain((i, j, k)):
                want = torch.tensor([_value(c, i, j, k) for c in range(11)],
                                    dtype=torch.float64)
                if not torch.equal(got, want):
                    bad.append((i, j, k))
            elif not torch.isnan(got).all():
                bad.append(("outflow ghost written", i, j, k))
        tr = Hw.TorchTransport()
        mx = tr.all_reduce(float(rank), "max", "cpu")
        sm = tr.all_reduce(float(rank + 1), "sum", "cpu")
        with open(os.path.join(result_dir, f"r{rank}.txt"), "w") as f:
            f.write(f"{len(bad)} {mx} {sm} {bad[:3]}\n")
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("layout,world", [("slabs2", 2), ("slabs3", 3),
                                          ("pencils2x2", 4)])
def test_gloo_halo_exchange(layout, world, tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), layout,
                                      str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        n, mx, sm, bad = open(tmp_path / f"r{r}.txt").read().split(" ", 3)
        assert int(n) == 0, bad
        assert float(mx) == world - 1
        assert float(sm) == world * (world + 1) / 2
