"""A single level split over ranks: one box per rank, the ghost exchange
between ranks, the global CFL bound and the SSPRK2 step.

The reference runs a level as a Chombo DisjointBoxLayout over MPI ranks;
`LevelData<FArrayBox>::exchange()` moves the 2-cell halos before every
directional RHS and before the sources (FixedBGFArrayBoxFiniteVolume.hpp:
310, 355), and the level's CFL bound is a reduction over ranks
(compute_leveldata_max_inverse_dt_from_fixed_background).  Here each rank
(one process per GPU) holds one LevelBox of the level:

  * `slab_boxes` / `pencil_boxes` cut the domain (z slabs, or x-y pencils
    for wide domains), the same on every rank;
  * `halo_plan` lists, for one rank, the regions it sends (its interior
    cells inside another box's in-domain ghosts) and the regions it
    receives (its in-domain ghosts inside another box's interior), in one
    order that every rank derives alike;
  * `HaloExchange` packs each send region into a contiguous device buffer
    (grhd_region_copy), posts all sends and receives as one batch of
    point-to-point operations (torch.distributed: NCCL over NVLink between
    GPUs, gloo on CPU), waits and unpacks.  `begin` / `end` split the two
    halves so that several virtual ranks can be driven in one process;
  * `DistributedLevel` puts the operator's methods on top: compute_rhs
    (exchange, then the box's RHS), compute_stable_dt (all-reduce MAX of
    the inverse dt), advance_ssprk2 (the reference's sequence with an
    exchange before each of its two RHS evaluations, grhd_ssprk2_stage).

Only the halo moves between ranks; the physical (outflow) ghosts are filled
by each box itself.  No kernel waits on another rank: the exchange is
ordered on the host by the batch's wait.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L
from .operator import LevelBox, _ptr, _stream

GHOST = 2


def _split(lo, hi, parts):
    n = hi - lo + 1
    if parts < 1 or parts > n:
        raise ValueError(f"cannot cut {n} cells into {parts} parts")
    return [(lo + (n * q) // parts, lo + (n * (q + 1)) // parts - 1)
            for q in range(parts)]


def slab_boxes(domain_lo, domain_hi, parts):
    """z slabs of (nearly) equal thickness, rank q holding slab q."""
    return [((domain_lo[0], domain_lo[1], zl), (domain_hi[0], domain_hi[1], zh))
            for zl, zh in _split(domain_lo[2], domain_hi[2], parts)]


def pencil_boxes(domain_lo, domain_hi, px, py):
    """x-y pencils (full z), rank q = qy * px + qx."""
    xs = _split(domain_lo[0], domain_hi[0], px)
    ys = _split(domain_lo[1], domain_hi[1], py)
    return [((xl, yl, domain_lo[2]), (xh, yh, domain_hi[2]))
            for yl, yh in ys for xl, xh in xs]


def _intersect(alo, ahi, blo, bhi):
    lo = tuple(max(alo[d], blo[d]) for d in range(3))
    hi = tuple(min(ahi[d], bhi[d]) for d in range(3))
    return (lo, hi) if all(lo[d] <= hi[d] for d in range(3)) else None


def _ghost_region(lo, hi, domain_lo, domain_hi, ghost):
    """The ghosted box clipped to the domain."""
    return (tuple(max(lo[d] - ghost, domain_lo[d]) for d in range(3)),
            tuple(min(hi[d] + ghost, domain_hi[d]) for d in range(3)))


def halo_plan(boxes, rank, domain_lo, domain_hi, ghost=GHOST):
    """(sends, recvs) of `rank`: lists of (peer, lo, hi), sorted by peer.

    A send is the part of this rank's interior inside the peer's
    in-domain ghosted box; a receive the part of this rank's in-domain
    ghosted box inside the peer's interior (corners included, as Chombo's
    default copier).  The send of p to q and the receive of q from p are
    the same region, so both ranks size their buffers alike."""
    lo, hi = boxes[rank]
    glo, ghi = _ghost_region(lo, hi, domain_lo, domain_hi, ghost)
    sends, recvs = [], []
    for peer, (plo, phi) in enumerate(boxes):
        if peer == rank:
            continue
        pglo, pghi = _ghost_region(plo, phi, domain_lo, domain_hi, ghost)
        r = _intersect(lo, hi, pglo, pghi)
        if r:
            sends.append((peer,) + r)
        r = _intersect(glo, ghi, plo, phi)
        if r:
            recvs.append((peer,) + r)
    return sends, recvs


def region_cells(lo, hi):
    return (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1)


class DeviceRegions:
    """Region pack / unpack on the device (grhd_region_copy); the state
    and the buffers are CUDA float64 tensors (anything else raises)."""

    def __init__(self):
        self._lib = L.load()

    def _copy(self, pack, level: LevelBox, lo, hi, buf: torch.Tensor):
        b = level.c_box()
        st = self._lib.grhd_region_copy_components(
            int(pack), _ptr(level.state), level.comp_stride(), C.byref(b),
            (C.c_int * 3)(*lo), (C.c_int * 3)(*hi),
            int(level.state.shape[0]), _ptr(buf), _stream())
        if st != L.GRHD_OK:
            raise L.InvalidArgument(st, None) \
                if st == L.GRHD_ERR_INVALID_ARG else L.GRHDError(st, None)

    def pack(self, level, lo, hi, buf):
        self._copy(True, level, lo, hi, buf)

    def unpack(self, level, lo, hi, buf):
        self._copy(False, level, lo, hi, buf)


class TorchTransport:
    """Point-to-point messages and reductions over a torch.distributed
    process group (NCCL between GPUs; gloo for CPU tensors)."""

    def __init__(self, group=None):
        self.group = group

    def start(self, sends, recvs):
        import torch.distributed as dist
        ops = [dist.P2POp(dist.isend, t, peer, self.group)
               for peer, t in sends]
        ops += [dist.P2POp(dist.irecv, t, peer, self.group)
                for peer, t in recvs]
        return dist.batch_isend_irecv(ops) if ops else []

    def wait(self, handle):
        for req in handle:
            req.wait()

    def all_reduce(self, value: float, op: str, device) -> float:
        import torch.distributed as dist
        t = torch.tensor([value], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max"
                        else dist.ReduceOp.SUM, group=self.group)
        return float(t.item())


class LocalTransport:
    """The ranks of a level driven one after another in one process (a
    level of several boxes without a process group, and tests): messages
    go through a mailbox shared by the ranks' transports; every rank's
    `begin` must come before any rank's `end`."""

    def __init__(self, mailbox: dict, rank: int):
        self.mailbox = mailbox
        self.rank = rank

    def start(self, sends, recvs):
        for peer, t in sends:
            key = (self.rank, peer)
            if key in self.mailbox:
                raise RuntimeError(f"message {key} posted twice")
            self.mailbox[key] = t
        return recvs

    def wait(self, recvs):
        for peer, t in recvs:
            key = (peer, self.rank)
            if key not in self.mailbox:
                raise RuntimeError(f"message {key} never posted")
            t.copy_(self.mailbox.pop(key))

    def all_reduce(self, value, op, device):
        raise RuntimeError("LocalTransport has no reduction; reduce over "
                           "the ranks' values on the host")


class HaloExchange:
    """LevelData::exchange() of one rank's box: pack the send regions,
    move them, unpack the receive regions."""

    def __init__(self, boxes, rank, domain_lo, domain_hi, transport,
                 regions=None, ghost=GHOST):
        self.rank = rank
        self.sends, self.recvs = halo_plan(boxes, rank, domain_lo,
                                           domain_hi, ghost)
        self.transport = transport
        self.regions = regions if regions is not None else DeviceRegions()
        self._bufs = None
        self._pending = None

    def _buffers(self, device, ncomp=11):
        if self._bufs is None or self._bufs[0] != (device, ncomp):
            def mk(plan):
                return [torch.empty(ncomp * region_cells(lo, hi),
                                    dtype=torch.float64, device=device)
                        for _, lo, hi in plan]
            self._bufs = ((device, ncomp), mk(self.sends), mk(self.recvs))
        return self._bufs[1], self._bufs[2]

    def bytes_per_exchange(self, ncomp=11) -> int:
        """Bytes this rank sends per exchange of an ncomp-component state."""
        return 8 * ncomp * sum(region_cells(lo, hi)
                               for _, lo, hi in self.sends)

    def begin(self, level: LevelBox):
        if self._pending is not None:
            raise RuntimeError("exchange already in flight")
        sbufs, rbufs = self._buffers(level.state.device,
                                     int(level.state.shape[0]))
        for (_, lo, hi), buf in zip(self.sends, sbufs):
            self.regions.pack(level, lo, hi, buf)
        self._pending = self.transport.start(
            [(peer, buf) for (peer, _, _), buf in zip(self.sends, sbufs)],
            [(peer, buf) for (peer, _, _), buf in zip(self.recvs, rbufs)])

    def end(self, level: LevelBox):
        if self._pending is None:
            raise RuntimeError("no exchange in flight")
        self.transport.wait(self._pending)
        self._pending = None
        _, rbufs = self._buffers(level.state.device,
                                 int(level.state.shape[0]))
        for (_, lo, hi), buf in zip(self.recvs, rbufs):
            self.regions.unpack(level, lo, hi, buf)

    def exchange(self, level: LevelBox):
        self.begin(level)
        self.end(level)


class DistributedLevel:
    """One rank's share of a level: its LevelBox (state and the SSPRK2
    stage buffer), its halo exchange and the operator's level methods.

    op: a FixedBG / TimeDependentFixedBG operator; boxes: the level's
    boxes (the same list on every rank, e.g. slab_boxes); transport:
    TorchTransport (default) or LocalTransport.  For the operator on
    CCZ4-stored geometry, drive a HaloExchange over its 36-component
    LevelBoxes and its ssprk2_stage directly (the exchange moves every
    component the state holds)."""

    def __init__(self, op, boxes, rank, domain_lo, domain_hi,
                 transport=None, device="cuda", regions=None):
        lo, hi = boxes[rank]
        self.op = op
        self.rank = rank
        self.boxes = list(boxes)
        self.state = LevelBox(lo=tuple(lo), hi=tuple(hi), ghost=GHOST,
                              domain_lo=tuple(domain_lo),
                              domain_hi=tuple(domain_hi), device=device)
        self.stage = LevelBox(lo=tuple(lo), hi=tuple(hi), ghost=GHOST,
                              domain_lo=tuple(domain_lo),
                              domain_hi=tuple(domain_hi), device=device)
        self.transport = transport if transport is not None \
            else TorchTransport()
        self.halo = HaloExchange(self.boxes, rank, domain_lo, domain_hi,
                                 self.transport, regions)

    def exchange(self):
        self.halo.exchange(self.state)

    def compute_rhs(self, rhs, inverse_dx_U=None, time=0.0):
        """compute_rhs of the level (:468-477): halo exchange, then the
        RHS of this rank's box."""
        self.halo.exchange(self.state)
        self.op._compute_rhs(rhs, self.state, inverse_dx_U, time)

    def local_max_inverse_dt(self, inverse_dx_U=None, time=0.0) -> float:
        return self.op._compute_max_inverse_dt(self.state, inverse_dx_U,
                                               time)

    def compute_stable_dt(self, cfl, inverse_dx_U=None, time=0.0) -> float:
        """compute_stable_dt (:544-555) with the level's max inverse dt an
        all-reduce MAX over ranks."""
        if not cfl > 0.0:
            raise L.InvalidArgument(L.GRHD_ERR_INVALID_ARG, None)
        m = self.transport.all_reduce(
            self.local_max_inverse_dt(inverse_dx_U, time), "max",
            self.state.state.device)
        return cfl / max(m, 1.0e-14)

    def stage_1(self, dt, inverse_dx_U=None, time=0.0):
        return self.op.ssprk2_stage(1, self.state, self.stage, dt,
                                    inverse_dx_U, time)

    def stage_2(self, dt, inverse_dx_U=None, time=0.0):
        return self.op.ssprk2_stage(2, self.state, self.stage, dt,
                                    inverse_dx_U, time)

    def advance_ssprk2(self, dt, inverse_dx_U=None, time=0.0):
        """advance_ssprk2 (:563-589) of the level: exchange, stage 1,
        exchange of the stage state, stage 2."""
        self.halo.exchange(self.state)
        self.stage_1(dt, inverse_dx_U, time)
        self.halo.exchange(self.stage)
        self.stage_2(dt, inverse_dx_U, time)

    def accretion_rate(self) -> float:
        """The level's rest-mass accretion rate of the last RHS: the sum
        over ranks of the boxes' sphere-face sums."""
        return self.transport.all_reduce(self.op.accretion()[0], "sum",
                                         self.state.state.device)


def advance_local_ssprk2(levels, dt, inverse_dx_U=None, time=0.0):
    """advance_ssprk2 of DistributedLevels that share one process and a
    LocalTransport mailbox, rank by rank in lockstep."""
    for lv in levels:
        lv.halo.begin(lv.state)
    for lv in levels:
        lv.halo.end(lv.state)
    for lv in levels:
        lv.stage_1(dt, inverse_dx_U, time)
    for lv in levels:
        lv.halo.begin(lv.stage)
    for lv in levels:
        lv.halo.end(lv.stage)
    for lv in levels:
        lv.stage_2(dt, inverse_dx_U, time)
