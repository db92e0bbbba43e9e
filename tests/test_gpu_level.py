"""A level cut into several boxes: LevelData::exchange() on the device
(grhd_level_exchange) followed by the per-box RHS.

The reference evaluates a level box by box after exchanging the ghosts
between boxes (compute_leveldata_flux_rhs_from_fixed_background,
FixedBGFArrayBoxFiniteVolume.hpp:322-363, its directional pass :300-320;
the physical ghosts of each box are the outflow fill of that box,
:113-177).  Cutting a level into boxes therefore leaves its RHS unchanged,
and that is the check here: every case's single-box level is cut into
disjoint boxes, the ghosts of each box that lie inside the domain are
poisoned with NaN, the exchange fills them from the owning boxes, and the
per-box RHS, CFL bound and accretion rate are compared with those of the
single box:

  * FP64: per component max|multi - single| / max|single| <= 1e-13 (the
    operator's 1e-12 parity tolerance and below; a shell cell recovers
    its primitives from the metric without derivatives, an interior cell
    from the one with derivatives, which may round differently; measured
    on B200: 0 to 2.7e-15);
  * mixed: <= 1e-6 (an interior cell's con2prim starts from the stored
    pressure, a shell cell's from the bracket, and the FP32 rounding of
    the two converged results can differ in the last place; measured
    1.2e-8 to 1.4e-7);
  * the CFL bound: equal up to 1e-14 relative; the accretion rate (a sum
    over sphere faces, in another order): 1e-12 relative.

A box that starts one cell inside the domain takes its outflow ghosts
from its own first cell (the reference's interior_box.smallEnd), not from
the domain's, so the cuts below leave no one-cell box on the domain
boundary.  Cuts that give one-cell boxes inside the level are included:
their ghosts come from two boxes away.
"""
import numpy as np
import pytest

import cases
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _boxes(box, cuts):
    """Disjoint boxes of the interior [box.lo, box.hi] cut before the
    level indices in cuts[d]."""
    edges = []
    for d in range(3):
        e = [box.lo[d]] + sorted(cuts[d]) + [box.hi[d] + 1]
        edges.append([(e[q], e[q + 1] - 1) for q in range(len(e) - 1)])
    out = []
    for z in edges[2]:
        for y in edges[1]:
            for x in edges[0]:
                out.append(((x[0], y[0], z[0]), (x[1], y[1], z[1])))
    return out


def _split_level(box, state_np, cuts):
    """LevelBoxes of the cut level: state copied from the single box's
    ghosted state, the ghosts inside the domain set to NaN."""
    import grdzhadzha_b200 as G
    V = O.state_view(box, state_np)
    parts = []
    for lo, hi in _boxes(box, cuts):
        sl = tuple(slice(lo[d] - 2 - box.glo[d], hi[d] + 3 - box.glo[d])
                   for d in (2, 1, 0))
        st = np.array(V[(slice(None),) + sl])
        ks, js, is_ = [np.arange(lo[d] - 2, hi[d] + 3) for d in (2, 1, 0)]
        K, J, I = np.meshgrid(ks, js, is_, indexing="ij")
        inside = ((I >= box.dlo[0]) & (I <= box.dhi[0]) &
                  (J >= box.dlo[1]) & (J <= box.dhi[1]) &
                  (K >= box.dlo[2]) & (K <= box.dhi[2]))
        own = ((I >= lo[0]) & (I <= hi[0]) & (J >= lo[1]) & (J <= hi[1]) &
               (K >= lo[2]) & (K <= hi[2]))
        st[:, inside & ~own] = np.nan
        lv = G.LevelBox(lo=lo, hi=hi, ghost=2, domain_lo=tuple(box.dlo),
                        domain_hi=tuple(box.dhi), state=torch.empty(0))
        lv.state = torch.from_numpy(np.ascontiguousarray(st)).cuda()
        parts.append(lv)
    return parts


def _interior_slice(box, lo, hi):
    return tuple(slice(lo[d] - box.lo[d], hi[d] + 1 - box.lo[d])
                 for d in (2, 1, 0))


CUTS = {
    # z slabs of 3, 2 and 4 cells; x and y halves
    "ksdisk": [[28], [20], [3, 5]],
    "pndisk": [[17, 39], [], [4]],
    # a one-cell box in the middle of x, quarters in z
    "torus_a09": [[15, 16], [16], [8, 16, 24]],
    "michel_c1": [[12], [6, 12, 18], [12, 13]],
}


def _compare(name, precision, tol):
    import grdzhadzha_b200 as G
    p, box, s, t = cases.CASES[name]()
    op = cases.gpu_operator(p, precision=precision)
    single = cases.gpu_level(box, s)
    rhs1 = single.new_rhs()
    op.compute_rhs(rhs1, single, time=t)
    inv1 = op.compute_max_inverse_dt(cases.gpu_level(box, s), time=t)
    parts = _split_level(box, s, CUTS[name])
    G.level_exchange(parts)
    for lv in parts:
        assert not torch.isnan(lv.state).any(), "exchange left a ghost"
    rhs_n = torch.empty_like(rhs1)
    inv_n = 0.0
    for lv in parts:
        r = lv.new_rhs()
        op.compute_rhs(r, lv, time=t)
        rhs_n[(slice(None),) + _interior_slice(box, lv.lo, lv.hi)] = r
    for lv in parts:
        inv_n = max(inv_n, op.compute_max_inverse_dt(lv, time=t))
    err = cases.rel_err(rhs_n.cpu().numpy().reshape(5, -1),
                        rhs1.cpu().numpy().reshape(5, -1))
    print(f"{name} {precision} {len(parts)} boxes: rhs err {err}")
    assert np.all(err <= tol), err
    assert abs(inv_n - inv1) <= 1e-14 * inv1


@pytest.mark.parametrize("name", list(CUTS))
def test_cut_level_rhs_fp64(name):
    _compare(name, "fp64", 1e-13)


@pytest.mark.parametrize("name", ["ksdisk", "torus_a09"])
def test_cut_level_rhs_mixed(name):
    _compare(name, "mixed", 1e-6)


def test_cut_level_accretion_rate():
    """Michel inflow with the accretion sphere r < 4 M crossing eight boxes:
    the per-box accretion rates add up to the single box's."""
    import grdzhadzha_b200 as G
    p, box, s, t = cases.CASES["michel_c1"]()
    p.accretion_radius = 4.0
    op = cases.gpu_operator(p)
    single = cases.gpu_level(box, s)
    op.compute_rhs(single.new_rhs(), single, time=t)
    m1, _ = op.accretion()
    parts = _split_level(box, s, [[12], [12], [12]])
    G.level_exchange(parts)
    total = 0.0
    for lv in parts:
        op.compute_rhs(lv.new_rhs(), lv, time=t)
        total += op.accretion()[0]
    assert m1 != 0.0
    assert abs(total - m1) <= 1e-12 * abs(m1), (total, m1)


def test_exchange_rejects_overlapping_boxes():
    import grdzhadzha_b200 as G
    a = G.LevelBox(lo=(0, 0, 0), hi=(7, 7, 3), domain_lo=(0, 0, 0),
                   domain_hi=(7, 7, 7))
    b = G.LevelBox(lo=(0, 0, 3), hi=(7, 7, 7), domain_lo=(0, 0, 0),
                   domain_hi=(7, 7, 7))
    with pytest.raises(G.InvalidArgument, match="overlap"):
        G.level_exchange([a, b])


def _split_stage(parts):
    import grdzhadzha_b200 as G
    return [G.LevelBox(lo=lv.lo, hi=lv.hi, ghost=2, domain_lo=lv.domain_lo,
                       domain_hi=lv.domain_hi,
                       state=torch.full_like(lv.state, float("nan")))
            for lv in parts]


def _gather(box, parts):
    z, y, x = [box.hi[d] - box.lo[d] + 1 for d in (2, 1, 0)]
    out = torch.empty((11, z, y, x), dtype=torch.float64, device="cuda")
    for lv in parts:
        out[(slice(None),) + _interior_slice(box, lv.lo, lv.hi)] = \
            lv.interior()
    return out


SSPRK2_TOL = 1e-12


@pytest.mark.parametrize("name", ["ksdisk", "pndisk", "torus_a09"])
def test_cut_level_ssprk2(name):
    """advance_ssprk2 of the cut level (exchange before each RHS,
    grhd_ssprk2_stage per box) against the single box's fused
    grhd_advance_ssprk2, three steps: <= 1e-12 of each component's scale
    (the split stage runs the per-cell pass of the stage RHS as its own
    kernel instead of fused into the update; same arithmetic; measured on
    B200: 0 to 7e-16)."""
    p, box, s, t = cases.CASES[name]()
    op = cases.gpu_operator(p)
    single = cases.gpu_level(box, s)
    dt = op.compute_stable_dt(single, cfl=0.3, time=t)
    parts = _split_level(box, s, CUTS[name])
    stages = _split_stage(parts)
    for n in range(3):
        op.advance_ssprk2(single, time=t + n * dt, dt=dt)
        op.advance_level_ssprk2(parts, stages, dt, time=t + n * dt)
    ref = single.interior().cpu().numpy().reshape(11, -1)
    got = _gather(box, parts).cpu().numpy().reshape(11, -1)
    err = cases.rel_err(got[:5], ref[:5])
    print(f"{name} ssprk2 {len(parts)} boxes: state err {err}")
    assert np.all(err <= SSPRK2_TOL), err


@pytest.mark.parametrize("layout", ["slabs", "pencils"])
def test_distributed_level_virtual_ranks(layout):
    """The multi-rank level (grdzhadzha_b200.halo) with its ranks driven in
    one process through a LocalTransport: device pack / unpack of the
    halos (grhd_region_copy), the RHS of each rank's box and three SSPRK2
    steps, against the single box."""
    import grdzhadzha_b200 as G
    from grdzhadzha_b200 import halo as H
    p, box, s, t = cases.CASES["torus_a09"]()
    op = cases.gpu_operator(p)
    dlo, dhi = tuple(box.dlo), tuple(box.dhi)
    boxes = (H.slab_boxes(dlo, dhi, 5) if layout == "slabs"
             else H.pencil_boxes(dlo, dhi, 3, 2))
    mailbox = {}
    ranks = [H.DistributedLevel(op, boxes, r, dlo, dhi,
                                transport=H.LocalTransport(mailbox, r))
             for r in range(len(boxes))]
    full = _split_level(box, s, [[], [], []])[0]
    parts = _split_level(box, s, [[], [], []])
    for lv in ranks:
        src = _split_level_box(box, s, lv.state.lo, lv.state.hi)
        lv.state.state.copy_(src.state)
        assert lv.halo.sends and lv.halo.recvs
    for lv in ranks:
        lv.halo.begin(lv.state)
    for lv in ranks:
        lv.halo.end(lv.state)
    assert not mailbox
    rhs1 = full.new_rhs()
    op.compute_rhs(rhs1, full, time=t)
    rhs_n = torch.empty_like(rhs1)
    for lv in ranks:
        assert not torch.isnan(lv.state.state).any()
        r = lv.state.new_rhs()
        op.compute_rhs(r, lv.state, time=t)
        rhs_n[(slice(None),) + _interior_slice(box, lv.state.lo,
                                               lv.state.hi)] = r
    err = cases.rel_err(rhs_n.cpu().numpy().reshape(5, -1),
                        rhs1.cpu().numpy().reshape(5, -1))
    assert np.all(err <= 1e-13), err
    single = parts[0]
    dt = op.compute_stable_dt(single, cfl=0.3, time=t)
    inv = max(lv.local_max_inverse_dt(time=t) for lv in ranks)
    assert abs(0.3 / inv - dt) <= 1e-14 * dt
    for n in range(3):
        op.advance_ssprk2(single, time=t + n * dt, dt=dt)
        H.advance_local_ssprk2(ranks, dt, time=t + n * dt)
    ref = single.interior().cpu().numpy().reshape(11, -1)
    got = _gather(box, [lv.state for lv in ranks]).cpu().numpy()
    err = cases.rel_err(got.reshape(11, -1)[:5], ref[:5])
    print(f"{layout} {len(ranks)} virtual ranks: state err {err}")
    assert np.all(err <= SSPRK2_TOL), err


def _split_level_box(box, s, lo, hi):
    """One box of the cut level with its in-domain ghosts poisoned."""
    cuts = [[c for c in (lo[d], hi[d] + 1) if box.lo[d] < c <= box.hi[d]]
            for d in range(3)]
    for lv in _split_level(box, s, cuts):
        if tuple(lv.lo) == tuple(lo):
            return lv
    raise AssertionError("box not found")


def test_region_copy_rejects_outside_regions():
    from grdzhadzha_b200 import halo as H
    import grdzhadzha_b200 as G
    lv = G.LevelBox(lo=(0, 0, 0), hi=(3, 3, 3))
    buf = torch.empty(11 * 64, dtype=torch.float64, device="cuda")
    with pytest.raises(G.InvalidArgument):
        H.DeviceRegions().pack(lv, (0, 0, 0), (3, 3, 6), buf)
