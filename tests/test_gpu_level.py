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
