"""Parity of the sm_100a operator on CCZ4-stored geometry (grhd_ccz4_*,
LevelDataFiniteVolumeOperator, Source/Matter/GRHD/FArrayBoxFiniteVolume.hpp:
1215-1364) with the oracle's restatement, through the C ABI.

Tolerances as for the fixed-background operator: one RHS, one recovery
and the CFL bound <= 1e-12 of each component's scale; three SSPRK2 steps
<= 1e-11 (the step composed in the test from the oracle's RHS and recovery
with the reference's add_scaled / combine arithmetic, :927-969).  The
reference's own equivalence check (Tests/GRHDFixedBGTest/
GRHDFixedBGTest.cpp:195-237, 1e-10) runs on the GPU too: CCZ4-geometry
flux RHS against the fixed-background flux RHS of this library.
"""
import numpy as np
import pytest

import cases
import oracle_lib as O
from test_oracle_ccz4 import _params, _reference_box, _test_state

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _gpu_op(p):
    import grdzhadzha_b200 as G
    atmo = G.AtmosphereOptions(p.atmo_rho_floor, p.atmo_pressure_floor,
                               p.atmo_max_velocity_squared,
                               p.atmo_metric_source_atmosphere_factor)
    rec = G.RecoveryOptions(p.rec_max_iterations, p.rec_tolerance,
                            p.rec_pressure_floor, p.rec_max_velocity_squared)
    return G.LevelDataFiniteVolumeOperator(
        G.IdealGasEOS(p.gamma), atmo, p.limiter_theta,
        bool(p.use_reconstruction), rec, bool(p.use_static_metric_sources))


def _gpu_level(box, s36):
    import grdzhadzha_b200 as G
    lv = G.LevelBox(lo=tuple(box.lo), hi=tuple(box.hi),
                    ghost=box.lo[0] - box.glo[0], domain_lo=tuple(box.dlo),
                    domain_hi=tuple(box.dhi), state=torch.empty(0),
                    ncomp=O.CCZ4_NUM_VARS)
    shape = (O.CCZ4_NUM_VARS,) + O.state_view(box, s36[:11 * box.comp_stride]
                                              ).shape[1:]
    lv.state = torch.from_numpy(s36.reshape(shape).copy()).cuda()
    return lv


def _case(name):
    if name == "reference_box":
        p = _params()
        box = _reference_box()
        return p, box, _test_state(p, box)
    p, box, s, t = cases.CASES[name]()
    p.excision_radius = 0.0
    return p, box, s


CASES = ["reference_box", "ksdisk", "pndisk", "fixedbg"]


def _inv(p):
    return [1.0 / p.dx] * 3


@pytest.mark.parametrize("name", CASES)
def test_ccz4_rhs_matches_oracle(name):
    p, box, s = _case(name)
    s36 = O.ccz4_state(p, box, s)
    op = _gpu_op(p)
    lv = _gpu_level(box, s36)
    rhs = lv.new_rhs()
    op.compute_rhs(rhs, lv, inverse_dx_U=_inv(p))
    ref36 = s36.copy()
    ref = O.ccz4_compute_rhs(p, box, ref36)
    err = cases.rel_err(rhs.cpu().numpy().reshape(5, -1), ref.reshape(5, -1))
    print(f"{name}: CCZ4 RHS err {err}")
    assert np.all(err <= 1e-12), err
    # the outflow fill of the state (conserved, chi, h, lapse, shift)
    got = lv.state.cpu().numpy().reshape(O.CCZ4_NUM_VARS, -1)
    want = ref36.reshape(O.CCZ4_NUM_VARS, -1)
    assert np.array_equal(got, want)


def test_ccz4_flux_rhs_equals_fixed_background_on_gpu():
    p = _params(use_static_metric_sources=0)
    box = _reference_box()
    s = _test_state(p, box)
    fixed_op = cases.gpu_operator(p)
    fixed_lv = cases.gpu_level(box, s)
    fixed = fixed_lv.new_rhs()
    fixed_op.compute_rhs(fixed, fixed_lv)
    op = _gpu_op(p)
    lv = _gpu_level(box, O.ccz4_state(p, box, s))
    rhs = lv.new_rhs()
    op.compute_rhs(rhs, lv, inverse_dx_U=_inv(p))
    err = cases.rel_err(rhs.cpu().numpy().reshape(5, -1),
                        fixed.cpu().numpy().reshape(5, -1))
    assert np.all(err <= 1e-10), err


@pytest.mark.parametrize("name", ["ksdisk", "fixedbg"])
def test_ccz4_recovery_and_cfl_match_oracle(name):
    import grdzhadzha_b200 as G
    p, box, s = _case(name)
    op = _gpu_op(p)
    s36 = O.ccz4_state(p, box, s)
    inv = op.compute_max_inverse_dt(_gpu_level(box, s36),
                                    inverse_dx_U=_inv(p))
    inv_ref = O.ccz4_max_inverse_dt(p, box, s36)
    assert abs(inv - inv_ref) <= 1e-12 * inv_ref
    # off the recovered manifold: floors and resets in the recovery; in the
    # disk's atmosphere the CFL recovery fails, at the same cell as the
    # oracle's (the reference throws there)
    V = O.state_view(box, s)
    rng = np.random.default_rng(cases.SEED + 9)
    V[O.D] *= 1.0 + 1e-3 * rng.uniform(-1, 1, V[O.D].shape)
    V[O.TAU] *= 1.0 + 1e-3 * rng.uniform(-1, 1, V[O.TAU].shape)
    s36 = O.ccz4_state(p, box, s)
    lv = _gpu_level(box, s36)
    try:
        O.ccz4_max_inverse_dt(p, box, s36)
        oracle_cell = None
    except O.OracleError as e:
        oracle_cell = tuple(e.err.cell)
    if oracle_cell is None:
        op.compute_max_inverse_dt(lv, inverse_dx_U=_inv(p))
    else:
        with pytest.raises(G.GRHDError) as gi:
            op.compute_max_inverse_dt(lv, inverse_dx_U=_inv(p))
        assert tuple(gi.value.cell) == oracle_cell
        assert "CFL" in str(gi.value)
    d = op.recover_primitives(lv)
    ref36 = s36.copy()
    dref = O.ccz4_recover_primitives(p, box, ref36)
    assert (d.num_cells, d.num_failed_recoveries, d.num_floored_primitives,
            d.num_conserved_resets) == dref.as_tuple()
    g0 = O.CCZ4_GRHD * box.comp_stride
    got = lv.state.cpu().numpy().reshape(-1)[g0:].reshape(11, -1)
    err = cases.rel_err(got, ref36[g0:].reshape(11, -1))
    assert np.all(err <= 1e-12), err


def _oracle_ssprk2(p, box, s36, dt):
    """advance_ssprk2 (:1323-1348) from the oracle's RHS and recovery."""
    cs = box.comp_stride
    g0 = O.CCZ4_GRHD * cs
    inner = O.interior(box, s36[g0:], comps=slice(0, 5))
    old = s36.copy()
    stage = s36.copy()
    k0 = O.ccz4_compute_rhs(p, box, s36).reshape(inner.shape)
    st = O.interior(box, stage[g0:], comps=slice(0, 5))
    st += dt * k0
    O.ccz4_recover_primitives(p, box, stage)
    k1 = O.ccz4_compute_rhs(p, box, stage).reshape(inner.shape)
    cur = O.interior(box, s36[g0:], comps=slice(0, 5))
    o_ = O.interior(box, old[g0:], comps=slice(0, 5))
    cur[...] = 0.5 * (o_ + O.interior(box, stage[g0:], comps=slice(0, 5)) +
                      dt * k1)
    O.ccz4_recover_primitives(p, box, s36)


@pytest.mark.parametrize("name", ["ksdisk", "fixedbg"])
def test_ccz4_ssprk2_matches_oracle(name):
    p, box, s = _case(name)
    s36 = O.ccz4_state(p, box, s)
    op = _gpu_op(p)
    lv = _gpu_level(box, s36)
    dt = op.compute_stable_dt(lv, inverse_dx_U=_inv(p), cfl=0.3)
    ref = s36.copy()
    for _ in range(3):
        op.advance_ssprk2(lv, inverse_dx_U=_inv(p), dt=dt)
        _oracle_ssprk2(p, box, ref, dt)
    g0 = O.CCZ4_GRHD * box.comp_stride
    got = lv.state.cpu().numpy().reshape(-1)[g0:].reshape(11, -1)
    err = cases.rel_err(got[:5], ref[g0:].reshape(11, -1)[:5])
    print(f"{name}: CCZ4 SSPRK2 err {err}")
    assert np.all(err <= 1e-11), err


def test_ccz4_rejects_an_eleven_component_state():
    import grdzhadzha_b200 as G
    p = _params()
    op = _gpu_op(p)
    lv = G.LevelBox(lo=(0, 0, 0), hi=(3, 3, 3))
    with pytest.raises(ValueError):
        op.compute_rhs(lv.new_rhs(), lv, inverse_dx_U=[4.0] * 3)


def test_ccz4_state_from_background_matches_oracle():
    """The library's device-side CCZ4 fill (via grhd_eval_background)
    against the oracle's restatement of the reference test's
    store_ccz4_background_vars: within 1e-14 of each variable's scale."""
    p, box, s = _case("ksdisk")
    op = cases.gpu_operator(p)
    lv = op.ccz4_state(cases.gpu_level(box, s))
    got = lv.state.cpu().numpy().reshape(O.CCZ4_NUM_VARS, -1)
    want = O.ccz4_state(p, box, s).reshape(O.CCZ4_NUM_VARS, -1)
    scale = np.maximum(np.abs(want).max(axis=1), 1e-300)
    err = np.abs(got - want).max(axis=1) / scale
    assert np.all(err <= 1e-14), err


def _split36(box, s36, cuts):
    """LevelBoxes of 36 components cut from a single-box CCZ4 state, the
    ghosts inside the domain set to NaN in every component."""
    import grdzhadzha_b200 as G
    from test_gpu_level import _boxes
    shape = (O.CCZ4_NUM_VARS,) + tuple(box.ghi[d] - box.glo[d] + 1
                                       for d in (2, 1, 0))
    V = s36.reshape(shape)
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
                        domain_hi=tuple(box.dhi), state=torch.empty(0),
                        ncomp=O.CCZ4_NUM_VARS)
        lv.state = torch.from_numpy(np.ascontiguousarray(st)).cuda()
        parts.append(lv)
    return parts


def test_ccz4_cut_level_matches_single_box():
    """LevelDataFiniteVolumeOperator on a level of several boxes: the
    exchange moves all 36 components (the geometry too), then the per-box
    RHS equals the single box's (<= 1e-13 of each component's scale;
    measured bit-identical or rounding)."""
    import grdzhadzha_b200 as G
    p, box, s = _case("ksdisk")
    s36 = O.ccz4_state(p, box, s)
    op = _gpu_op(p)
    single = _gpu_level(box, s36)
    rhs1 = single.new_rhs()
    op.compute_rhs(rhs1, single, inverse_dx_U=_inv(p))
    parts = _split36(box, s36, [[28], [20], [3, 5]])
    G.level_exchange(parts)
    for lv in parts:
        assert not torch.isnan(lv.state).any()
    rhs_n = torch.empty_like(rhs1)
    for lv in parts:
        r = lv.new_rhs()
        op.compute_rhs(r, lv, inverse_dx_U=_inv(p))
        sl = tuple(slice(lv.lo[d] - box.lo[d], lv.hi[d] + 1 - box.lo[d])
                   for d in (2, 1, 0))
        rhs_n[(slice(None),) + sl] = r
    err = cases.rel_err(rhs_n.cpu().numpy().reshape(5, -1),
                        rhs1.cpu().numpy().reshape(5, -1))
    print("CCZ4 cut level err", err)
    assert np.all(err <= 1e-13), err


def test_ccz4_halo_exchange_of_36_components():
    """The multi-rank halo exchange (device pack / unpack, virtual ranks in
    one process) moves the same 36 components as the level exchange."""
    import grdzhadzha_b200 as G
    from grdzhadzha_b200 import halo as H
    p, box, s = _case("ksdisk")
    s36 = O.ccz4_state(p, box, s)
    cuts = [[], [], [3, 6]]
    a = _split36(box, s36, cuts)
    b = _split36(box, s36, cuts)
    G.level_exchange(a)
    boxes = [(tuple(lv.lo), tuple(lv.hi)) for lv in b]
    mailbox = {}
    ex = [H.HaloExchange(boxes, r, tuple(box.dlo), tuple(box.dhi),
                         H.LocalTransport(mailbox, r))
          for r in range(len(b))]
    for r, lv in enumerate(b):
        ex[r].begin(lv)
    for r, lv in enumerate(b):
        ex[r].end(lv)
    assert not mailbox
    for la, lb in zip(a, b):
        assert torch.equal(torch.nan_to_num(la.state, nan=7.0),
                           torch.nan_to_num(lb.state, nan=7.0))
        assert not torch.isnan(lb.state).any()


def test_ccz4_cut_level_ssprk2_matches_single_box():
    """advance_ssprk2 of a CCZ4-geometry level cut into 12 boxes (exchange
    of 36 components before each RHS, grhd_ccz4_ssprk2_stage per box)
    against the single box's grhd_ccz4_advance_ssprk2, three steps:
    <= 1e-13 of each component's scale."""
    import grdzhadzha_b200 as G
    p, box, s = _case("ksdisk")
    s36 = O.ccz4_state(p, box, s)
    op = _gpu_op(p)
    single = _gpu_level(box, s36)
    dt = op.compute_stable_dt(single, inverse_dx_U=_inv(p), cfl=0.3)
    parts = _split36(box, s36, [[28], [20], [3, 5]])
    stages = [G.LevelBox(lo=lv.lo, hi=lv.hi, ghost=2, domain_lo=lv.domain_lo,
                         domain_hi=lv.domain_hi, ncomp=O.CCZ4_NUM_VARS)
              for lv in parts]
    for _ in range(3):
        op.advance_ssprk2(single, inverse_dx_U=_inv(p), dt=dt)
        op.advance_level_ssprk2(parts, stages, dt, inverse_dx_U=_inv(p))
    g0 = O.CCZ4_GRHD
    want = single.interior(slice(g0, g0 + 5)).cpu().numpy()
    got = np.empty_like(want)
    for lv in parts:
        sl = tuple(slice(lv.lo[d] - box.lo[d], lv.hi[d] + 1 - box.lo[d])
                   for d in (2, 1, 0))
        got[(slice(None),) + sl] = lv.interior(slice(g0, g0 + 5)).cpu().numpy()
    err = cases.rel_err(got.reshape(5, -1), want.reshape(5, -1))
    print("CCZ4 cut level SSPRK2 err", err)
    assert np.all(err <= 1e-13), err
