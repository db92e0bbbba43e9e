"""Batched ensemble (new; no reference counterpart): one persistent launch
advancing members of different sizes, spins, EOS and floors.

FP64 members reproduce the single-box advance_rk4_cfl to rounding: the
conserved state to 1e-13 of its scale, the primitives to the con2prim
tolerance band (1e-10), time and accretion integral to 1e-12, the
recovery counters exactly (the persistent kernel runs the same item
functions, but the compiler contracts multiply-adds differently inside
it, which moves results by an ulp).  Mixed members agree with the
single-box mixed path to 2e-7 of the state's scale (measured 1.0e-7 in the
in-plane momentum of the a = 0.9 torus): their FP64 con2prim starts from a
different nearby pressure, and a 1e-12 change of a primitive can flip its
FP32 rounding in the primitive cache (the mixed path's own error against
FP64 is ~1e-6).  Graph replay and direct
launch of the same ensemble are bit-identical."""
import numpy as np
import pytest

import cases
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CFL = 0.25
# (case, accretion radius or 0)
MEMBERS = [("michel_c1", 6.0), ("torus_a09", 2.5), ("ksdisk", 20.0),
           ("fixedbg", 0.0), ("michel18", 0.0)]


def _members(precision="fp64"):
    out = []
    for name, R in MEMBERS:
        p, box, s, _ = cases.CASES[name]()
        p.accretion_radius = R
        out.append((cases.gpu_operator(p, precision=precision),
                    cases.gpu_level(box, s)))
    return out


def _check_fp64(got, want, what):
    ec = cases.rel_err(got[:5], want[:5])
    ep = cases.rel_err(got[5:], want[5:])
    assert np.all(ec <= 1e-13) and np.all(ep <= 1e-10), (what, ec, ep)


def _single(members, steps):
    """Each member advanced alone: (states, times, Mdot integrals, resets)."""
    res = []
    for op, lv in members:
        op.accretion(reset=True)
        t, mi, resets, cells = 0.0, 0.0, 0, 0
        for _ in range(steps):
            dt, mi, d = op.advance_rk4_cfl(lv, CFL, time=t, max_inverse_dt=mi)
            t += dt
            resets += d.num_conserved_resets
            cells += d.num_cells
        res.append((lv.state.cpu().numpy(), t, op.accretion()[1], resets,
                    cells))
    return res


def test_fp64_ensemble_matches_single_box():
    import grdzhadzha_b200 as G
    steps = 3
    ref = _single(_members(), steps)
    mem = _members()
    ens = G.Ensemble(mem, cfl=CFL)
    n0 = ens.launch_count()
    ens.advance(steps, use_graph=False)
    assert ens.launch_count() == n0 + 1
    for i, (op, lv) in enumerate(mem):
        st, t, integ, resets, cells = ref[i]
        info = ens.member_info(i)
        _check_fp64(lv.state.cpu().numpy(), st, MEMBERS[i])
        assert abs(info["time"] - t) <= 1e-12 * t
        assert abs(info["mdot_integral"] - integ) <= 1e-12 * abs(integ)
        assert info["diagnostics"].num_conserved_resets == resets
        assert info["diagnostics"].num_cells == cells
        assert info["max_inverse_dt"] > 0.0


def test_graph_replay_matches_direct_launch():
    import grdzhadzha_b200 as G
    a, b = _members(), _members()
    ea, eb = G.Ensemble(a, cfl=CFL), G.Ensemble(b, cfl=CFL)
    ea.advance(4, use_graph=False)
    n0 = eb.launch_count()
    eb.advance(2, use_graph=True)
    eb.advance(2, use_graph=True)   # replay of the captured graph
    assert eb.launch_count() == n0 + 2
    for i in range(len(a)):
        assert torch.equal(a[i][1].state, b[i][1].state), MEMBERS[i]
        assert ea.member_info(i)["time"] == eb.member_info(i)["time"]


def test_mixed_ensemble_matches_single_box_mixed():
    import grdzhadzha_b200 as G
    steps = 3
    ref = _single(_members("mixed"), steps)
    mem = _members("mixed")
    ens = G.Ensemble(mem, cfl=CFL)
    ens.advance(steps)
    for i, (op, lv) in enumerate(mem):
        st, t, integ, _, _ = ref[i]
        got = lv.state.cpu().numpy()
        err = cases.rel_err(got[:5], st[:5])
        assert np.all(err <= 2e-7), (MEMBERS[i], err)
        info = ens.member_info(i)
        assert abs(info["time"] - t) <= 1e-12 * t
        if integ != 0.0:
            assert abs(info["mdot_integral"] - integ) <= 1e-6 * abs(integ)


def test_autotune_restores_members():
    import grdzhadzha_b200 as G
    mem = _members()
    ens = G.Ensemble(mem, cfl=CFL)
    ens.advance(1, use_graph=False)
    before = [lv.state.clone() for _, lv in mem]
    infos = [ens.member_info(i) for i in range(len(mem))]
    best = ens.autotune(trial_steps=1)
    assert best["zchunk"] in (8, 16, 32, 64)
    assert 1 <= best["blocks_per_sm"] <= ens.tuning["max_blocks_per_sm"]
    assert best["ms_per_step"] > 0.0
    for i, (_, lv) in enumerate(mem):
        assert torch.equal(lv.state, before[i])
        assert ens.member_info(i)["time"] == infos[i]["time"]
        assert ens.member_info(i)["mdot_integral"] == \
            infos[i]["mdot_integral"]
    # the tuned ensemble keeps advancing (results equal up to the
    # tile-order of the accretion partials)
    ens.advance(1)


def test_invalid_members_rejected():
    import grdzhadzha_b200 as G
    p, box, s, _ = cases.CASES["pndisk"]()
    pn = (cases.gpu_operator(p), cases.gpu_level(box, s))
    with pytest.raises(G.InvalidArgument, match="Kerr-Schild"):
        G.Ensemble([pn])
    a = _members()[0]
    p, box, s, _ = cases.CASES["michel18"]()
    b = (cases.gpu_operator(p, precision="mixed"), cases.gpu_level(box, s))
    with pytest.raises(G.InvalidArgument, match="same precision"):
        G.Ensemble([a, b])
    with pytest.raises(G.InvalidArgument, match="CFL"):
        G.Ensemble([a], cfl=0.0)


def test_barrier_wait_runs_out_and_ensemble_recovers():
    """A barrier that waits for blocks that never arrive: every wait ends
    after its 50 ms limit, the launch returns an error the host reads, and
    the ensemble (and the context) stay usable."""
    import grdzhadzha_b200 as G
    mem = _members()[:2]
    saved = [lv.state.clone() for _, lv in mem]
    ens = G.Ensemble(mem, cfl=CFL)
    ens.set_barrier_test(1, 0.05)
    with pytest.raises(G.GRHDError, match="barrier wait ran out"):
        ens.advance(1, use_graph=False)
    ens.set_barrier_test(0, 4.0)
    for (_, lv), s in zip(mem, saved):
        lv.state.copy_(s)
    ens.invalidate()
    ens.advance(1, use_graph=False)
    ref = _single(_members()[:2], 1)
    for i, (_, lv) in enumerate(mem):
        _check_fp64(lv.state.cpu().numpy(), ref[i][0], MEMBERS[i])


def test_fp64_ensemble_members_match_oracle():
    """Members of the persistent launch against the oracle directly: a
    Michel inflow and an a = 0.9 torus, three RK4 steps in k_ensemble
    (graph replay) with each member's dt capped at half its CFL step (the
    cap binds, so the oracle takes the same steps), against the oracle's
    advance_rk4: conserved state <= 1e-13 of its scale, the three steps'
    change <= 1e-11 of its scale (the single-box parity tests' bounds),
    member time exact to rounding."""
    import grdzhadzha_b200 as G
    steps = 3
    names = ["michel_c1", "torus_a09"]
    cs = [cases.CASES[n]() for n in names]
    caps = [0.5 * O.stable_dt(p, box, s.copy(), CFL, t)
            for p, box, s, t in cs]
    mem = [(cases.gpu_operator(p), cases.gpu_level(box, s))
           for p, box, s, t in cs]
    ens = G.Ensemble(mem, cfl=CFL, max_dt=caps)
    ens.advance(steps, use_graph=True)
    for i, (p, box, s, t) in enumerate(cs):
        ref = s.copy()
        for k in range(steps):
            O.advance_rk4(p, box, ref, t + k * caps[i], caps[i])
        got = mem[i][1].state.cpu().numpy().reshape(-1)
        start = O.interior(box, s)
        es = cases.rel_err(O.interior(box, got), O.interior(box, ref))
        ei = cases.rel_err(O.interior(box, got) - start,
                           O.interior(box, ref) - start)
        print(f"ensemble member {names[i]} vs oracle: state {es}, "
              f"change {ei}")
        assert np.all(es <= 1e-13), (names[i], es)
        assert np.all(ei <= 1e-11), (names[i], ei)
        info = ens.member_info(i)
        assert abs(info["time"] - (t + steps * caps[i])) <= 1e-12 * steps * caps[i]
