"""grhd_advance_rk4_cfl_host (new): one CFL-limited RK4 step of a state in
host memory, against grhd_advance_rk4_cfl on the same state in device
memory.  The host call copies to the device only what the step reads (the
conserved components, the primitives of the z planes holding excised
cells, the pressure in mixed precision), so the test poisons every other
primitive slot of the host state with NaN: the results must still equal
the device call's bit for bit (both run the same kernels on the same
inputs), in FP64 and in mixed precision, over three steps.  The first
call computes the CFL speed and runs copy in, step, copy out in turn;
the later calls are given it and run the step as a wavefront over z
chunks of 8 planes with the copies overlapped (3, 4 and 4 chunks here,
the last one short for 30 planes)."""
import numpy as np
import pytest

import cases
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _excised_planes(p, box):
    """Ghosted z-plane indices of the state array that hold excised cells
    or their one-plane margin (as the entry point copies them)."""
    R, dx, cz = p.excision_radius, p.dx, p.center[2]
    k0 = int(np.floor((cz - R) / dx - 0.5)) - 1
    k1 = int(np.ceil((cz + R) / dx - 0.5)) + 1
    k0, k1 = max(k0, box.glo[2]), min(k1, box.ghi[2])
    return slice(k0 - box.glo[2], k1 - box.glo[2] + 1)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["torus_a09", "torus_a09_n30", "michel_c1"])
def test_host_step_equals_device_step(name, precision):
    if name == "torus_a09_n30":
        p, box, s, t = cases.torus_a09(n=30)
    else:
        p, box, s, t = cases.CASES[name]()
    assert p.excision_radius > 0.0
    op = cases.gpu_operator(p, precision=precision)
    lv = cases.gpu_level(box, s)
    host = torch.from_numpy(s.copy()).reshape(lv.state.shape).pin_memory()
    V = host.numpy()
    keep = _excised_planes(p, box)
    for c in range(5, 11):
        if precision == "mixed" and c == O.PRESS:
            continue
        poisoned = np.full_like(V[c], np.nan)
        poisoned[keep] = V[c][keep]
        V[c] = poisoned
    mi_d = mi_h = 0.0
    for _ in range(3):
        dt_d, mi_d, d_d = op.advance_rk4_cfl(lv, 0.25, time=t,
                                             max_inverse_dt=mi_d)
        dt_h, mi_h, d_h, hb, db = op.advance_rk4_cfl_host(
            host, lv, 0.25, time=t, max_inverse_dt=mi_h)
        assert dt_h == dt_d and mi_h == mi_d
        assert (d_h.num_cells, d_h.num_conserved_resets) == \
            (d_d.num_cells, d_d.num_conserved_resets)
        t += dt_d
    dev = lv.state.cpu()
    assert torch.isfinite(host).all()
    assert torch.equal(host, dev), (host - dev).abs().max()
    n = lv.state[0].numel()
    plane = lv.state.shape[2] * lv.state.shape[3]
    nplanes = keep.stop - keep.start
    want_in = 8 * (5 * n + (n if precision == "mixed" else 0)
                   + (6 - (precision == "mixed")) * nplanes * plane)
    assert hb == want_in and db == 8 * 11 * n, (hb, db, want_in)


def test_host_step_rejects_a_box_that_is_not_the_domain():
    import grdzhadzha_b200 as G
    p, _, _, _ = cases.CASES["fixedbg"]()
    op = cases.gpu_operator(p)
    lv = G.LevelBox(lo=(0, 0, 0), hi=(7, 7, 7), ghost=2,
                    domain_lo=(0, 0, 0), domain_hi=(15, 15, 15),
                    device="cuda")
    host = lv.state.cpu()
    with pytest.raises(G.InvalidArgument):
        op.advance_rk4_cfl_host(host, lv, 0.25)


@pytest.mark.parametrize("cell,where", [((13, 14, 17), 2), ((0, 9, 17), 1)])
def test_host_step_recovery_failure_matches_the_device_step(cell, where):
    """A planted D < 0 (host-side; no device fault) in the third of four
    z chunks: the wavefront host step (given the CFL speed) fails with the
    device step's error record (the cell's recovery, or for a boundary cell
    the outflow fill of its ghosts first), returns only after its copies
    have finished, and the context steps cleanly afterwards."""
    import grdzhadzha_b200 as G
    p, box, s, t = cases.CASES["torus_a09"]()
    i, j, k = cell
    g = [box.lo[d] - box.glo[d] for d in range(3)]
    bad = s.copy()
    O.state_view(box, bad)[O.D, g[2] + k, g[1] + j, g[0] + i] = -1.0
    op = cases.gpu_operator(p)
    lv = cases.gpu_level(box, bad)
    host = torch.from_numpy(bad.copy()).reshape(lv.state.shape).pin_memory()
    mi = op.compute_max_inverse_dt(cases.gpu_level(box, s), time=t)
    with pytest.raises(G.GRHDError) as eh:
        op.advance_rk4_cfl_host(host, lv, 0.25, time=t, max_inverse_dt=mi)
    with pytest.raises(G.GRHDError) as ed:
        op.advance_rk4_cfl(lv, 0.25, time=t, max_inverse_dt=mi)
    assert (eh.value.where, eh.value.cell) == (ed.value.where, ed.value.cell)
    assert eh.value.where == where and eh.value.cell == cell
    good = torch.from_numpy(s.copy()).reshape(lv.state.shape).pin_memory()
    dev = cases.gpu_level(box, s)
    dt_h, mi_h, _, _, _ = op.advance_rk4_cfl_host(good, dev, 0.25, time=t,
                                                  max_inverse_dt=mi)
    dt_d, mi_d, _ = op.advance_rk4_cfl(dev, 0.25, time=t, max_inverse_dt=mi)
    assert (dt_h, mi_h) == (dt_d, mi_d)
    assert torch.equal(good, dev.state.cpu())
