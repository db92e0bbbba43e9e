"""grhd_compute_rhs_static (no reference counterpart): the RHS with its
scratch in a fixed device array, checked against grhd_compute_rhs.

Kept in a file collected last so that it also runs after every other GPU
test has used the allocating entry points in the same process."""
import ctypes as C

import numpy as np
import pytest

import cases
import oracle_lib as O

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the per-RHS parity tolerance; both paths run the same kernels


def _call(op, fn, rhs, rhs_cs, lv, t):
    from grdzhadzha_b200.operator import _stream
    b = lv.c_box()
    return fn(op._ctx, C.c_void_p(rhs.data_ptr()), rhs_cs,
              C.c_void_p(lv.state.data_ptr()), lv.comp_stride(), C.byref(b),
              op._inv(None), t, _stream())


def _pair(name, precision="fp64", accretion_radius=0.0, pad=0):
    """(static RHS, allocating RHS, Mdot of each) on the same input."""
    p, box, s, t = cases.CASES[name]()
    p.accretion_radius = accretion_radius
    op = cases.gpu_operator(p, precision=precision)
    lib = op._lib
    out = []
    for fn in (lib.grhd_compute_rhs_static, lib.grhd_compute_rhs):
        lv = cases.gpu_level(box, s)
        n = lv.num_cells
        rhs = torch.full((5, n + pad), np.nan, dtype=torch.float64,
                         device="cuda")
        op._check(_call(op, fn, rhs, n + pad, lv, t))
        mdot, _ = op.accretion(reset=True)
        out.append((rhs[:, :n].cpu().numpy(), mdot))
    return out


def test_static_rhs_two_calls_match_allocating_entry_point():
    # two calls in a row on different boxes; the second also fills the
    # accretion partials of the static array
    (a1, _), (b1, _) = _pair("michel_c1")
    (a2, ma), (b2, mb) = _pair("torus_a09", accretion_radius=2.5)
    assert np.all(cases.rel_err(a1, b1) <= TOL)
    assert np.all(cases.rel_err(a2, b2) <= TOL)
    assert mb != 0.0 and abs(ma - mb) <= TOL * abs(mb)


def test_static_rhs_mixed_and_strided():
    (a, _), (b, _) = _pair("ksdisk", precision="mixed", pad=37)
    assert np.all(np.isfinite(a))
    assert np.all(cases.rel_err(a, b) <= TOL)


def test_static_rhs_rejects_oversized_box():
    import grdzhadzha_b200 as G
    p, box, s, t = cases.CASES["michel_c1"]()
    op = cases.gpu_operator(p)
    lv = G.LevelBox.cube(40, device="cuda")
    rhs = torch.zeros((5, lv.num_cells), dtype=torch.float64, device="cuda")
    st = _call(op, op._lib.grhd_compute_rhs_static, rhs, lv.num_cells, lv,
               0.0)
    with pytest.raises(G.GRHDError, match="too large for the static RHS"):
        op._check(st)


@pytest.mark.parametrize("name,precision", [("torus_a09", "fp64"),
                                            ("ksdisk", "mixed")])
def test_static_rhs_does_not_depend_on_what_the_array_holds(name, precision):
    """Nothing in the fixed array has to start at any value: filled with
    NaN, then with 1e300, before each of two calls, the RHS (and the
    accretion rate) equal the allocating entry point's."""
    p, box, s, t = cases.CASES[name]()
    p.accretion_radius = 2.5 if name == "torus_a09" else 0.0
    op = cases.gpu_operator(p, precision=precision)
    lib = op._lib
    from grdzhadzha_b200.operator import _stream
    lv = cases.gpu_level(box, s)
    n = lv.num_cells
    want = torch.full((5, n), np.nan, dtype=torch.float64, device="cuda")
    op._check(_call(op, lib.grhd_compute_rhs, want, n, lv, t))
    m_want, _ = op.accretion(reset=True)
    for fill in (float("nan"), 1e300):
        op._check(lib.grhd_static_scratch_fill(op._ctx, fill, _stream()))
        lv = cases.gpu_level(box, s)
        got = torch.full((5, n), np.nan, dtype=torch.float64, device="cuda")
        op._check(_call(op, lib.grhd_compute_rhs_static, got, n, lv, t))
        m_got, _ = op.accretion(reset=True)
        g = got.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert np.all(cases.rel_err(g, want.cpu().numpy()) <= TOL)
        if m_want != 0.0:
            assert abs(m_got - m_want) <= TOL * abs(m_want)


def test_static_rhs_allocates_no_device_memory():
    """After a first call (which may load the library's kernels on the
    device), two more calls on two different boxes leave the device's free
    memory (cudaMemGetInfo) unchanged.  Every buffer the test passes is
    created before the first reading."""
    cs = []
    for name in ("michel_c1", "torus_a09"):
        p, box, s, t = cases.CASES[name]()
        op = cases.gpu_operator(p)
        lv = cases.gpu_level(box, s)
        rhs = torch.empty((5, lv.num_cells), dtype=torch.float64,
                          device="cuda")
        cs.append((op, lv, rhs, t))
    for op, lv, rhs, t in cs:
        op._check(_call(op, op._lib.grhd_compute_rhs_static, rhs,
                        lv.num_cells, lv, t))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for op, lv, rhs, t in cs:
        op._check(_call(op, op._lib.grhd_compute_rhs_static, rhs,
                        lv.num_cells, lv, t))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
