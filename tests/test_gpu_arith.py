"""The FP64 division, reciprocal, square root and reciprocal square root
the kernels compute with (approximate reciprocal / reciprocal square root
refined by Newton-Raphson steps, grhd_device.cuh), through grhd_eval_arith,
against IEEE results computed by numpy: within one ulp over operands spread
across the normal range, and mostly the IEEE result itself on the ranges
the kernels use them on (densities, pressures, enthalpies, metric
functions, speeds).  numpy's 1/sqrt(a) is rounded twice, so the reciprocal
square root is held to two ulp of it."""
import numpy as np
import pytest

import cases

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def op():
    p, _, _, _ = cases.CASES["fixedbg"]()
    return cases.gpu_operator(p)


def _eval(op, a, b):
    da = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    out = torch.empty(4 * a.size, dtype=torch.float64, device="cuda")
    st = op._lib.grhd_eval_arith(op._ctx, a.size, da.data_ptr(),
                                 db.data_ptr(), out.data_ptr(), None)
    assert st == 0, st
    return out.cpu().numpy().reshape(-1, 4)


def _ulps(got, want):
    return np.abs(got - want) / np.spacing(np.abs(want))


def _signed(rng, n, lo, hi):
    mag = 10.0 ** rng.uniform(lo, hi, n)
    return np.where(rng.random(n) < 0.5, -mag, mag)


def test_wide_range_within_one_ulp(op):
    rng = np.random.default_rng(20261204)
    n = 1 << 20
    a = _signed(rng, n, -150.0, 150.0)
    b = _signed(rng, n, -150.0, 150.0)
    out = _eval(op, np.abs(a), b)
    u = [_ulps(out[:, 0], np.abs(a) / b), _ulps(out[:, 1], 1.0 / b),
         _ulps(out[:, 2], np.sqrt(np.abs(a))),
         _ulps(out[:, 3], 1.0 / np.sqrt(np.abs(a)))]
    print("max ulp (a/b, 1/b, sqrt a, 1/sqrt a):",
          [float(x.max()) for x in u])
    for x, bound in zip(u, (1.0, 1.0, 1.0, 2.0)):
        assert x.max() <= bound


def test_kernel_ranges_mostly_ieee(op):
    rng = np.random.default_rng(7)
    n = 1 << 20
    a = 10.0 ** rng.uniform(-12.0, 2.0, n)
    b = 10.0 ** rng.uniform(-10.0, 2.0, n)
    out = _eval(op, a, b)
    for name, got, want in (("a/b", out[:, 0], a / b),
                            ("1/b", out[:, 1], 1.0 / b),
                            ("sqrt", out[:, 2], np.sqrt(a)),
                            ("rsqrt", out[:, 3], 1.0 / np.sqrt(a))):
        u = _ulps(got, want)
        print(name, "max ulp", float(u.max()), "IEEE result",
              float(np.mean(u == 0.0)))
        if name == "rsqrt":
            assert u.max() <= 2.0
        else:
            assert u.max() <= 1.0
            assert np.mean(u == 0.0) > 0.9


def test_square_root_of_zero_and_negative(op):
    a = np.array([0.0, -0.0, -1.0, 4.0, 2.0])
    out = _eval(op, a, np.ones(5))
    assert out[0, 2] == 0.0 and out[1, 2] == 0.0
    assert np.isnan(out[2, 2])
    assert out[3, 2] == 2.0
    assert out[4, 2] == np.sqrt(2.0)
