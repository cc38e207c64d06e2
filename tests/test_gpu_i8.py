"""The FP64-accuracy SP2 step on the tcgen05 integer tensor cores (kind::i8).

The iterate is split into eight int8 digit planes in fixed point (2^-6 first digit, base
2^7), the product is the sum of the digit-pair products by weight, each an exact int32
tensor-core product (the Ozaki scheme with fixed-point splits), combined in fp64. Checked
against an extended-precision product on SP2-like iterates (spectrum in [0, 1]) at sizes
that cover one tile, ragged tiles and several tile rows: the error must stay within a few
fp64 GEMM roundings (2e-17 n of the largest element), the result exactly symmetric, and the
step's trace partials equal to the trace and Frobenius norm of what it wrote.
"""
import numpy as np
import pytest

from pm7b200 import api

pytestmark = pytest.mark.gpu


def _iterate(n, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    lam = rng.uniform(0.0, 1.0, size=n)
    x = (q * lam) @ q.T
    return 0.5 * (x + x.T)


@pytest.mark.parametrize("n", [40, 64, 128, 131, 200, 300, 517])
@pytest.mark.parametrize("square", [True, False])
def test_step_matches_extended_precision(n, square):
    x = _iterate(n, n)
    y, norms = api.sp2_step_i8(x, square)
    xl = x.astype(np.longdouble)
    ref = xl @ xl if square else 2 * xl - xl @ xl
    err = float(np.max(np.abs(y - ref)))
    assert err < 2e-17 * max(n, 64) * 4, err
    np.testing.assert_array_equal(y, y.T)
    assert abs(norms[0] - np.trace(y)) < 1e-12 * n
    assert abs(norms[1] - np.sum(y * y)) < 1e-12 * n


def test_step_is_deterministic():
    x = _iterate(300, 7)
    a, na = api.sp2_step_i8(x, True)
    b, nb = api.sp2_step_i8(x, True)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(na, nb)
