"""The exact dot-product yardstick (tests/exact_ref.py) against rational
arithmetic: every result must be the exact value rounded once to double
(CPU only)."""
from fractions import Fraction

import numpy as np
import pytest

from tests.exact_ref import exact_dot, exact_gemm_columns, exact_residual, two_product


def fraction_dot(x, y):
    return float(sum((Fraction(float(a)) * Fraction(float(b)) for a, b in zip(x, y)),
                     Fraction(0)))


@pytest.mark.parametrize("spread", [0, 8, 30])
def test_two_product_is_exact(spread):
    rng = np.random.default_rng(spread)
    a = rng.uniform(-1, 1, 2000) * np.exp2(rng.integers(-spread, spread + 1, 2000))
    b = rng.uniform(-1, 1, 2000) * np.exp2(rng.integers(-spread, spread + 1, 2000))
    p, e = two_product(a, b)
    for i in range(0, 2000, 37):
        assert Fraction(float(p[i])) + Fraction(float(e[i])) == \
            Fraction(float(a[i])) * Fraction(float(b[i]))


@pytest.mark.parametrize("spread", [0, 8, 30])
def test_exact_dot_is_correctly_rounded(spread):
    rng = np.random.default_rng(100 + spread)
    for trial in range(6):
        k = 64 + 150 * trial
        x = rng.uniform(-1, 1, k) * np.exp2(rng.integers(-spread, spread + 1, k))
        y = rng.uniform(-1, 1, k) * np.exp2(rng.integers(-spread, spread + 1, k))
        assert exact_dot(x, y) == fraction_dot(x, y)


def test_exact_dot_under_cancellation():
    """Terms that cancel to far below their size: plain summation loses every
    digit, the exact dot keeps them."""
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, 400)
    y = rng.uniform(-1, 1, 400)
    x = np.concatenate([x, x, [2.0 ** -60]])
    y = np.concatenate([y, -y, [3.0]])
    assert exact_dot(x, y) == fraction_dot(x, y) == 3.0 * 2.0 ** -60


def test_exact_gemm_columns_and_residual():
    rng = np.random.default_rng(6)
    m, k, n = 20, 300, 7
    a = rng.uniform(-1, 1, (m, k)) * np.exp2(rng.integers(-20, 21, (m, k)))
    b = rng.uniform(-1, 1, (k, n))
    out = exact_gemm_columns(a, b, [1, 5], rows=[0, 3, 19])
    for ii, i in enumerate([0, 3, 19]):
        for jj, j in enumerate([1, 5]):
            assert out[ii, jj] == fraction_dot(a[i], b[:, j])
    sq = rng.uniform(-1, 1, (k, k))
    x = rng.uniform(-1, 1, k)
    rhs = rng.uniform(-1, 1, k)
    r = exact_residual(sq, x, rhs)
    for i in (0, 17, k - 1):
        exact = Fraction(float(rhs[i])) - sum(
            (Fraction(float(sq[i, p])) * Fraction(float(x[p])) for p in range(k)), Fraction(0))
        assert r[i] == float(exact)


def test_exact_ref_rejects_what_it_cannot_split():
    with pytest.raises(ValueError):
        exact_dot([np.inf], [1.0])
    with pytest.raises(ValueError):
        exact_dot([2.0 ** -600], [2.0 ** -600])
