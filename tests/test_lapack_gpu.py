"""GPU parity of the LU/Cholesky path through the C ABI against the oracle:
factors, pivots and INFO bit-identical (tests/lapack/getrf_test.cc,
potrf_test.cc, linear_test.cc, posv_test.cc cases), plus the configuration
dgetrf n=4096 with its LU ratio."""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits, first_diff
from tests.test_oracle_pins import GETRF_SHAPES, lu_ratio, spd, laswp_direct

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("m,n", GETRF_SHAPES + [(1000, 1000), (16, 200), (3, 50)])
def test_dgetrf_bitexact(hb, orc, recursive, m, n):
    rng = np.random.default_rng(m * 31 + n)
    lda = m + 1
    a = rand(rng, lda, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(min(m, n), np.int32)
    p2 = np.zeros(min(m, n), np.int32)
    f1 = hb.dgetrf2 if recursive else hb.dgetrf
    f2 = orc.dgetrf2 if recursive else orc.dgetrf
    assert f1(m, n, a1, lda, p1) == f2(m, n, a2, lda, p2)
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2), first_diff(a1, a2)


def test_dgetrf_config_4096(hb, orc):
    """dgetrf n=4096, U[-1,1]: ipiv identical to the reference, factors
    bit-identical, and ||PA - LU|| / (n eps ||A||) reported small."""
    rng = np.random.default_rng(2024)
    n = 4096
    a = rand(rng, n, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(n, np.int32)
    p2 = np.zeros(n, np.int32)
    assert hb.dgetrf(n, n, a1, n, p1) == 0
    orc.set_threads(8)
    assert orc.dgetrf(n, n, a2, n, p2) == 0
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2), first_diff(a1, a2)
    assert lu_ratio(a, a1, p1, n, n) < 30


def test_dgetrf_8192(hb, orc):
    """dgetrf n=8192: 128 trailing updates with many tiles per persistent CTA
    and 8-CTA cooperative leaves; factors and ipiv bit-identical."""
    import os
    rng = np.random.default_rng(8192)
    n = 8192
    a = rand(rng, n, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(n, np.int32)
    p2 = np.zeros(n, np.int32)
    assert hb.dgetrf(n, n, a1, n, p1) == 0
    orc.set_threads(os.cpu_count() or 8)
    assert orc.dgetrf(n, n, a2, n, p2) == 0
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2), first_diff(a1, a2)


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("n", [5, 40])
def test_tiny_pivots(hb, recursive, n):
    a = np.zeros((n, n), order="F")
    tiny = np.finfo(np.float64).tiny / 4
    power = [-min(i, 20) for i in range(n)]
    for i in range(n):
        a[i, 0] = np.ldexp(tiny, power[i])
    for k in range(1, n):
        a[0, k] = 1.0
        a[k, k] = 4.0
    ipiv = np.zeros(n, np.int32)
    f = hb.dgetrf2 if recursive else hb.dgetrf
    assert f(n, n, a, n, ipiv) == 0
    assert list(ipiv) == list(range(1, n + 1))
    for i in range(1, n):
        assert a[i, 0] == np.ldexp(1.0, power[i])


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("k", [1, 2, 8, 9, 17, 30])
def test_exactly_singular(hb, orc, recursive, k):
    rng = np.random.default_rng(11)
    m, n = 40, 30
    a = rand(rng, m, n)
    a[:, k - 1] = 0.0
    if k < n:
        a[:, n - 1] = 0.0
    lu, lu2 = a.copy(order="F"), a.copy(order="F")
    ipiv, ipiv2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    f = hb.dgetrf2 if recursive else hb.dgetrf
    assert f(m, n, lu, m, ipiv) == k
    assert lu[k - 1, k - 1] == 0.0
    (orc.dgetrf2 if recursive else orc.dgetrf)(m, n, lu2, m, ipiv2)
    assert same_bits(lu, lu2) and np.array_equal(ipiv, ipiv2)


def test_getrf_quick_returns_and_invalid(hb):
    for m, n in [(0, 0), (0, 5), (5, 0)]:
        a = np.full(25, 3.0)
        ipiv = np.full(5, -7, np.int32)
        assert hb.dgetrf(m, n, a, 5, ipiv) == 0
        assert np.all(a == 3.0) and np.all(ipiv == -7)
    for recursive, name in [(False, "DGETRF"), (True, "DGETRF2")]:
        f = hb.dgetrf2 if recursive else hb.dgetrf
        a = np.full(16, 3.0)
        ipiv = np.full(4, -7, np.int32)
        with hb.ErrorCapture() as cap:
            assert f(-1, 4, a, 4, ipiv) == -1
            assert f(4, -1, a, 4, ipiv) == -2
            assert f(4, 4, a, 3, ipiv) == -4
            assert f(0, 4, a, 0, ipiv) == -4
        assert cap.errors == [(name, 1), (name, 2), (name, 4), (name, 4)]
        assert np.all(a == 3.0) and np.all(ipiv == -7)


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 70])
@pytest.mark.parametrize("incx", [1, -1, 2, -2, 0])
def test_dlaswp(hb, n, incx):
    rng = np.random.default_rng(3)
    lda, k1, k2 = 12, 2, 9
    ipiv = rng.integers(1, lda + 1, size=k1 + (k2 - k1) * max(1, abs(incx))).astype(np.int32)
    a = rng.uniform(-1, 1, lda * max(n, 1))
    act = a.copy()
    hb.dlaswp(n, act, lda, k1, k2, ipiv, incx)
    assert np.array_equal(act, laswp_direct(a, lda, n, k1, k2, ipiv, incx))


@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (50, 3), (300, 17), (129, 64)])
def test_dgetrs_dgesv_bitexact(hb, orc, trans, n, nrhs):
    rng = np.random.default_rng(n + nrhs)
    a = rand(rng, n, n)
    b = rand(rng, n, nrhs)
    lu = a.copy(order="F")
    ipiv = np.zeros(n, np.int32)
    assert orc.dgetrf(n, n, lu, n, ipiv) == 0
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    assert hb.dgetrs(trans, n, nrhs, lu, n, ipiv, x1, n) == 0
    assert orc.dgetrs(trans, n, nrhs, lu, n, ipiv, x2, n) == 0
    assert same_bits(x1, x2), first_diff(x1, x2)
    if trans == "N":
        a1, a2 = a.copy(order="F"), a.copy(order="F")
        y1, y2 = b.copy(order="F"), b.copy(order="F")
        p1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
        assert hb.dgesv(n, nrhs, a1, n, p1, y1, n) == orc.dgesv(n, nrhs, a2, n, p2, y2, n)
        assert same_bits(a1, a2) and same_bits(y1, y2) and np.array_equal(p1, p2)


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n", [1, 7, 32, 33, 64, 65, 100, 200, 777])
def test_dpotrf_bitexact(hb, orc, recursive, uplo, n):
    rng = np.random.default_rng(n)
    a = spd(rng, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    f1 = hb.dpotrf2 if recursive else hb.dpotrf
    f2 = orc.dpotrf2 if recursive else orc.dpotrf
    assert f1(uplo, n, a1, n) == f2(uplo, n, a2, n) == 0
    assert same_bits(a1, a2), first_diff(a1, a2)


@pytest.mark.parametrize("n", [9, 70])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("k", [1, 2, 4, 9, 33, 70])
@pytest.mark.parametrize("value", [0.0, -1.0, np.nan])
def test_potrf_not_positive_definite(hb, orc, n, recursive, uplo, k, value):
    if k > n:
        pytest.skip("k > n")
    a = np.zeros((n, n), order="F")
    np.fill_diagonal(a, 4.0)
    a[k - 1, k - 1] = value
    a2 = a.copy(order="F")
    f = hb.dpotrf2 if recursive else hb.dpotrf
    assert f(uplo, n, a, n) == k
    for i in range(k - 1):
        assert a[i, i] == 2.0
    (orc.dpotrf2 if recursive else orc.dpotrf)(uplo, n, a2, n)
    assert same_bits(a, a2)


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (60, 4), (300, 64)])
def test_dpotrs_dposv_bitexact(hb, orc, uplo, n, nrhs):
    rng = np.random.default_rng(n * 3 + nrhs)
    a = spd(rng, n)
    b = rand(rng, n, nrhs)
    f = a.copy(order="F")
    assert orc.dpotrf(uplo, n, f, n) == 0
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    assert hb.dpotrs(uplo, n, nrhs, f, n, x1, n) == 0
    orc.dpotrs(uplo, n, nrhs, f, n, x2, n)
    assert same_bits(x1, x2)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    y1, y2 = b.copy(order="F"), b.copy(order="F")
    assert hb.dposv(uplo, n, nrhs, a1, n, y1, n) == orc.dposv(uplo, n, nrhs, a2, n, y2, n) == 0
    assert same_bits(a1, a2) and same_bits(y1, y2)
