"""Single-precision entry points through the C ABI: strsm_, cblas_strsm,
ssyrk_, sgetrf_, sgetrf2_, slaswp_, sgetrs_, sgesv_, spotrf_, spotrf2_,
spotrs_, sposv_.

The reference instantiates its LU and Cholesky families, TRSM and SYRK for
float from the same templates as for double (src/lapack/getrf.cc:507-546,
potrf.cc:747-773, src/trsm.cc:190, src/level3.cc:410), so the bar is the
same: factors, pivots, INFO and solutions bit-identical to the oracle's float
restatement (itself pinned against the reference's own getrf.cc and potrf.cc
at float in test_oracle_pins.py), the float GEMM chains in chunks of 384.
"""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits, first_diff
from tests.test_oracle_pins import GETRF_SHAPES, laswp_direct

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("m", [1, 5, 31, 33, 100, 400])
def test_strsm_bitexact(hb, orc, side, uplo, trans, diag, m):
    rng = np.random.default_rng(m + 29)
    n = 7 if m < 100 else 45
    ka = m if side == "L" else n
    lda = ka + 1
    a = rand(rng, lda, ka, np.float32)
    a[:ka, :ka] = a[:ka, :ka] / ka + np.diag(1.5 + rng.uniform(0, 1, ka)).astype(np.float32)
    # Unreferenced triangle (and unit diagonal) poisoned with NaN.
    tri = np.tril(np.ones((ka, ka), bool)) if uplo == "L" else np.triu(np.ones((ka, ka), bool))
    if diag == "U":
        np.fill_diagonal(tri, False)
    a[:ka, :ka][~tri] = np.nan
    b = rand(rng, m + 2, n, np.float32)
    for alpha in (1.0, -0.75):
        x1, x2 = b.copy(order="F"), b.copy(order="F")
        hb.strsm(side, uplo, trans, diag, m, n, alpha, a, lda, x1, m + 2)
        orc.strsm(side, uplo, trans, diag, m, n, np.float32(alpha), a, lda, x2, m + 2)
        assert same_bits(x1, x2), first_diff(x1, x2)
        assert not np.isnan(x1[:m]).any()


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("r,few", [(500, 3), (900, 16)])
def test_strsm_few_rhs_cooperative(hb, orc, side, uplo, trans, r, few):
    """The cooperative subtree path in single precision (chains restarted
    every 384)."""
    rng = np.random.default_rng(r + few + ord(side) + ord(uplo) + ord(trans))
    m, n = (r, few) if side == "L" else (few, r)
    ka = r
    a = rand(rng, ka, ka, np.float32)
    a = (a / ka + np.diag(1.5 + rng.uniform(0, 1, ka))).astype(np.float32, order="F")
    b = rand(rng, m, n, np.float32)
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    hb.strsm(side, uplo, trans, "N", m, n, 1.0, a, ka, x1, m)
    orc.strsm(side, uplo, trans, "N", m, n, np.float32(1.0), a, ka, x2, m)
    assert same_bits(x1, x2), first_diff(x1, x2)


def test_strsm_alpha_zero_and_invalid(hb):
    a = np.full(9, np.nan, np.float32)
    b = np.ones(6, np.float32)
    hb.strsm("L", "L", "N", "N", 3, 2, 0.0, a, 3, b, 3)
    assert np.all(b == 0.0)
    b[:] = 5.0
    with hb.ErrorCapture() as cap:
        hb.strsm("X", "L", "N", "N", 3, 2, 1.0, a, 3, b, 3)
        hb.strsm("L", "L", "N", "N", 3, 2, 1.0, a, 2, b, 3)
        hb.strsm("L", "L", "N", "N", 3, 2, 1.0, a, 3, b, 2)
    assert cap.errors == [("STRSM", 1), ("STRSM", 9), ("STRSM", 11)]
    assert np.all(b == 5.0)


def test_cblas_strsm_row_major(hb, orc):
    rng = np.random.default_rng(9)
    m, n = 45, 12
    a = (rng.uniform(-1, 1, (m, m)) / m + 2 * np.eye(m)).astype(np.float32)
    b = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    x = np.ascontiguousarray(b)
    hb.cblas_strsm(hb.CblasRowMajor, hb.CblasLeft, hb.CblasLower, hb.CblasNoTrans,
                   hb.CblasNonUnit, m, n, 1.0, np.ascontiguousarray(a), m, x, n)
    # Row-major: the other side and triangle on the transposes.
    xt = np.asfortranarray(b.T)
    orc.strsm("R", "U", "N", "N", n, m, np.float32(1.0), np.asfortranarray(a.T), m, xt, n)
    assert same_bits(x, np.ascontiguousarray(xt.T))
    # Column-major goes straight through.
    x2, x3 = np.asfortranarray(b), np.asfortranarray(b)
    hb.cblas_strsm(hb.CblasColMajor, hb.CblasLeft, hb.CblasUpper, hb.CblasTrans,
                   hb.CblasUnit, m, n, 0.5, np.asfortranarray(a), m, x2, m)
    orc.strsm("L", "U", "T", "U", m, n, np.float32(0.5), np.asfortranarray(a), m, x3, m)
    assert same_bits(x2, x3)


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("m,n", GETRF_SHAPES + [(1000, 1000), (16, 200), (3, 50)])
def test_sgetrf_bitexact(hb, orc, recursive, m, n):
    rng = np.random.default_rng(m * 37 + n)
    lda = m + 1
    a = rand(rng, lda, n, np.float32)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(min(m, n), np.int32)
    p2 = np.zeros(min(m, n), np.int32)
    f1 = hb.sgetrf2 if recursive else hb.sgetrf
    f2 = orc.sgetrf2 if recursive else orc.sgetrf
    assert f1(m, n, a1, lda, p1) == f2(m, n, a2, lda, p2)
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2), first_diff(a1, a2)


@pytest.mark.parametrize("recursive", [False, True])
def test_sgetrf_singular(hb, orc, recursive):
    """A zero column: INFO is the first zero pivot, the rest still factored."""
    rng = np.random.default_rng(11)
    m, n = 90, 80
    a = rand(rng, m, n, np.float32)
    a[:, 37] = 0.0
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(n, np.int32)
    p2 = np.zeros(n, np.int32)
    f1 = hb.sgetrf2 if recursive else hb.sgetrf
    f2 = orc.sgetrf2 if recursive else orc.sgetrf
    i1 = f1(m, n, a1, m, p1)
    assert i1 == f2(m, n, a2, m, p2) and i1 > 0
    assert np.array_equal(p1, p2) and same_bits(a1, a2)


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 70])
@pytest.mark.parametrize("incx", [1, -1, 2, -2, 0])
def test_slaswp(hb, n, incx):
    rng = np.random.default_rng(4)
    lda, k1, k2 = 12, 2, 9
    ipiv = rng.integers(1, lda + 1, size=k1 + (k2 - k1) * max(1, abs(incx))).astype(np.int32)
    a = rng.uniform(-1, 1, lda * max(n, 1)).astype(np.float32)
    act = a.copy()
    hb.slaswp(n, act, lda, k1, k2, ipiv, incx)
    assert np.array_equal(act, laswp_direct(a, lda, n, k1, k2, ipiv, incx))


@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (40, 3), (129, 17), (300, 64)])
def test_sgetrs_bitexact(hb, orc, trans, n, nrhs):
    rng = np.random.default_rng(n + nrhs)
    a = rand(rng, n, n, np.float32)
    p = np.zeros(n, np.int32)
    assert orc.sgetrf(n, n, a, n, p) == 0
    b = rand(rng, n + 1, nrhs, np.float32)
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    assert hb.sgetrs(trans, n, nrhs, a, n, p, x1, n + 1) == 0
    assert orc.sgetrs(trans, n, nrhs, a, n, p, x2, n + 1) == 0
    assert same_bits(x1, x2), first_diff(x1, x2)


@pytest.mark.parametrize("n,nrhs", [(1, 1), (64, 5), (257, 1), (700, 20)])
def test_sgesv_bitexact(hb, orc, n, nrhs):
    rng = np.random.default_rng(3 * n + nrhs)
    a = rand(rng, n, n, np.float32)
    b = rand(rng, n, nrhs, np.float32)
    a1, a2, b1, b2 = (x.copy(order="F") for x in (a, a, b, b))
    p1 = np.zeros(n, np.int32)
    p2 = np.zeros(n, np.int32)
    assert hb.sgesv(n, nrhs, a1, n, p1, b1, n) == orc.sgesv(n, nrhs, a2, n, p2, b2, n) == 0
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2) and same_bits(b1, b2), first_diff(b1, b2)


def test_single_invalid_arguments(hb):
    a = np.zeros(16, np.float32)
    p = np.zeros(4, np.int32)
    with hb.ErrorCapture() as cap:
        assert hb.sgetrf(-1, 4, a, 4, p) == -1
        assert hb.sgetrf2(4, 4, a, 3, p) == -4
        assert hb.sgetrs("X", 4, 1, a, 4, p, a, 4) == -1
        assert hb.sgesv(4, 1, a, 4, p, a, 3) == -7
    assert cap.errors == [("SGETRF", 1), ("SGETRF2", 4), ("SGETRS", 1), ("SGESV", 7)]


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,k", [(1, 1), (30, 10), (100, 300), (257, 64)])
# beta 0.3: beta*C is inexact, so the crossing-tile merge alpha*acc + beta*C
# (two roundings) differs from fma(C, beta, alpha*acc).
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.5, 0.3])
def test_ssyrk_bitexact(hb, orc, uplo, trans, n, k, beta):
    rng = np.random.default_rng(n + k + 5)
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = rand(rng, ra, ca, np.float32)
    c = rand(rng, n + 1, n, np.float32)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    hb.ssyrk(uplo, trans, n, k, -0.75, a, ra, beta, c1, n + 1)
    orc.ssyrk(uplo, trans, n, k, np.float32(-0.75), a, ra, np.float32(beta), c2, n + 1)
    assert same_bits(c1, c2), first_diff(c1, c2)


def _spd32(rng, n):
    g = rng.standard_normal((n, n))
    return np.asfortranarray((g @ g.T / n + 1e-1 * np.eye(n)).astype(np.float32))


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n", [1, 7, 32, 33, 64, 65, 100, 200, 600])
def test_spotrf_bitexact(hb, orc, recursive, uplo, n):
    rng = np.random.default_rng(n + 41)
    a = _spd32(rng, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    f1 = hb.spotrf2 if recursive else hb.spotrf
    f2 = orc.spotrf2 if recursive else orc.spotrf
    assert f1(uplo, n, a1, n) == f2(uplo, n, a2, n) == 0
    assert same_bits(a1, a2), first_diff(a1, a2)


@pytest.mark.parametrize("uplo", ["U", "L"])
def test_spotrf_not_positive_definite(hb, orc, uplo):
    rng = np.random.default_rng(3)
    n = 90
    a = _spd32(rng, n)
    a[50, 50] = -1.0
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    i1 = hb.spotrf(uplo, n, a1, n)
    assert i1 == orc.spotrf(uplo, n, a2, n) and i1 > 0
    assert same_bits(a1, a2)


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (65, 3), (200, 17)])
def test_spotrs_sposv_bitexact(hb, orc, uplo, n, nrhs):
    rng = np.random.default_rng(n * 3 + nrhs)
    a = _spd32(rng, n)
    b = rand(rng, n, nrhs, np.float32)
    f = a.copy(order="F")
    assert orc.spotrf(uplo, n, f, n) == 0
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    assert hb.spotrs(uplo, n, nrhs, f, n, x1, n) == orc.spotrs(uplo, n, nrhs, f, n, x2, n) == 0
    assert same_bits(x1, x2), first_diff(x1, x2)
    a1, a2, y1, y2 = (v.copy(order="F") for v in (a, a, b, b))
    assert hb.sposv(uplo, n, nrhs, a1, n, y1, n) == orc.sposv(uplo, n, nrhs, a2, n, y2, n) == 0
    assert same_bits(a1, a2) and same_bits(y1, y2)
