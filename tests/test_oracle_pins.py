"""Pins the oracle before it is trusted (CPU only).

1. Against the reference's own driver code: oracle/_ref builds the reference's
   src/lapack/getrf.cc, potrf.cc and environment.cc unmodified on top of the
   oracle's restated BLAS and leaves; the oracle's own LU/Cholesky restatement
   must match them bit for bit (pivots, INFO and every element).
2. Against the known answers of the reference's tests:
   tests/lapack/getrf_test.cc:142-165 (ExactlySingular), 172-200
   (TinyPivots), 202-232 (QuickReturns, InvalidArguments), 236-274 (Laswp);
   tests/lapack/potrf_test.cc:102-131 (NotPositiveDefinite);
   tests/gemm_test.cc:46-113 (element-wise bound 4(k+2)eps, padding kept),
   169-212 (alpha/beta special cases, empty and invalid arguments);
   tests/level3_test.cc:479-520 (TRSM residual bound 8(ka+2)eps);
   IAMAX semantics (src/level1-inl.h:343-353: first index of max |x|, NaN
   only when x[0] is NaN).
"""
import numpy as np
import pytest

from tests.oracle_lib import (creal, rand, ref_call_getrf, ref_call_gesv, ref_call_potrf,
                              same_bits, first_diff)

EPS = np.finfo(np.float64).eps


def spd(rng, n):
    g = rng.standard_normal((n, n))
    return np.asfortranarray(g @ g.T / n + 1e-3 * np.eye(n))


# --------------------------------------------------------------------------
# 1. Bit-exact against the reference's own driver sources.

GETRF_SHAPES = [(1, 1), (5, 5), (16, 16), (17, 17), (33, 20), (20, 33), (64, 64),
                (65, 65), (100, 64), (64, 100), (129, 129), (150, 70), (70, 150),
                (300, 300), (513, 257)]


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("m,n", GETRF_SHAPES)
def test_getrf_matches_reference_driver(orc, ref_drivers, recursive, m, n):
    rng = np.random.default_rng(m * 1000 + n)
    lda = m + 3
    a = rand(rng, lda, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(min(m, n), np.int32)
    p2 = np.zeros(min(m, n), np.int32)
    f = orc.dgetrf2 if recursive else orc.dgetrf
    i1 = f(m, n, a1, lda, p1)
    i2 = ref_call_getrf(ref_drivers, recursive, m, n, a2, lda, p2)
    assert i1 == i2
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2), first_diff(a1, a2)


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("m,n", GETRF_SHAPES)
def test_sgetrf_matches_reference_driver(orc, ref_drivers, recursive, m, n):
    """The single-precision LU: the reference's getrf.cc at float on the
    oracle's float BLAS against the oracle's restatement (getrf.cc:507-546)."""
    rng = np.random.default_rng(m * 1000 + n + 7)
    lda = m + 2
    a = rand(rng, lda, n, np.float32)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(min(m, n), np.int32)
    p2 = np.zeros(min(m, n), np.int32)
    f = orc.sgetrf2 if recursive else orc.sgetrf
    i1 = f(m, n, a1, lda, p1)
    i2 = ref_call_getrf(ref_drivers, recursive, m, n, a2, lda, p2)
    assert i1 == i2
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2), first_diff(a1, a2)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (40, 3), (129, 17), (300, 1)])
def test_gesv_matches_reference_driver(orc, ref_drivers, dtype, n, nrhs):
    rng = np.random.default_rng(n + nrhs)
    a = rand(rng, n, n, dtype)
    b = rand(rng, n, nrhs, dtype)
    a1, a2, b1, b2 = (x.copy(order="F") for x in (a, a, b, b))
    p1 = np.zeros(n, np.int32)
    p2 = np.zeros(n, np.int32)
    f = orc.sgesv if dtype == np.float32 else orc.dgesv
    assert f(n, nrhs, a1, n, p1, b1, n) == ref_call_gesv(ref_drivers, n, nrhs, a2, n, p2,
                                                         b2, n)
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2) and same_bits(b1, b2), first_diff(b1, b2)


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n", [1, 7, 32, 33, 64, 65, 100, 200])
def test_potrf_matches_reference_driver(orc, ref_drivers, recursive, uplo, n):
    rng = np.random.default_rng(n)
    a = spd(rng, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    f = orc.dpotrf2 if recursive else orc.dpotrf
    assert f(uplo, n, a1, n) == ref_call_potrf(ref_drivers, recursive, uplo, n, a2, n)
    assert same_bits(a1, a2), first_diff(a1, a2)


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n", [1, 7, 32, 33, 64, 65, 100, 200])
def test_spotrf_matches_reference_driver(orc, ref_drivers, recursive, uplo, n):
    """The single-precision Cholesky: the reference's potrf.cc at float (with
    the oracle's float SYRK, TRSM, GEMM and leaf) against the restatement."""
    rng = np.random.default_rng(n + 99)
    a = spd(rng, n).astype(np.float32)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    f = orc.spotrf2 if recursive else orc.spotrf
    assert f(uplo, n, a1, n) == ref_call_potrf(ref_drivers, recursive, uplo, n, a2, n)
    assert same_bits(a1, a2), first_diff(a1, a2)


def test_getrf_singular_matches_reference_driver(orc, ref_drivers):
    rng = np.random.default_rng(5)
    m, n = 90, 80
    a = rand(rng, m, n)
    a[:, 37] = 0.0
    a[:, 70] = 0.0
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(n, np.int32)
    p2 = np.zeros(n, np.int32)
    assert orc.dgetrf(m, n, a1, m, p1) == ref_call_getrf(ref_drivers, False, m, n, a2, m, p2) == 38
    assert np.array_equal(p1, p2) and same_bits(a1, a2)


# --------------------------------------------------------------------------
# 2. Known answers of the reference's tests.

def lu_ratio(a, lu, ipiv, m, n):
    """||P L U - A||_1 / (n ||A||_1 eps) (tests/lapack/getrf_test.cc:39-75)."""
    mn = min(m, n)
    L = np.tril(lu[:m, :mn], -1) + np.eye(m, mn)
    U = np.triu(lu[:mn, :n])
    pa = a[:m, :n].copy()
    for i in range(mn):
        p = ipiv[i] - 1
        pa[[i, p]] = pa[[p, i]]
    num = np.abs(pa - L @ U).sum(axis=0).max()
    den = max(n, 1) * np.abs(a[:m, :n]).sum(axis=0).max() * EPS / 2
    return num / den if den > 0 else num


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("n", [5, 40])
def test_tiny_pivots_known_answer(orc, recursive, n):
    a = np.zeros((n, n), order="F")
    tiny = np.finfo(np.float64).tiny / 4
    power = [-min(i, 20) for i in range(n)]
    for i in range(n):
        a[i, 0] = np.ldexp(tiny, power[i])
    for k in range(1, n):
        a[0, k] = 1.0
        a[k, k] = 4.0
    ipiv = np.zeros(n, np.int32)
    f = orc.dgetrf2 if recursive else orc.dgetrf
    assert f(n, n, a, n, ipiv) == 0
    assert list(ipiv) == list(range(1, n + 1))
    for i in range(1, n):
        assert a[i, 0] == np.ldexp(1.0, power[i])


@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("k", [1, 2, 8, 9, 17, 30])
def test_exactly_singular_known_answer(orc, recursive, k):
    rng = np.random.default_rng(11)
    m, n = 40, 30
    a = rand(rng, m, n)
    a[:, k - 1] = 0.0
    if k < n:
        a[:, n - 1] = 0.0
    lu = a.copy(order="F")
    ipiv = np.zeros(n, np.int32)
    f = orc.dgetrf2 if recursive else orc.dgetrf
    assert f(m, n, lu, m, ipiv) == k
    assert lu[k - 1, k - 1] == 0.0
    assert lu_ratio(a, lu, ipiv, m, n) < 30


@pytest.mark.parametrize("m,n", [(0, 0), (0, 5), (5, 0)])
def test_getrf_quick_returns(orc, m, n):
    a = np.full(25, 3.0)
    ipiv = np.full(5, -7, np.int32)
    assert orc.dgetrf(m, n, a, 5, ipiv) == 0
    assert np.all(a == 3.0) and np.all(ipiv == -7)


def test_getrf_invalid_arguments(orc):
    a = np.full(16, 3.0)
    ipiv = np.full(4, -7, np.int32)
    assert orc.dgetrf(-1, 4, a, 4, ipiv) == -1
    assert orc.dgetrf(4, -1, a, 4, ipiv) == -2
    assert orc.dgetrf(4, 4, a, 3, ipiv) == -4
    assert orc.dgetrf(0, 4, a, 0, ipiv) == -4
    assert np.all(a == 3.0) and np.all(ipiv == -7)


def laswp_direct(a, lda, n, k1, k2, ipiv, incx):
    exp = a.copy()
    if incx == 0:
        return exp
    inc = abs(incx)
    rows = range(k1, k2 + 1) if incx > 0 else range(k2, k1 - 1, -1)
    for i in rows:
        ip = ipiv[k1 - 1 + (i - k1) * inc]
        for j in range(n):
            x, y = (i - 1) + j * lda, (ip - 1) + j * lda
            exp[x], exp[y] = exp[y], exp[x]
    return exp


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 70])
@pytest.mark.parametrize("incx", [1, -1, 2, -2, 0])
def test_laswp_known_answer(orc, n, incx):
    rng = np.random.default_rng(3)
    lda, k1, k2 = 12, 2, 9
    ipiv = rng.integers(1, lda + 1, size=k1 + (k2 - k1) * max(1, abs(incx))).astype(np.int32)
    a = rng.uniform(-1, 1, lda * max(n, 1))
    act = a.copy()
    orc.dlaswp(n, act, lda, k1, k2, ipiv, incx)
    assert np.array_equal(act, laswp_direct(a, lda, n, k1, k2, ipiv, incx))


@pytest.mark.parametrize("n", [9, 70])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("k", [1, 2, 4, 9, 33, 70])
@pytest.mark.parametrize("value", [0.0, -1.0, np.nan])
def test_potrf_not_positive_definite(orc, n, recursive, uplo, k, value):
    if k > n:
        pytest.skip("k > n")
    a = np.zeros((n, n), order="F")
    np.fill_diagonal(a, 4.0)
    a[k - 1, k - 1] = value
    f = orc.dpotrf2 if recursive else orc.dpotrf
    assert f(uplo, n, a, n) == k
    for i in range(k - 1):
        assert a[i, i] == 2.0


def gemm_bound_check(c, expected, bound, k, m, n):
    tol = 4.0 * (k + 2) * EPS / 2
    err = np.abs(c[:m, :n] - expected[:m, :n])
    return bool(np.all(err <= tol * bound[:m, :n]))


@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("tb", ["N", "T"])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 13, 9), (37, 23, 300), (64, 50, 513)])
@pytest.mark.parametrize("alpha,beta", [(1.5, 0.5), (1.0, 0.0), (-1.0, 1.0), (0.5, -1.0)])
def test_gemm_elementwise_bound(orc, ta, tb, m, n, k, alpha, beta):
    rng = np.random.default_rng(m + n + k)
    pad = 2
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a = rand(rng, ra + pad, ca)
    b = rand(rng, rb + pad, cb)
    c = rand(rng, m + pad, n)
    if beta == 0.0:
        c[:] = np.nan
    c0 = c.copy(order="F")
    opa = a[:ra, :ca] if ta == "N" else a[:ra, :ca].T
    opb = b[:rb, :cb] if tb == "N" else b[:rb, :cb].T
    A = opa.astype(np.longdouble)
    B = opb.astype(np.longdouble)
    exp = alpha * (A @ B)
    bound = abs(alpha) * (np.abs(A) @ np.abs(B))
    if beta != 0.0:
        exp = exp + beta * c0[:m, :n].astype(np.longdouble)
        bound = bound + abs(beta) * np.abs(c0[:m, :n])
    bound = bound + np.finfo(np.float64).tiny
    assert orc.dgemm(ta, tb, m, n, k, alpha, a, ra + pad, b, rb + pad, beta, c, m + pad) == 0
    assert gemm_bound_check(c, exp, bound, k, m, n)
    # Padding rows untouched (NaN-poisoned when beta == 0).
    assert same_bits(c[m:, :], c0[m:, :])


def test_gemm_special_cases(orc):
    a = np.zeros(4)
    b = np.zeros(4)
    c = np.full(4, 7.0)
    assert orc.dgemm("N", "N", 0, 2, 2, 1.0, a, 1, b, 2, 0.0, c, 1) == 0
    assert orc.dgemm("N", "N", 2, 0, 2, 1.0, a, 2, b, 2, 0.0, c, 2) == 0
    assert np.all(c == 7.0)
    one = np.ones(4)
    assert orc.dgemm("X", "N", 2, 2, 2, 1.0, one, 2, one, 2, 1.0, c, 2) == 1
    assert orc.dgemm("N", "N", -1, 2, 2, 1.0, one, 2, one, 2, 1.0, c, 2) == 3
    assert orc.dgemm("N", "N", 2, 2, 2, 1.0, one, 1, one, 2, 1.0, c, 2) == 8
    assert orc.dgemm("N", "N", 2, 2, 2, 1.0, one, 2, one, 2, 1.0, c, 1) == 13
    assert np.all(c == 7.0)


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("m", [1, 5, 31, 32, 33, 100])
def test_trsm_residual_bound(orc, side, uplo, trans, diag, m):
    """op(A) X = alpha B residual within 8 (ka + 2) eps (level3_test.cc:479-520)."""
    rng = np.random.default_rng(m)
    n = 7
    ka = m if side == "L" else n
    a = rand(rng, ka, ka)
    # Well-conditioned triangle: scaled off-diagonal, dominant diagonal.
    a = np.asfortranarray(a / ka + np.diag(1.5 + rng.uniform(0, 1, ka)))
    b = rand(rng, m, n)
    alpha = 0.75
    x = b.copy(order="F")
    assert orc.dtrsm(side, uplo, trans, diag, m, n, alpha, a, ka, x, m) == 0
    t = np.tril(a) if uplo == "L" else np.triu(a)
    if diag == "U":
        np.fill_diagonal(t, 1.0)
    op = t if trans == "N" else t.T
    X = x.astype(np.longdouble)
    lhs = op.astype(np.longdouble) @ X if side == "L" else X @ op.astype(np.longdouble)
    res = np.abs(lhs - alpha * b)
    scale = (np.abs(op) @ np.abs(x)) if side == "L" else (np.abs(x) @ np.abs(op))
    scale = scale + abs(alpha) * np.abs(b) + np.finfo(np.float64).tiny
    assert np.all(res <= 8 * (ka + 2) * EPS / 2 * scale)


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("m", [1, 31, 33, 100])
def test_strsm_residual_bound(orc, side, uplo, trans, diag, m):
    """The single-precision TRSM restatement: the same residual bound with the
    float epsilon (level3_test.cc:479-520 runs it for float and double)."""
    rng = np.random.default_rng(m + 3)
    n = 7
    ka = m if side == "L" else n
    a = rand(rng, ka, ka)
    a = np.asfortranarray((a / ka + np.diag(1.5 + rng.uniform(0, 1, ka))).astype(np.float32))
    b = rand(rng, m, n, np.float32)
    alpha = np.float32(0.75)
    x = b.copy(order="F")
    assert orc.strsm(side, uplo, trans, diag, m, n, alpha, a, ka, x, m) == 0
    t = np.tril(a) if uplo == "L" else np.triu(a)
    if diag == "U":
        np.fill_diagonal(t, 1.0)
    op = (t if trans == "N" else t.T).astype(np.float64)
    X = x.astype(np.float64)
    lhs = op @ X if side == "L" else X @ op
    res = np.abs(lhs - float(alpha) * b.astype(np.float64))
    scale = (np.abs(op) @ np.abs(X)) if side == "L" else (np.abs(X) @ np.abs(op))
    scale = scale + abs(float(alpha)) * np.abs(b) + np.finfo(np.float32).tiny
    assert np.all(res <= 8 * (ka + 2) * np.finfo(np.float32).eps / 2 * scale)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_syrk_elementwise_bound(orc, dtype, uplo, trans):
    """C := alpha op(A) op(A)^T + beta C on the uplo triangle within the GEMM
    element-wise bound 4(k+2)eps (gemm_test.cc:46-113), the other triangle
    untouched (level3.cc:84-139)."""
    rng = np.random.default_rng(17)
    n, k = 70, 130
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = rand(rng, ra, ca, dtype)
    c = rand(rng, n, n, dtype)
    c1 = c.copy(order="F")
    alpha, beta = dtype(-0.75), dtype(0.5)
    f = orc.ssyrk if dtype == np.float32 else orc.dsyrk
    assert f(uplo, trans, n, k, alpha, a, ra, beta, c1, n) == 0
    A = a.astype(np.float64)
    op = A if trans == "N" else A.T
    want = float(alpha) * (op @ op.T) + float(beta) * c.astype(np.float64)
    bound = 4 * (k + 2) * np.finfo(dtype).eps * (abs(float(alpha)) * (np.abs(op) @ np.abs(op.T))
                                                  + abs(float(beta)) * np.abs(c))
    tri = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    assert np.all(np.abs(c1.astype(np.float64) - want)[tri] <= bound[tri])
    assert np.array_equal(c1[~tri], c[~tri])


def _structured(rng, n, ld, uplo, dtype, diag="G"):
    """n x n matrix (leading dimension ld) with NaN wherever the routine must
    not read: the other triangle, the padding and, for a unit diagonal, the
    diagonal (tests/test_util.h:274-304)."""
    a = np.full((ld, n), np.nan, dtype=dtype, order="F")
    for j in range(n):
        for i in range(n):
            if (i > j) if uplo == "L" else (i < j):
                a[i, j] = rng.uniform(-1, 1)
        if diag == "N":
            a[j, j] = (1.5 if rng.uniform() >= 0.5 else -1.5) + 0.5 * rng.uniform(-1, 1)
        elif diag == "G":
            a[j, j] = rng.uniform(-1, 1)
    return a


def _dense(a, n, uplo, kind):
    """The dense matrix a structured argument stands for: symmetric ("S"),
    triangular ("N") or unit triangular ("U")."""
    t = np.array(a[:n, :n], dtype=np.float64)
    low = np.tril(np.ones((n, n), bool), -1)
    keep = low if uplo == "L" else low.T
    d = np.where(keep, t, 0.0)
    if kind == "S":
        return d + d.T + np.diag(np.diag(t))
    return d + (np.eye(n) if kind == "U" else np.diag(np.diag(t)))


def _within(got, want, bound, tol):
    return np.all(np.abs(got.astype(np.float64) - want) <= tol * bound + 1e-300)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("m,n", [(1, 7), (13, 40), (100, 7), (300, 40)])
def test_symm_bound(orc, dtype, side, uplo, m, n):
    """SYMM within 4(ka+2)eps of the exact product, reading only the stored
    triangle; beta = 0 does not read C (tests/level3_test.cc:33-89)."""
    p = "s" if dtype == np.float32 else "d"
    rng = np.random.default_rng(m * 7 + n)
    ka = m if side == "L" else n
    lda, ldb, ldc = ka + 2, m + 1, m + 3
    a = _structured(rng, ka, lda, uplo, dtype)
    b = rand(rng, ldb, n, dtype)
    A, B = _dense(a, ka, uplo, "S"), b[:m].astype(np.float64)
    for alpha, beta in [(1.5, 0.5), (-1.0, 0.0)]:
        c = rand(rng, ldc, n, dtype)
        if beta == 0.0:
            c[:] = np.nan
        c0 = c[:m].astype(np.float64)
        prod = A @ B if side == "L" else B @ A
        aprod = np.abs(A) @ np.abs(B) if side == "L" else np.abs(B) @ np.abs(A)
        want = alpha * prod + (beta * c0 if beta != 0 else 0.0)
        bound = abs(alpha) * aprod + (abs(beta) * np.abs(c0) if beta != 0 else 0.0)
        assert orc.symm(p, side, uplo, m, n, dtype(alpha), a, lda, b, ldb, dtype(beta), c,
                        ldc) == 0
        assert _within(c[:m], want, bound, 4 * (ka + 2) * np.finfo(dtype).eps)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,k", [(1, 3), (37, 13), (100, 300)])
def test_syr2k_gemmtr_bound(orc, dtype, uplo, trans, n, k):
    """SYR2K within 4(2k+2)eps and GEMMTR within 4(k+2)eps on the uplo
    triangle, the other triangle untouched, beta = 0 not reading C
    (tests/level3_test.cc:150-200, 300-360)."""
    p = "s" if dtype == np.float32 else "d"
    rng = np.random.default_rng(n * 31 + k)
    rows, cols = (n, k) if trans == "N" else (k, n)
    lda = ldb = rows + 1
    ldc = n + 2
    a, b = rand(rng, lda, cols, dtype), rand(rng, ldb, cols, dtype)
    A, B = a[:rows].astype(np.float64), b[:rows].astype(np.float64)
    opA, opB = (A, B) if trans == "N" else (A.T, B.T)
    tri = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    eps = np.finfo(dtype).eps
    for alpha, beta in [(0.75, -0.5), (-1.25, 0.0)]:
        c = rand(rng, ldc, n, dtype)
        if beta == 0.0:
            c[:n][tri] = np.nan
        c0 = c.copy(order="F")
        cc = c0[:n].astype(np.float64)
        bc = beta * cc if beta != 0 else 0.0
        abc = abs(beta) * np.abs(cc) if beta != 0 else 0.0
        want = alpha * (opA @ opB.T + opB @ opA.T) + bc
        bound = abs(alpha) * (np.abs(opA) @ np.abs(opB.T) + np.abs(opB) @ np.abs(opA.T)) + abc
        assert orc.syr2k(p, uplo, trans, n, k, dtype(alpha), a, lda, b, ldb, dtype(beta), c,
                         ldc) == 0
        assert _within(c[:n][tri], want[tri], bound[tri], 4 * (2 * k + 2) * eps)
        assert same_bits(c[:n][~tri], c0[:n][~tri])
        # GEMMTR with op(B) = B^T for trans N (and the mirror for T).
        ta, tb = trans, ("T" if trans == "N" else "N")
        c = c0.copy(order="F")
        want = alpha * (opA @ opB.T) + bc
        bound = abs(alpha) * (np.abs(opA) @ np.abs(opB.T)) + abc
        assert orc.gemmtr(p, uplo, ta, tb, n, k, dtype(alpha), a, lda, b, ldb, dtype(beta), c,
                          ldc) == 0
        assert _within(c[:n][tri], want[tri], bound[tri], 4 * (k + 2) * eps)
        assert same_bits(c[:n][~tri], c0[:n][~tri])


TRI_CASES = [(s, u, t, d) for s in "LR" for u in "LU" for t in "NT" for d in "NU"]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("side,uplo,trans,diag", TRI_CASES)
def test_trmm_bound(orc, dtype, side, uplo, trans, diag):
    """TRMM within 4(ka+2)eps of the exact product for every side, uplo,
    trans and diag, never reading the other triangle or a unit diagonal
    (tests/level3_test.cc:417-475)."""
    p = "s" if dtype == np.float32 else "d"
    eps = np.finfo(dtype).eps
    for m, n in [(1, 19), (37, 19), (300, 19), (11, 5), (11, 300)]:
        rng = np.random.default_rng(m * 100 + n)
        ka = m if side == "L" else n
        lda, ldb = ka + 1, m + 2
        a = _structured(rng, ka, lda, uplo, dtype, diag)
        b = rand(rng, ldb, n, dtype)
        T = _dense(a, ka, uplo, diag)
        op = T if trans == "N" else T.T
        B = b[:m].astype(np.float64)
        alpha = 1.5
        want = alpha * (op @ B if side == "L" else B @ op)
        bound = alpha * (np.abs(op) @ np.abs(B) if side == "L" else np.abs(B) @ np.abs(op))
        pad = b[m:].copy()
        assert orc.trmm(p, side, uplo, trans, diag, m, n, dtype(alpha), a, lda, b, ldb) == 0
        assert _within(b[:m], want, bound, 4 * (ka + 2) * eps), (m, n)
        assert same_bits(b[m:], pad)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("side,uplo,trans,diag", TRI_CASES)
def test_trmm_is_the_gemm_chain(orc, dtype, side, uplo, trans, diag):
    """For finite data the per-micro-tile k range only drops products with a
    structural zero, so TRMM equals the GEMM problem on the explicit triangle
    bit for bit (src/gemm-inl.h:62-85, 202-209), chunk boundaries included."""
    p = "s" if dtype == np.float32 else "d"
    m, n = (700, 45) if side == "L" else (45, 700)
    rng = np.random.default_rng(5)
    ka = m if side == "L" else n
    a = _structured(rng, ka, ka, uplo, dtype, diag)
    b = rand(rng, m, n, dtype)
    T = np.asfortranarray(_dense(a, ka, uplo, diag).astype(dtype))
    b1, c = b.copy(order="F"), np.zeros((m, n), dtype, order="F")
    assert orc.trmm(p, side, uplo, trans, diag, m, n, dtype(-0.5), a, ka, b1, m) == 0
    gemm = orc.sgemm if dtype == np.float32 else orc.dgemm
    if side == "L":
        gemm(trans, "N", m, n, ka, dtype(-0.5), T, ka, b, m, dtype(0), c, m)
    else:
        gemm("N", trans, m, n, ka, dtype(-0.5), b, m, T, ka, dtype(0), c, m)
    assert same_bits(b1, c), first_diff(b1, c)


def test_trmm_micro_tile_ranges_known_answer(orc):
    """The reference multiplies the whole k range of a micro-tile, structural
    zeros included (src/gemm-inl.h:62-85, 202-215): with B(20, :) infinite, a
    lower op(A) (micro-tiles of 16 rows) gives finite rows 0-15, NaN rows
    16-19 (0 * inf inside tile [16, 32)) and infinite or NaN rows 20 on."""
    m, n = 40, 3
    a = np.asfortranarray(np.tril(np.full((m, m), 0.5)))
    b = np.ones((m, n), order="F")
    b[20, :] = np.inf
    assert orc.trmm("d", "L", "L", "N", "N", m, n, 1.0, a, m, b, m) == 0
    assert np.all(np.isfinite(b[:16]))
    assert np.all(np.isnan(b[16:20]))
    assert not np.any(np.isfinite(b[20:]))
    # Right side, lower op(A): column tiles of 12 take k from their first
    # column on, so a non-finite B(:, 5) reaches columns 0-11 only.
    b = np.ones((n, m), order="F")
    b[:, 5] = np.inf
    assert orc.trmm("d", "R", "L", "N", "N", n, m, 1.0, a, m, b, n) == 0
    assert not np.any(np.isfinite(b[:, :6]))
    assert np.all(np.isnan(b[:, 6:12]))
    assert np.all(np.isfinite(b[:, 12:]))


def test_level3_quick_returns_and_errors(orc):
    """Argument checks (INFO positions) and quick returns of SYMM, SYR2K,
    GEMMTR and TRMM (src/level3.cc:26-342): alpha = 0 and beta = 1 leave C,
    alpha = 0 scales without reading A or B, TRMM with alpha = 0 zeroes B."""
    nan = np.full(16, np.nan)
    c = np.arange(16.0)
    c1 = c.copy()
    assert orc.symm("d", "L", "U", 4, 4, 0.0, nan, 4, nan, 4, 1.0, c1, 4) == 0
    assert same_bits(c1, c)
    assert orc.symm("d", "L", "U", 4, 4, 0.0, nan, 4, nan, 4, 2.0, c1, 4) == 0
    assert np.array_equal(c1, 2 * c)
    c1 = c.copy()
    assert orc.syr2k("d", "L", "N", 4, 0, 1.0, nan, 4, nan, 4, 0.0, c1, 4) == 0
    tri = np.tril(np.ones((4, 4), bool)).ravel(order="F")
    assert np.all(c1[tri] == 0) and np.array_equal(c1[~tri], c[~tri])
    c1 = c.copy()
    assert orc.gemmtr("d", "U", "N", "N", 4, 3, 0.0, nan, 4, nan, 4, 3.0, c1, 4) == 0
    assert np.array_equal(c1[~tri | np.eye(4, dtype=bool).ravel()],
                          3 * c[~tri | np.eye(4, dtype=bool).ravel()])
    b = np.arange(16.0)
    assert orc.trmm("d", "L", "L", "N", "N", 4, 4, 0.0, nan, 4, b, 4) == 0
    assert np.all(b == 0)
    z = np.zeros(16)
    assert orc.symm("d", "X", "U", 4, 4, 1.0, z, 4, z, 4, 0.0, z, 4) == 1
    assert orc.symm("d", "L", "X", 4, 4, 1.0, z, 4, z, 4, 0.0, z, 4) == 2
    assert orc.symm("d", "R", "U", 4, 5, 1.0, z, 4, z, 4, 0.0, z, 4) == 7
    assert orc.symm("d", "L", "U", 4, 4, 1.0, z, 4, z, 3, 0.0, z, 4) == 9
    assert orc.symm("d", "L", "U", 4, 4, 1.0, z, 4, z, 4, 0.0, z, 3) == 12
    assert orc.syr2k("d", "U", "X", 4, 4, 1.0, z, 4, z, 4, 0.0, z, 4) == 2
    assert orc.syr2k("d", "U", "T", 4, 5, 1.0, z, 4, z, 5, 0.0, z, 4) == 7
    assert orc.syr2k("d", "U", "N", 4, 4, 1.0, z, 4, z, 3, 0.0, z, 4) == 9
    assert orc.gemmtr("d", "U", "N", "X", 4, 4, 1.0, z, 4, z, 4, 0.0, z, 4) == 3
    assert orc.gemmtr("d", "U", "N", "N", 4, -1, 1.0, z, 4, z, 4, 0.0, z, 4) == 5
    assert orc.gemmtr("d", "U", "N", "T", 4, 4, 1.0, z, 4, z, 3, 0.0, z, 4) == 10
    assert orc.gemmtr("d", "U", "N", "N", 4, 4, 1.0, z, 4, z, 4, 0.0, z, 3) == 13
    assert orc.trmm("d", "L", "U", "N", "X", 4, 4, 1.0, z, 4, z, 4) == 4
    assert orc.trmm("d", "R", "U", "N", "N", 4, 5, 1.0, z, 4, z, 4) == 9
    assert orc.trmm("d", "L", "U", "N", "N", 4, 4, 1.0, z, 4, z, 3) == 11


@pytest.mark.parametrize("unblocked", [False, True])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("n", [1, 3, 4, 5, 17, 64, 65, 130, 300])
def test_trtri_matches_reference_driver(orc, ref_drivers, unblocked, uplo, diag, n):
    """The oracle's triangular inverse against the reference's own xTRTRI and
    xTRTI2 (src/lapack/triangular.cc:18-166) on the oracle's TRMM, TRSM, TRMV
    and SCAL, bit for bit; the unread triangle and a unit diagonal hold NaN."""
    from tests.oracle_lib import ref_call_trtri
    for dtype in (np.float64, np.float32):
        rng = np.random.default_rng(n * 3 + (diag == "U"))
        lda = n + 2
        a = np.full((lda, n), np.nan, dtype=dtype, order="F")
        t = rng.uniform(-1, 1, (n, n)) / np.sqrt(n)
        keep = np.tril(np.ones((n, n), bool), -1)
        if uplo == "U":
            keep = keep.T
        a[:n][keep] = t[keep]
        if diag == "N":
            a[np.arange(n), np.arange(n)] = 1.0 + rng.uniform(0, 1, n)
        a1, a2 = a.copy(order="F"), a.copy(order="F")
        i1 = orc.trtri(uplo, diag, n, a1, lda, unblocked=unblocked)
        i2 = ref_call_trtri(ref_drivers, unblocked, uplo, diag, n, a2, lda)
        assert i1 == i2 == 0
        assert same_bits(a1, a2), first_diff(a1, a2)


@pytest.mark.parametrize("n", [1, 2, 5, 33, 64, 65, 100, 200, 300])
@pytest.mark.parametrize("lwork_kind", ["opt", "min", "mid"])
def test_getri_matches_reference_driver(orc, ref_drivers, n, lwork_kind):
    """The oracle's GETRI against the reference's own xGETRI
    (src/lapack/getrf.cc:369-483) after the same LU: blocked (lwork = 64 n),
    unblocked (lwork = n) and a reduced block width (lwork = 20 n)."""
    from tests.oracle_lib import ref_call_getri
    for dtype in (np.float64, np.float32):
        rng = np.random.default_rng(n + 11)
        lda = n + 1
        a = rand(rng, lda, n, dtype)
        ipiv = np.zeros(n, np.int32)
        assert orc.dgetrf(n, n, a, lda, ipiv) == 0 if dtype == np.float64 else \
            orc.sgetrf(n, n, a, lda, ipiv) == 0
        lwork = {"opt": 64 * n, "min": n, "mid": 20 * n}[lwork_kind]
        a1, a2 = a.copy(order="F"), a.copy(order="F")
        w1, w2 = np.zeros(max(lwork, 1), dtype), np.zeros(max(lwork, 1), dtype)
        i1 = orc.getri(n, a1, lda, ipiv, w1, lwork)
        i2 = ref_call_getri(ref_drivers, n, a2, lda, ipiv, w2, lwork)
        assert i1 == i2 == 0
        assert same_bits(a1, a2), first_diff(a1, a2)
        assert w1[0] == w2[0]


def test_getri_singular_and_arguments(orc, ref_drivers):
    """INFO = i for U(i, i) exactly zero (A left as TRTRI's check found it),
    argument errors and the workspace query, as the reference's xGETRI."""
    from tests.oracle_lib import ref_call_getri
    n = 6
    a = np.asfortranarray(np.triu(np.ones((n, n))) + np.eye(n))
    a[3, 3] = 0.0
    ipiv = np.arange(1, n + 1, dtype=np.int32)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    w1, w2 = np.zeros(64 * n), np.zeros(64 * n)
    assert orc.getri(n, a1, n, ipiv, w1, 64 * n) == 4
    assert ref_call_getri(ref_drivers, n, a2, n, ipiv, w2, 64 * n) == 4
    assert same_bits(a1, a2)
    w = np.zeros(1)
    assert orc.getri(100, a1, 100, ipiv, w, -1) == 0 and w[0] == 6400
    assert orc.getri(-1, a1, 1, ipiv, w, 1) == -1
    assert orc.getri(n, a1, n - 1, ipiv, w, 64 * n) == -3
    assert orc.getri(n, a1, n, ipiv, w, n - 1) == -6


def test_getri_inverse_residual(orc):
    """inv(A) from GETRF + GETRI satisfies |A inv(A) - I| <= c n eps |A| |inv(A)|."""
    rng = np.random.default_rng(2)
    n = 150
    a = rand(rng, n, n)
    inv = a.copy(order="F")
    ipiv = np.zeros(n, np.int32)
    assert orc.dgetrf(n, n, inv, n, ipiv) == 0
    w = np.zeros(64 * n)
    assert orc.getri(n, inv, n, ipiv, w, 64 * n) == 0
    r = np.abs(a @ inv - np.eye(n))
    assert np.all(r <= 10 * n * EPS * (np.abs(a) @ np.abs(inv)))


def gerfs_case(rng, n, dtype, cond_spread=1.0):
    """A with column scales spread over cond_spread, a copy for its LU and
    the pivot array."""
    scale = np.exp(np.linspace(0, np.log(cond_spread), n))[None, :]
    a = np.asfortranarray((rand(rng, n, n) * scale).astype(dtype))
    return a, a.copy(order="F"), np.zeros(max(n, 1), np.int32)


@pytest.mark.parametrize("trans", ["N", "T", "C"])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (2, 3), (5, 2), (17, 1), (64, 2), (150, 3)])
@pytest.mark.parametrize("spread", [1.0, 1e6])
def test_gerfs_matches_reference_driver(orc, ref_drivers, trans, n, nrhs, spread):
    """The oracle's GERFS and LACN2 against the reference's own gesvx.cc and
    trsen.cc on the oracle's BLAS: X, FERR, BERR and the work arrays bit for
    bit (src/lapack/gesvx.cc:319-456; src/lapack/trsen.cc:2243-2366)."""
    from tests.oracle_lib import ref_call_gerfs
    for dtype in (np.float64, np.float32):
        rng = np.random.default_rng(n * 13 + nrhs + int(spread))
        a, af, ipiv = gerfs_case(rng, n, dtype, spread)
        assert ref_call_getrf(ref_drivers, False, n, n, af, n, ipiv) == 0
        b = rand(rng, n, nrhs, dtype)
        x = b.copy(order="F")
        assert orc.dgetrs(trans, n, nrhs, af, n, ipiv, x, n) == 0 if dtype == np.float64 \
            else orc.sgetrs(trans, n, nrhs, af, n, ipiv, x, n) == 0
        x = np.asfortranarray((x * (1 + 1e-4 * rng.standard_normal(x.shape))).astype(dtype))
        outs = []
        for call in ("orc", "ref"):
            xx = x.copy(order="F")
            ferr, berr = np.zeros(nrhs, dtype), np.zeros(nrhs, dtype)
            work, iwork = np.zeros(3 * n, dtype), np.zeros(n, np.int32)
            if call == "orc":
                info = orc.gerfs(trans, n, nrhs, a, n, af, n, ipiv, b, n, xx, n, ferr, berr,
                                 work, iwork)
            else:
                info = ref_call_gerfs(ref_drivers, trans, n, nrhs, a, n, af, n, ipiv, b, n, xx,
                                      n, ferr, berr, work, iwork)
            assert info == 0
            outs.append((xx, ferr, berr, work, iwork))
        for u, v in zip(outs[0], outs[1]):
            assert same_bits(u, v) if u.dtype != np.int32 else np.array_equal(u, v)


def test_gerfs_bounds_and_arguments(orc):
    """BERR near eps after refinement, FERR bounding the true error, and the
    argument checks and quick return of xGERFS."""
    rng = np.random.default_rng(6)
    n, nrhs = 120, 2
    a = rand(rng, n, n)
    af = a.copy(order="F")
    ipiv = np.zeros(n, np.int32)
    assert orc.dgetrf(n, n, af, n, ipiv) == 0
    xt = rand(rng, n, nrhs)
    b = np.asfortranarray(a @ xt)
    x = b.copy(order="F")
    assert orc.dgetrs("N", n, nrhs, af, n, ipiv, x, n) == 0
    x += 1e-6
    ferr, berr = np.zeros(nrhs), np.zeros(nrhs)
    work, iwork = np.zeros(3 * n), np.zeros(n, np.int32)
    assert orc.gerfs("N", n, nrhs, a, n, af, n, ipiv, b, n, x, n, ferr, berr, work, iwork) == 0
    assert np.all(berr < 4 * EPS)
    err = np.max(np.abs(x - xt), axis=0) / np.max(np.abs(x), axis=0)
    assert np.all(err <= ferr)
    f0, b0 = np.full(2, 7.0), np.full(2, 7.0)
    assert orc.gerfs("N", 0, 2, a, 1, af, 1, ipiv, b, 1, x, 1, f0, b0, work, iwork) == 0
    assert np.all(f0 == 0) and np.all(b0 == 0)
    assert orc.gerfs("X", n, 1, a, n, af, n, ipiv, b, n, x, n, ferr, berr, work, iwork) == -1
    assert orc.gerfs("N", -1, 1, a, n, af, n, ipiv, b, n, x, n, ferr, berr, work, iwork) == -2
    assert orc.gerfs("N", n, -1, a, n, af, n, ipiv, b, n, x, n, ferr, berr, work, iwork) == -3
    assert orc.gerfs("N", n, 1, a, n - 1, af, n, ipiv, b, n, x, n, ferr, berr, work,
                     iwork) == -5
    assert orc.gerfs("N", n, 1, a, n, af, n - 1, ipiv, b, n, x, n, ferr, berr, work,
                     iwork) == -7
    assert orc.gerfs("N", n, 1, a, n, af, n, ipiv, b, n - 1, x, n, ferr, berr, work,
                     iwork) == -10
    assert orc.gerfs("N", n, 1, a, n, af, n, ipiv, b, n, x, n - 1, ferr, berr, work,
                     iwork) == -12


def crand(rng, rows, cols, dtype=np.complex128):
    return np.asfortranarray((rng.uniform(-1, 1, (rows, cols))
                              + 1j * rng.uniform(-1, 1, (rows, cols))).astype(dtype))


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("ta", ["N", "T", "C"])
@pytest.mark.parametrize("tb", ["N", "T", "C"])
def test_zgemm_elementwise_bound(orc, dtype, ta, tb):
    """Complex GEMM within the element-wise bound 4(k+2)eps of the exact
    product (tests/gemm_test.cc:46-113 with complex types), op C conjugating,
    across KC chunks."""
    rng = np.random.default_rng(3)
    m, n, k = 37, 23, 300
    a = crand(rng, m if ta == "N" else k, k if ta == "N" else m, dtype)
    b = crand(rng, k if tb == "N" else n, n if tb == "N" else k, dtype)
    c = crand(rng, m, n, dtype)
    op = lambda x, t: x if t == "N" else (x.T if t == "T" else x.conj().T)  # noqa: E731
    A, B = op(a.astype(np.complex128), ta), op(b.astype(np.complex128), tb)
    alpha, beta = 1.5 - 0.5j, 0.25 + 0.75j
    want = alpha * (A @ B) + beta * c.astype(np.complex128)
    bound = abs(alpha) * (np.abs(A) @ np.abs(B)) + abs(beta) * np.abs(c)
    c1 = c.copy(order="F")
    assert orc.zgemm(ta, tb, m, n, k, alpha, a, a.shape[0], b, b.shape[0], beta, c1, m) == 0
    eps = np.finfo(dtype).eps
    assert np.all(np.abs(c1.astype(np.complex128) - want) <= 4 * (k + 2) * eps * bound * 2)


def test_zgemm_special_cases(orc):
    """alpha = 0 scales C (beta 0 writes zeros without reading C), beta = 1
    with alpha = 0 leaves C, argument checks (src/gemm.cc:67-123)."""
    rng = np.random.default_rng(4)
    nan = np.full((4, 4), np.nan + 1j * np.nan, order="F")
    c = crand(rng, 4, 4)
    c1 = c.copy(order="F")
    assert orc.zgemm("N", "N", 4, 4, 4, 0.0, nan, 4, nan, 4, 1.0, c1, 4) == 0
    assert same_bits(creal(c1), creal(c))
    assert orc.zgemm("N", "N", 4, 4, 4, 0.0, nan, 4, nan, 4, 2.0 - 1.0j, c1, 4) == 0
    assert np.allclose(c1, (2 - 1j) * c, rtol=1e-15)
    c2 = nan.copy(order="F")
    assert orc.zgemm("C", "T", 4, 4, 0, 1.0, nan, 4, nan, 4, 0.0, c2, 4) == 0
    assert np.all(c2 == 0)
    z = np.zeros((4, 4), np.complex128, order="F")
    assert orc.zgemm("X", "N", 4, 4, 4, 1.0, z, 4, z, 4, 0.0, z, 4) == 1
    assert orc.zgemm("N", "X", 4, 4, 4, 1.0, z, 4, z, 4, 0.0, z, 4) == 2
    assert orc.zgemm("N", "N", 4, 4, -1, 1.0, z, 4, z, 4, 0.0, z, 4) == 5
    assert orc.zgemm("T", "N", 4, 4, 5, 1.0, z, 4, z, 5, 0.0, z, 4) == 8
    assert orc.zgemm("N", "C", 4, 5, 4, 1.0, z, 4, z, 4, 0.0, z, 4) == 10
    assert orc.zgemm("N", "N", 5, 4, 4, 1.0, z, 5, z, 4, 0.0, z, 4) == 13


CTRI_CASES = [(s, u, t, d) for s in "LR" for u in "LU" for t in "NTC" for d in "NU"]


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("side,uplo,trans,diag", CTRI_CASES)
def test_ztrsm_residual_bound(orc, dtype, side, uplo, trans, diag):
    """Complex TRSM: |op(A) X - alpha B| within 8(ka+2)eps |op(A)||X| + ...
    (tests/level3_test.cc:479-520 with complex types), the unread triangle and
    a unit diagonal holding NaN."""
    rng = np.random.default_rng(21)
    m, n = (70, 13) if side == "L" else (13, 70)
    ka = m if side == "L" else n
    a = np.full((ka, ka), np.nan + 1j * np.nan, dtype=dtype, order="F")
    t = (rng.uniform(-1, 1, (ka, ka)) + 1j * rng.uniform(-1, 1, (ka, ka))) / ka
    keep = np.tril(np.ones((ka, ka), bool), -1)
    if uplo == "U":
        keep = keep.T
    a[keep] = t[keep]
    if diag == "N":
        a[np.arange(ka), np.arange(ka)] = 1.5 + rng.uniform(0, 0.5, ka) + 0.5j
    T = np.where(keep, a, 0).astype(np.complex128)
    T[np.arange(ka), np.arange(ka)] = 1.0 if diag == "U" else a[np.arange(ka), np.arange(ka)]
    op = T if trans == "N" else (T.T if trans == "T" else T.conj().T)
    b = crand(rng, m, n, dtype)
    alpha = 0.75 - 0.25j
    x = b.copy(order="F")
    assert orc.ztrsm(side, uplo, trans, diag, m, n, alpha, a, ka, x, m) == 0
    X = x.astype(np.complex128)
    lhs = op @ X if side == "L" else X @ op
    bound = (np.abs(op) @ np.abs(X) if side == "L" else np.abs(X) @ np.abs(op))
    eps = np.finfo(dtype).eps
    assert np.all(np.abs(lhs - alpha * b.astype(np.complex128)) <= 8 * (ka + 2) * eps * 2 * bound
                  + 1e-300)


def test_complex_reciprocal_is_the_runtime_quotient(orc):
    """The oracle's 1/d is the C++ runtime's complex quotient (what the
    reference computes for the TRSM diagonal); sanity against numpy within
    a few ulps on ordinary values."""
    rng = np.random.default_rng(2)
    d = (rng.uniform(-1, 1, 1000) * 2.0 ** rng.integers(-40, 40, 1000)
         + 1j * rng.uniform(-1, 1, 1000) * 2.0 ** rng.integers(-40, 40, 1000))
    out = np.zeros(1000, np.complex128)
    orc.lib.orc_zrecip(1000, d.ctypes.data, out.ctypes.data)
    assert np.allclose(out, 1 / d, rtol=1e-14, atol=0)


def test_trsm_alpha_zero_does_not_read_a(orc):
    a = np.full(9, np.nan)
    b = np.ones(6)
    assert orc.dtrsm("L", "L", "N", "N", 3, 2, 0.0, a, 3, b, 3) == 0
    assert np.all(b == 0.0)


def test_iamax_semantics(orc):
    x = np.array([1.0, -3.0, 3.0, 2.0])
    assert orc.idamax(4, x, 1) == 2
    assert orc.idamax(0, x, 1) == 0
    assert orc.idamax(4, x, 0) == 0
    assert orc.idamax(1, x, 1) == 1
    assert orc.idamax(2, x, 2) == 2  # elements 1.0, 3.0
    y = np.array([1.0, np.nan, 5.0, np.nan, -5.0])
    assert orc.idamax(5, y, 1) == 3
    z = np.array([np.nan, 9.0, 10.0])
    assert orc.idamax(3, z, 1) == 1
    w = np.array([0.0, -0.0, 0.0])
    assert orc.idamax(3, w, 1) == 1


def test_lu_ratio_random(orc):
    rng = np.random.default_rng(7)
    for m, n in [(100, 100), (200, 120), (120, 200)]:
        a = rand(rng, m, n)
        lu = a.copy(order="F")
        ipiv = np.zeros(min(m, n), np.int32)
        assert orc.dgetrf(m, n, lu, m, ipiv) == 0
        assert lu_ratio(a, lu, ipiv, m, n) < 30


def test_potrf_ratio_random(orc):
    rng = np.random.default_rng(8)
    n = 150
    a = spd(rng, n)
    for uplo in "UL":
        f = a.copy(order="F")
        assert orc.dpotrf(uplo, n, f, n) == 0
        if uplo == "L":
            L = np.tril(f)
            r = np.abs(L @ L.T - a).sum(axis=0).max()
        else:
            U = np.triu(f)
            r = np.abs(U.T @ U - a).sum(axis=0).max()
        assert r / (n * np.abs(a).sum(axis=0).max() * EPS / 2) < 30


def test_gesv_posv_solve(orc):
    rng = np.random.default_rng(9)
    n, nrhs = 120, 3
    a = rand(rng, n, n) + 2 * np.eye(n)
    x0 = rand(rng, n, nrhs)
    b = np.asfortranarray(a @ x0)
    lu, x = a.copy(order="F"), b.copy(order="F")
    ipiv = np.zeros(n, np.int32)
    assert orc.dgesv(n, nrhs, lu, n, ipiv, x, n) == 0
    assert np.abs(x - x0).max() < 1e-10
    s = spd(rng, n)
    b = np.asfortranarray(s @ x0)
    for uplo in "UL":
        f, x = s.copy(order="F"), b.copy(order="F")
        assert orc.dposv(uplo, n, nrhs, f, n, x, n) == 0
        assert np.abs(x - x0).max() < 1e-8


# --------------------------------------------------------------------------
# Complex LU (zgetrf_, cgetrf_): the reference's own getrf.cc at std::complex,
# built on the oracle's complex leaf, GEMM and TRSM, against the oracle's
# restatement of the drivers; then the reference tests' checks of the leaf
# itself (tests/lapack/getrf_test.cc:78-200).

ZGETRF_SHAPES = [(1, 1), (1, 6), (6, 1), (3, 7), (16, 16), (17, 17), (33, 17), (17, 33),
                 (64, 64), (65, 70), (90, 150), (150, 90), (200, 200)]


def _zlu_residual(a0, lu, ipiv, m, n):
    """||P L U - A||_1 / (n ||A||_1 eps) for the m x n leading block."""
    k = min(m, n)
    L = np.tril(lu[:m, :k], -1) + np.eye(m, k)
    U = np.triu(lu[:k, :n])
    prod = (L @ U).astype(np.complex128)
    for i in range(k - 1, -1, -1):
        p = ipiv[i] - 1
        prod[[i, p], :] = prod[[p, i], :]
    orig = a0[:m, :n].astype(np.complex128)
    eps = np.finfo(np.float64 if a0.dtype == np.complex128 else np.float32).eps / 2
    an = np.abs(orig).sum(axis=0).max()
    return np.abs(prod - orig).sum(axis=0).max() / max(n, 1) / an / eps


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("m,n", ZGETRF_SHAPES)
def test_zgetrf_matches_reference_driver(orc, ref_drivers, dtype, recursive, m, n):
    from tests.oracle_lib import crand, ref_call_zgetrf
    rng = np.random.default_rng(m * 977 + n)
    lda = m + 3
    a = crand(rng, lda, n, dtype)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(min(m, n), np.int32)
    p2 = np.zeros(min(m, n), np.int32)
    i1 = orc.zgetrf(m, n, a1, lda, p1, recursive=recursive)
    i2 = ref_call_zgetrf(ref_drivers, recursive, m, n, a2, lda, p2)
    assert i1 == i2 == 0
    assert np.array_equal(p1, p2)
    assert same_bits(creal(a1), creal(a2)), first_diff(creal(a1), creal(a2))
    # The reference test's checks: pivots in range, |L| <= sqrt(2) (pivots by
    # |re| + |im|), a small residual; rows below m untouched.
    assert np.all(p1 >= np.arange(1, min(m, n) + 1)) and np.all(p1 <= m)
    eps = np.finfo(np.float64 if dtype == np.complex128 else np.float32).eps
    Lpart = np.tril(a1[:m, :min(m, n)], -1)
    assert np.all(np.abs(Lpart) <= np.sqrt(2) * (1 + 4 * eps))
    assert _zlu_residual(a, a1, p1, m, n) < 30
    assert np.array_equal(a1[m:, :], a[m:, :])


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
def test_zgetrs_matches_reference_driver(orc, ref_drivers, dtype, trans):
    from tests.oracle_lib import crand, ref_call_zgetrs
    rng = np.random.default_rng(5)
    n, nrhs = 130, 3
    a = crand(rng, n, n, dtype)
    ipiv = np.zeros(n, np.int32)
    assert orc.zgetrf(n, n, a, n, ipiv) == 0
    b = crand(rng, n, nrhs, dtype)
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    assert orc.zgetrs(trans, n, nrhs, a, n, ipiv, b1, n) == 0
    assert ref_call_zgetrs(ref_drivers, trans, n, nrhs, a, n, ipiv, b2, n) == 0
    assert same_bits(creal(b1), creal(b2)), first_diff(creal(b1), creal(b2))


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("k", [1, 2, 8, 9, 17, 30])
def test_zgetrf_exactly_singular(orc, dtype, recursive, k):
    """A zero column k: INFO = k, U(k, k) = 0, the factorization completed
    (tests/lapack/getrf_test.cc:142-165)."""
    from tests.oracle_lib import crand
    rng = np.random.default_rng(11 + k)
    m, n = 40, 30
    a = crand(rng, m, n, dtype)
    a[:, k - 1] = 0
    if k < n:
        a[:, n - 1] = 0
    lu = a.copy(order="F")
    ipiv = np.zeros(n, np.int32)
    assert orc.zgetrf(m, n, lu, m, ipiv, recursive=recursive) == k
    assert lu[k - 1, k - 1] == 0
    assert _zlu_residual(a, lu, ipiv, m, n) < 30


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("n", [5, 40])
def test_zgetrf_tiny_pivots_golden(orc, dtype, recursive, n):
    """Pivots below the safe minimum divide the column: L(i, 0) = 2^-min(i, 20)
    exactly and ipiv(i) = i (tests/lapack/getrf_test.cc:172-200)."""
    rt = np.float64 if dtype == np.complex128 else np.float32
    tiny = np.finfo(rt).tiny / 4
    a = np.zeros((n, n), dtype, order="F")
    for i in range(n):
        a[i, 0] = np.ldexp(tiny, -min(i, 20))
    for k in range(1, n):
        a[0, k] = 1
        a[k, k] = 4
    ipiv = np.zeros(n, np.int32)
    assert orc.zgetrf(n, n, a, n, ipiv, recursive=recursive) == 0
    assert np.array_equal(ipiv, np.arange(1, n + 1))
    for i in range(1, n):
        assert a[i, 0] == np.ldexp(rt(1), -min(i, 20)), i


# --------------------------------------------------------------------------
# Complex Cholesky (zpotrf_, cpotrf_): the reference's own potrf.cc at
# std::complex on the oracle's complex leaf, HERK, TRSM and GEMM, against the
# oracle's restatement of the drivers; then the reference tests' checks
# (tests/lapack/potrf_test.cc:55-120): residual and the non-positive minor.

@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("n", [1, 5, 32, 33, 64, 65, 100, 150, 257])
def test_zpotrf_matches_reference_driver(orc, ref_drivers, dtype, uplo, recursive, n):
    from tests.oracle_lib import hpd, ref_call_zpotrf
    rng = np.random.default_rng(n * 7 + (uplo == "U"))
    lda = n + 2
    a = np.zeros((lda, n), dtype, order="F")
    a[:n, :] = hpd(rng, n, dtype)
    a[:n, :] += 1j * np.diag(rng.uniform(-1, 1, n)).astype(dtype)  # ignored imaginary diagonal
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    i1 = orc.zpotrf(uplo, n, a1, lda, recursive=recursive)
    i2 = ref_call_zpotrf(ref_drivers, recursive, uplo, n, a2, lda)
    assert i1 == i2 == 0
    assert same_bits(creal(a1), creal(a2)), first_diff(creal(a1), creal(a2))
    f = np.triu(a1[:n]) if uplo == "U" else np.tril(a1[:n])
    prod = f.conj().T @ f if uplo == "U" else f @ f.conj().T
    h = a[:n].astype(np.complex128)
    h[np.diag_indices(n)] = h.diagonal().real
    eps = np.finfo(np.float64 if dtype == np.complex128 else np.float32).eps
    assert np.abs(prod - h).max() <= 50 * n * eps * np.abs(h).max()
    assert np.all(f.diagonal().imag == 0)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("recursive", [False, True])
def test_zpotrf_not_positive_definite(orc, ref_drivers, dtype, uplo, recursive):
    from tests.oracle_lib import hpd, ref_call_zpotrf
    rng = np.random.default_rng(4)
    n = 120
    for bad in (1, 40, 77, 120):
        a = hpd(rng, n, dtype)
        a[bad - 1, bad - 1] = -1.0
        a1, a2 = a.copy(order="F"), a.copy(order="F")
        i1 = orc.zpotrf(uplo, n, a1, n, recursive=recursive)
        i2 = ref_call_zpotrf(ref_drivers, recursive, uplo, n, a2, n)
        assert i1 == i2 and 0 < i1 <= bad
        assert same_bits(creal(a1), creal(a2))


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "C"])
def test_zherk_against_numpy(orc, dtype, uplo, trans):
    """The oracle's HERK is alpha op(A) op(A)^H + beta C on the triangle with a
    real diagonal, the other triangle untouched (numerically, in complex128)."""
    from tests.oracle_lib import crand
    rng = np.random.default_rng(8)
    n, k = 45, 300
    a = crand(rng, n if trans == "N" else k, k if trans == "N" else n, dtype)
    c = crand(rng, n, n, dtype)
    c1 = c.copy(order="F")
    assert orc.zherk(uplo, trans, n, k, -0.75, a, a.shape[0], 0.5, c1, n) == 0
    opa = a.astype(np.complex128) if trans == "N" else a.astype(np.complex128).conj().T
    h = c.astype(np.complex128)
    h[np.diag_indices(n)] = h.diagonal().real
    want = -0.75 * opa @ opa.conj().T + 0.5 * h
    tri = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    eps = np.finfo(np.float64 if dtype == np.complex128 else np.float32).eps
    assert np.abs(c1[tri] - want[tri]).max() <= 20 * k * eps
    assert np.array_equal(c1[~tri], c[~tri])
    assert np.all(c1.diagonal().imag == 0)
    with pytest.raises(AssertionError):
        assert orc.zherk(uplo, "T", n, k, 1.0, a, a.shape[0], 1.0, c1, n) == 0
