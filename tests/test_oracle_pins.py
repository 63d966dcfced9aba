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

from tests.oracle_lib import (rand, ref_call_getrf, ref_call_gesv, ref_call_potrf,
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
