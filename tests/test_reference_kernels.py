"""The oracle against the reference library itself (CPU).

oracle/_ref/libhwyblas_ref.so is the reference's own source tree compiled
unmodified against the Highway-API shim (oracle/hwy_shim: one AVX-512-class
target, 8 doubles a vector). These tests require the oracle's restatement of
the kernels' rounding (GEMM chains and merges, TRSM base solves, the LU and
Cholesky leaves, IAMAX) to give the reference's own results bit for bit, so
that the GPU tests, which compare with the oracle, compare with the
reference. Skipped where the reference's sources were not available to
build the library.
"""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits


def _fill(rng, rows, cols, dtype=np.float64):
    return np.asfortranarray(rng.uniform(-1, 1, (rows, cols)).astype(dtype))


GEMM_SHAPES = [(1, 1, 1), (16, 12, 7), (17, 13, 256), (33, 25, 257), (100, 80, 300),
               (129, 65, 513), (40, 200, 1000), (257, 3, 70)]


@pytest.mark.parametrize("m,n,k", GEMM_SHAPES)
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("alpha,beta", [(1.5, 0.5), (1.0, 1.0), (-1.0, 0.0), (0.7, -0.3)])
def test_dgemm_oracle_is_the_reference(orc, refblas, m, n, k, ta, tb, alpha, beta):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = _fill(rng, m if ta == "N" else k, k if ta == "N" else m)
    b = _fill(rng, k if tb == "N" else n, n if tb == "N" else k)
    c = _fill(rng, m, n)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    orc.dgemm(ta, tb, m, n, k, alpha, a, a.shape[0], b, b.shape[0], beta, c1, m)
    refblas.dgemm(ta, tb, m, n, k, alpha, a, a.shape[0], b, b.shape[0], beta, c2, m)
    assert same_bits(c1, c2)


@pytest.mark.parametrize("m,n,k", [(32, 24, 385), (100, 50, 800), (7, 9, 3)])
def test_sgemm_oracle_is_the_reference(orc, refblas, m, n, k):
    rng = np.random.default_rng(m + n + k)
    a, b, c = _fill(rng, m, k, np.float32), _fill(rng, k, n, np.float32), _fill(rng, m, n,
                                                                                  np.float32)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    orc.sgemm("N", "N", m, n, k, 1.5, a, m, b, k, 0.5, c1, m)
    refblas.dgemm("N", "N", m, n, k, 1.5, a, m, b, k, 0.5, c2, m, single=True)
    assert same_bits(c1, c2)


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
def test_dtrsm_oracle_is_the_reference(orc, refblas, side, uplo, trans, diag):
    rng = np.random.default_rng(ord(side) + 2 * ord(uplo) + 3 * ord(trans) + 5 * ord(diag))
    m, n = 150, 70
    ka = m if side == "L" else n
    a = _fill(rng, ka, ka) / ka
    a[np.diag_indices(ka)] = rng.uniform(0.5, 2.0, ka)
    b = _fill(rng, m, n)
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    orc.dtrsm(side, uplo, trans, diag, m, n, 0.75, a, ka, b1, m)
    refblas.dtrsm(side, uplo, trans, diag, m, n, 0.75, a, ka, b2, m)
    assert same_bits(b1, b2)


def test_dtrsm_config_shape_oracle_is_the_reference(orc, refblas):
    """The configuration's dtrsm, L/L/N/U, M = 4096, N = 512 (scaled so that
    the solution stays finite)."""
    rng = np.random.default_rng(2)
    m, n = 4096, 512
    a = _fill(rng, m, m) / m
    b = _fill(rng, m, n)
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    orc.dtrsm("L", "L", "N", "U", m, n, 1.0, a, m, b1, m)
    refblas.dtrsm("L", "L", "N", "U", m, n, 1.0, a, m, b2, m)
    assert same_bits(b1, b2)


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.3])
def test_dsyrk_oracle_is_the_reference(orc, refblas, uplo, trans, beta):
    rng = np.random.default_rng(ord(uplo) + ord(trans) + int(10 * beta))
    n, k = 130, 300
    a = _fill(rng, n, k) if trans == "N" else _fill(rng, k, n)
    c = _fill(rng, n, n)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    orc.dsyrk(uplo, trans, n, k, -1.0, a, a.shape[0], beta, c1, n)
    refblas.dsyrk(uplo, trans, n, k, -1.0, a, a.shape[0], beta, c2, n)
    assert same_bits(c1, c2)


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
def test_dtrmm_oracle_is_the_reference(orc, refblas, side, uplo, trans, diag):
    """TRMM multiplies each micro-tile only over its nonzero k range: the
    reference's own tile geometry (16 x 12 at 8 lanes) decides which
    products are formed, here with an Inf that meets structural zeros."""
    rng = np.random.default_rng(ord(side) * 3 + ord(uplo) + ord(trans) * 7 + ord(diag))
    m, n = 77, 53
    ka = m if side == "L" else n
    a = _fill(rng, ka, ka)
    b = _fill(rng, m, n)
    b[5, 7] = np.inf
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    orc.trmm("d", side, uplo, trans, diag, m, n, 1.25, a, ka, b1, m)
    refblas.dtrmm(side, uplo, trans, diag, m, n, 1.25, a, ka, b2, m)
    assert same_bits(b1, b2)


@pytest.mark.parametrize("mode", ["rand", "ties", "nan_first", "nan_inside", "inf"])
@pytest.mark.parametrize("n,incx", [(1, 1), (7, 1), (1000, 1), (1000, 3), (33, 2)])
def test_idamax_oracle_is_the_reference(orc, refblas, mode, n, incx):
    rng = np.random.default_rng(n + incx)
    x = rng.uniform(-1, 1, (n - 1) * incx + 1)
    if mode == "ties":
        x = np.round(x * 3) / 3
    elif mode == "nan_first":
        x[0] = np.nan
    elif mode == "nan_inside":
        x[(n // 2) * incx] = np.nan
    elif mode == "inf":
        x[(n // 3) * incx] = -np.inf
    assert orc.idamax(n, x, incx) == refblas.idamax(n, x, incx)


@pytest.mark.parametrize("m,n", [(1, 1), (16, 16), (17, 40), (300, 300), (517, 260),
                                 (100, 333), (1200, 64)])
def test_dgetrf_oracle_is_the_reference(orc, refblas, m, n):
    rng = np.random.default_rng(m * 13 + n)
    a = rand(rng, m, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1, p2 = np.zeros(min(m, n), np.int32), np.zeros(min(m, n), np.int32)
    assert orc.dgetrf(m, n, a1, m, p1) == refblas.dgetrf(m, n, a2, m, p2)
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2)


def test_dgetrf_singular_and_tiny_pivots_oracle_is_the_reference(orc, refblas):
    rng = np.random.default_rng(3)
    n = 90
    a = rand(rng, n, n)
    a[:, 40] = a[:, 3] * 2.0  # exactly dependent column
    t = np.asfortranarray(np.tril(np.exp2(-np.minimum(np.arange(n)[:, None], 20.0)) *
                                  np.ones((n, n))))
    for m in (a, t):
        a1, a2 = m.copy(order="F"), m.copy(order="F")
        p1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
        assert orc.dgetrf(n, n, a1, n, p1) == refblas.dgetrf(n, n, a2, n, p2)
        assert np.array_equal(p1, p2)
        assert same_bits(a1, a2)


@pytest.mark.parametrize("n", [1, 31, 64, 200, 450])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_dpotrf_oracle_is_the_reference(orc, refblas, n, uplo):
    rng = np.random.default_rng(n + ord(uplo))
    g = rng.standard_normal((n, n))
    a = np.asfortranarray(g @ g.T / n + np.eye(n))
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    assert orc.dpotrf(uplo, n, a1, n) == refblas.dpotrf(uplo, n, a2, n) == 0
    assert same_bits(a1, a2)
    # Not positive definite: the same INFO and the same partial factor.
    b = a.copy(order="F")
    b[n // 2, n // 2] = -1.0
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    assert orc.dpotrf(uplo, n, b1, n) == refblas.dpotrf(uplo, n, b2, n)


def test_solvers_oracle_is_the_reference(orc, refblas):
    rng = np.random.default_rng(11)
    n, nrhs = 260, 5
    a = rand(rng, n, n)
    lu = a.copy(order="F")
    piv = np.zeros(n, np.int32)
    orc.dgetrf(n, n, lu, n, piv)
    b = rand(rng, n, nrhs)
    for trans in ("N", "T"):
        x1, x2 = b.copy(order="F"), b.copy(order="F")
        assert orc.dgetrs(trans, n, nrhs, lu, n, piv, x1, n) == 0
        assert refblas.dgetrs(trans, n, nrhs, lu, n, piv, x2, n) == 0
        assert same_bits(x1, x2)
    g = rng.standard_normal((n, n))
    s = np.asfortranarray(g @ g.T / n + np.eye(n))
    orc.dpotrf("L", n, s, n)
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    assert orc.dpotrs("L", n, nrhs, s, n, x1, n) == refblas.dpotrs("L", n, nrhs, s, n, x2, n)
    assert same_bits(x1, x2)
