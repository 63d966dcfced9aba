"""GPU parity of the level-3 BLAS path through the C ABI against the oracle.

The oracle reproduces the reference's per-element rounding, so the bar here is
bit-exact (NaN payloads aside): GEMM (tests/gemm_test.cc shapes, edge tiles,
blocked shapes across KC, alpha/beta special values, padding, NaN/Inf
propagation as tests/semantics_test.cc:93-139), TRSM over all
side/uplo/trans/diag and the sizes of tests/level3_test.cc:522-538, SYRK,
IAMAX, CBLAS layouts and the xerbla positions.
"""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits, first_diff

pytestmark = pytest.mark.gpu


def run_gemm(hb, orc, ta, tb, m, n, k, alpha, beta, pad=0, seed=0, poison_beta0=True,
             special=None):
    rng = np.random.default_rng(seed)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    lda, ldb, ldc = max(1, ra + pad), max(1, rb + pad), max(1, m + pad)
    a = rand(rng, lda, max(ca, 1))
    b = rand(rng, ldb, max(cb, 1))
    c = rand(rng, ldc, max(n, 1))
    if special is not None:
        special(a, b, c)
    if beta == 0.0 and poison_beta0:
        c[:] = np.nan
    c_gpu, c_orc = c.copy(order="F"), c.copy(order="F")
    hb.dgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_gpu, ldc)
    orc.dgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_orc, ldc)
    assert same_bits(c_gpu, c_orc), (first_diff(c_gpu, c_orc), ta, tb, m, n, k, alpha,
                                     beta, pad)


@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("tb", ["N", "T"])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 13, 9), (37, 23, 300), (64, 50, 513),
                                   (128, 64, 256), (129, 65, 257), (200, 300, 1000)])
@pytest.mark.parametrize("pad", [0, 3])
def test_dgemm_bitexact_shapes(hb, orc, ta, tb, m, n, k, pad):
    run_gemm(hb, orc, ta, tb, m, n, k, 1.5, 0.5, pad=pad, seed=m * 7 + n + k)


@pytest.mark.parametrize("alpha", [0.0, 1.0, -1.0, 0.5])
@pytest.mark.parametrize("beta", [0.0, 1.0, -1.0, 0.5])
@pytest.mark.parametrize("k", [0, 5, 300])
def test_dgemm_alpha_beta_special(hb, orc, alpha, beta, k):
    run_gemm(hb, orc, "N", "T", 37, 23, k, alpha, beta, pad=2, seed=1000 + k)


@pytest.mark.parametrize("m,n,k,pad,alpha,beta", [
    (2000, 1500, 64, 0, -1.0, 1.0),   # the LU's trailing update
    (1999, 1501, 33, 1, 1.5, 0.5),    # ragged tiles, odd k
    (4097, 1100, 1, 1, 0.7, -0.3),
    (1000, 4160, 64, 2, 1.0, 0.0),    # beta 0: C not read (poisoned)
    (640, 700, 17, 0, 0.0, 1.0),
    (3001, 2500, 64, 0, -1.0, 1.0),   # odd leading dimension: the tile kernel
])
def test_dgemm_short_k(hb, orc, m, n, k, pad, alpha, beta):
    """k <= 64 (one reference chunk) on the short-product kernel: persistent
    CTAs over 64 x 64 tiles with the next tile's operands prefetched; the
    same chains and merges as the reference."""
    run_gemm(hb, orc, "N", "N", m, n, k, alpha, beta, pad=pad, seed=m + n + k)


def test_dgemm_short_k_special_values(hb, orc):
    def special(a, b, c):
        a[5, 3] = np.inf
        b[3, 40] = np.nan
        c[100, 7] = -np.inf
        a[70, 0] = -0.0
    run_gemm(hb, orc, "N", "N", 1500, 1200, 64, -1.0, 1.0, seed=9, special=special)


def test_dgemm_config_1024(hb, orc):
    """M=N=K=1024 NN, alpha=1.5, beta=0.5 (the reference-runnable config)."""
    run_gemm(hb, orc, "N", "N", 1024, 1024, 1024, 1.5, 0.5, seed=1)


def test_dgemm_persistent_many_tiles_repeated(hb, orc):
    """The LU trailing-update shape at n = 8192 (8128^2 x 64, ~55 tiles per
    persistent CTA, the shared-memory ring reused across tiles), four times:
    every run bit-identical to the oracle. This shape exposed a stale-stage
    read (generic reads vs TMA rewrites of the ring without a proxy fence)."""
    import os
    rng = np.random.default_rng(77)
    m = n = 8128
    k = 64
    a, b, c = rand(rng, m, k), rand(rng, k, n), rand(rng, m, n)
    c_orc = c.copy(order="F")
    orc.set_threads(os.cpu_count() or 8)
    orc.dgemm("N", "N", m, n, k, -1.0, a, m, b, k, 1.0, c_orc, m)
    for _ in range(4):
        c_gpu = c.copy(order="F")
        hb.dgemm("N", "N", m, n, k, -1.0, a, m, b, k, 1.0, c_gpu, m)
        assert same_bits(c_gpu, c_orc), first_diff(c_gpu, c_orc)


@pytest.mark.parametrize("kind", ["nan_a", "inf_b", "inf_times_zero", "nan_c"])
def test_dgemm_special_values(hb, orc, kind):
    def special(a, b, c):
        if kind == "nan_a":
            a[3, 5] = np.nan
        elif kind == "inf_b":
            b[5, 2] = np.inf
            b[7, 9] = -np.inf
        elif kind == "inf_times_zero":
            a[:, 4] = 0.0
            b[4, :] = np.inf
        else:
            c[2, 2] = np.nan
    for beta in (0.0, 1.0, 0.5):
        run_gemm(hb, orc, "N", "N", 40, 30, 20, 1.0, beta, seed=3, special=special,
                 poison_beta0=False)


def test_dgemm_padding_untouched_and_device_pointers(hb, orc, cuda):
    torch = cuda
    rng = np.random.default_rng(5)
    m, n, k, pad = 70, 50, 300, 5
    a = rand(rng, m + pad, k)
    b = rand(rng, k + pad, n)
    c = rand(rng, m + pad, n)
    c0 = c.copy(order="F")
    orc_c = c.copy(order="F")
    orc.dgemm("N", "N", m, n, k, 1.5, a, m + pad, b, k + pad, 0.5, orc_c, m + pad)
    da = torch.from_numpy(a.ravel(order="F")).cuda()
    db = torch.from_numpy(b.ravel(order="F")).cuda()
    dc = torch.from_numpy(c.ravel(order="F")).cuda()
    hb.dgemm("N", "N", m, n, k, 1.5, da, m + pad, db, k + pad, 0.5, dc, m + pad)
    out = dc.cpu().numpy().reshape((m + pad, n), order="F")
    assert same_bits(out, orc_c)
    assert same_bits(out[m:, :], c0[m:, :])
    # Host pointers: padding rows untouched as well.
    hb.dgemm("N", "N", m, n, k, 1.5, a, m + pad, b, k + pad, 0.5, c, m + pad)
    assert same_bits(c, orc_c)


def test_dgemm_empty_and_invalid(hb):
    c = np.full(4, 7.0)
    a = np.ones(4)
    hb.dgemm("N", "N", 0, 2, 2, 1.0, a, 1, a, 2, 0.0, c, 1)
    hb.dgemm("N", "N", 2, 0, 2, 1.0, a, 2, a, 2, 0.0, c, 2)
    with hb.ErrorCapture() as cap:
        hb.dgemm("X", "N", 2, 2, 2, 1.0, a, 2, a, 2, 1.0, c, 2)
        hb.dgemm("N", "Y", 2, 2, 2, 1.0, a, 2, a, 2, 1.0, c, 2)
        hb.dgemm("N", "N", -1, 2, 2, 1.0, a, 2, a, 2, 1.0, c, 2)
        hb.dgemm("N", "N", 2, -1, 2, 1.0, a, 2, a, 2, 1.0, c, 2)
        hb.dgemm("N", "N", 2, 2, -1, 1.0, a, 2, a, 2, 1.0, c, 2)
        hb.dgemm("N", "N", 2, 2, 2, 1.0, a, 1, a, 2, 1.0, c, 2)
        hb.dgemm("N", "N", 2, 2, 2, 1.0, a, 2, a, 1, 1.0, c, 2)
        hb.dgemm("N", "N", 2, 2, 2, 1.0, a, 2, a, 2, 1.0, c, 1)
    assert cap.errors == [("DGEMM", p) for p in (1, 2, 3, 4, 5, 8, 10, 13)]
    assert np.all(c == 7.0)


def test_sgemm_bitexact(hb, orc):
    rng = np.random.default_rng(2)
    for (ta, tb, m, n, k) in [("N", "N", 65, 33, 800), ("T", "N", 20, 70, 384), ("N", "T", 5, 5, 1)]:
        ra, ca = (m, k) if ta == "N" else (k, m)
        rb, cb = (k, n) if tb == "N" else (n, k)
        a = rand(rng, ra, ca, np.float32)
        b = rand(rng, rb, cb, np.float32)
        c = rand(rng, m, n, np.float32)
        c1, c2 = c.copy(order="F"), c.copy(order="F")
        hb.sgemm(ta, tb, m, n, k, 1.5, a, ra, b, rb, 0.5, c1, m)
        orc.sgemm(ta, tb, m, n, k, 1.5, a, ra, b, rb, 0.5, c2, m)
        assert same_bits(c1, c2), first_diff(c1, c2)


def test_cblas_dgemm_layouts(hb, orc):
    rng = np.random.default_rng(4)
    m, n, k = 33, 21, 300
    a = rng.uniform(-1, 1, (m, k))   # row-major storage (C order)
    b = rng.uniform(-1, 1, (k, n))
    c = rng.uniform(-1, 1, (m, n))
    c_row = np.ascontiguousarray(c)
    hb.cblas_dgemm(hb.CblasRowMajor, hb.CblasNoTrans, hb.CblasNoTrans, m, n, k, 1.5,
                   np.ascontiguousarray(a), k, np.ascontiguousarray(b), n, 0.5, c_row, n)
    # Row-major C^T = B^T A^T as a column-major product (src/cblas.cc:529-535).
    c_ref = np.asfortranarray(c.T)
    orc.dgemm("N", "N", n, m, k, 1.5, np.asfortranarray(b.T), n, np.asfortranarray(a.T),
              k, 0.5, c_ref, n)
    assert same_bits(c_row, np.ascontiguousarray(c_ref.T))
    with hb.ErrorCapture() as cap:
        hb.cblas_dgemm(hb.CblasRowMajor, hb.CblasNoTrans, hb.CblasNoTrans, -1, n, k, 1.0,
                       a, k, b, n, 0.0, c_row, n)
        hb.cblas_dgemm(hb.CblasColMajor, hb.CblasNoTrans, hb.CblasNoTrans, -1, n, k, 1.0,
                       a, k, b, n, 0.0, c_row, n)
        hb.cblas_dgemm(7, hb.CblasNoTrans, hb.CblasNoTrans, m, n, k, 1.0, a, k, b, n,
                       0.0, c_row, n)
    assert cap.errors == [("cblas_dgemm", 4), ("cblas_dgemm", 4), ("cblas_dgemm", 1)]


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("m", [1, 2, 5, 31, 32, 33, 100, 300])
def test_dtrsm_bitexact(hb, orc, side, uplo, trans, diag, m):
    rng = np.random.default_rng(m + 17)
    n = 7 if m < 100 else 40
    ka = m if side == "L" else n
    lda = ka + 1
    a = rand(rng, lda, ka)
    a[:ka, :ka] = a[:ka, :ka] / ka + np.diag(1.5 + rng.uniform(0, 1, ka))
    # Unreferenced triangle (and unit diagonal) poisoned with NaN.
    tri = np.tril(np.ones((ka, ka), bool)) if uplo == "L" else np.triu(np.ones((ka, ka), bool))
    if diag == "U":
        np.fill_diagonal(tri, False)
    a[:ka, :ka][~tri] = np.nan
    b = rand(rng, m + 2, n)
    for alpha in (1.0, 0.75):
        x1, x2 = b.copy(order="F"), b.copy(order="F")
        hb.dtrsm(side, uplo, trans, diag, m, n, alpha, a, lda, x1, m + 2)
        orc.dtrsm(side, uplo, trans, diag, m, n, alpha, a, lda, x2, m + 2)
        assert same_bits(x1, x2), first_diff(x1, x2)
        assert not np.isnan(x1[:m]).any()


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("r,few", [(64, 1), (500, 3), (512, 16), (1100, 2), (613, 16),
                                   (700, 40), (512, 64), (500, 100), (1100, 512),
                                   (512, 1024)])
def test_dtrsm_few_rhs_cooperative(hb, orc, side, uplo, trans, diag, r, few):
    """Up to 1024 right-hand sides: each subtree of at most 512 rows of
    the recursion runs in one cooperative launch (base solves and updates
    with grid barriers between them; right-side updates computed
    transposed; from 32 right-hand sides the updates on the FP64 tensor
    pipe). Bits must equal the oracle's, subtree sizes that are not powers
    of two and problems above one subtree included."""
    rng = np.random.default_rng(r * 31 + few + ord(side) + ord(uplo) * 3 + ord(trans) * 5)
    m, n = (r, few) if side == "L" else (few, r)
    ka = r
    lda = ka + 3
    a = rand(rng, lda, ka)
    a[:ka, :ka] = a[:ka, :ka] / ka + np.diag(1.5 + rng.uniform(0, 1, ka))
    tri = np.tril(np.ones((ka, ka), bool)) if uplo == "L" else np.triu(np.ones((ka, ka), bool))
    if diag == "U":
        np.fill_diagonal(tri, False)
    a[:ka, :ka][~tri] = np.nan
    b = rand(rng, m + 2, n)
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    hb.dtrsm(side, uplo, trans, diag, m, n, 1.0, a, lda, x1, m + 2)
    orc.dtrsm(side, uplo, trans, diag, m, n, 1.0, a, lda, x2, m + 2)
    assert same_bits(x1, x2), first_diff(x1, x2)
    assert not np.isnan(x1[:m]).any()


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("r,many", [(500, 300), (1300, 257), (512, 1500)])
def test_dtrsm_many_rhs_column_owned(hb, orc, uplo, trans, diag, r, many):
    """Left side, at least 256 right-hand sides: each subtree of at most 512
    rows runs with the columns of X split among CTAs (8 a CTA, the last one
    ragged), each walking the whole recursion for its own columns. A 500-row
    upper subtree has a 276-deep update (a KC restart inside it). Bits must
    equal the oracle's."""
    rng = np.random.default_rng(r * 7 + many + ord(uplo) * 3 + ord(trans) * 5 + ord(diag))
    m, n = r, many
    lda = r + 3
    a = rand(rng, lda, r)
    a[:r, :r] = a[:r, :r] / r + np.diag(1.5 + rng.uniform(0, 1, r))
    tri = np.tril(np.ones((r, r), bool)) if uplo == "L" else np.triu(np.ones((r, r), bool))
    if diag == "U":
        np.fill_diagonal(tri, False)
    a[:r, :r][~tri] = np.nan
    b = rand(rng, m + 2, n)
    for alpha in (1.0, -0.5):
        x1, x2 = b.copy(order="F"), b.copy(order="F")
        hb.dtrsm("L", uplo, trans, diag, m, n, alpha, a, lda, x1, m + 2)
        orc.dtrsm("L", uplo, trans, diag, m, n, alpha, a, lda, x2, m + 2)
        assert same_bits(x1, x2), first_diff(x1, x2)
        assert not np.isnan(x1[:m]).any()


def test_dtrsm_config_4096x512(hb, orc):
    """side=L uplo=L trans=N diag=U, M=4096 N=512, U[-1,1] entries (scaled
    off-diagonal, as tests/level3_test.cc:491-494, so that X stays finite)."""
    rng = np.random.default_rng(42)
    m, n = 4096, 512
    a = rand(rng, m, m) / 64.0
    b = rand(rng, m, n)
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    hb.dtrsm("L", "L", "N", "U", m, n, 1.0, a, m, x1, m)
    orc.dtrsm("L", "L", "N", "U", m, n, 1.0, a, m, x2, m)
    assert same_bits(x1, x2), first_diff(x1, x2)


def test_dtrsm_alpha_zero_and_invalid(hb):
    a = np.full(9, np.nan)
    b = np.ones(6)
    hb.dtrsm("L", "L", "N", "N", 3, 2, 0.0, a, 3, b, 3)
    assert np.all(b == 0.0)
    b[:] = 5.0
    with hb.ErrorCapture() as cap:
        hb.dtrsm("X", "L", "N", "N", 3, 2, 1.0, a, 3, b, 3)
        hb.dtrsm("L", "X", "N", "N", 3, 2, 1.0, a, 3, b, 3)
        hb.dtrsm("L", "L", "X", "N", 3, 2, 1.0, a, 3, b, 3)
        hb.dtrsm("L", "L", "N", "X", 3, 2, 1.0, a, 3, b, 3)
        hb.dtrsm("L", "L", "N", "N", -1, 2, 1.0, a, 3, b, 3)
        hb.dtrsm("L", "L", "N", "N", 3, -1, 1.0, a, 3, b, 3)
        hb.dtrsm("L", "L", "N", "N", 3, 2, 1.0, a, 2, b, 3)
        hb.dtrsm("L", "L", "N", "N", 3, 2, 1.0, a, 3, b, 2)
    assert cap.errors == [("DTRSM", p) for p in (1, 2, 3, 4, 5, 6, 9, 11)]
    assert np.all(b == 5.0)


def test_cblas_dtrsm_row_major(hb, orc):
    rng = np.random.default_rng(8)
    m, n = 45, 12
    a = rng.uniform(-1, 1, (m, m)) / m + 2 * np.eye(m)
    b = rng.uniform(-1, 1, (m, n))
    x = np.ascontiguousarray(b)
    hb.cblas_dtrsm(hb.CblasRowMajor, hb.CblasLeft, hb.CblasLower, hb.CblasNoTrans,
                   hb.CblasNonUnit, m, n, 1.0, np.ascontiguousarray(a), m, x, n)
    # Row-major: the other side and triangle on the transposes.
    xt = np.asfortranarray(b.T)
    orc.dtrsm("R", "U", "N", "N", n, m, 1.0, np.asfortranarray(a.T), m, xt, n)
    assert same_bits(x, np.ascontiguousarray(xt.T))


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,k", [(1, 1), (30, 10), (100, 300), (257, 64)])
# beta 0.3: beta*C is inexact, so the crossing-tile merge alpha*acc + beta*C
# (two roundings) differs from fma(C, beta, alpha*acc).
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.5, 0.3])
def test_dsyrk_bitexact(hb, orc, uplo, trans, n, k, beta):
    rng = np.random.default_rng(n + k)
    ra, ca = (n, k) if trans == "N" else (k, n)
    a = rand(rng, ra, ca)
    c = rand(rng, n + 1, n)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    hb.dsyrk(uplo, trans, n, k, -0.75, a, ra, beta, c1, n + 1)
    orc.dsyrk(uplo, trans, n, k, -0.75, a, ra, beta, c2, n + 1)
    assert same_bits(c1, c2), first_diff(c1, c2)


def test_idamax(hb, orc):
    rng = np.random.default_rng(1)
    for n in (1, 2, 7, 1000, 100000):
        x = rng.uniform(-1, 1, n)
        for incx in (1, 2, 3):
            nn = (n + incx - 1) // incx
            assert hb.idamax(nn, x, incx) == orc.idamax(nn, x, incx)
    x = rng.uniform(-1, 1, 5000)
    x[100] = 7.0
    x[4000] = -7.0
    assert hb.idamax(5000, x, 1) == 101
    x[0] = np.nan
    assert hb.idamax(5000, x, 1) == 1
    y = np.array([1.0, np.nan, 5.0, np.nan, -5.0])
    assert hb.idamax(5, y, 1) == 3
    assert hb.idamax(0, y, 1) == 0
    assert hb.idamax(5, y, 0) == 0
    assert hb.cblas_idamax(5, y, 1) == 2
