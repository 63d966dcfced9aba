"""GPU parity of the complex GEMM (zgemm_, cgemm_, cblas_zgemm, cblas_cgemm)
through the C ABI against the oracle, bit for bit.

The oracle restates the reference's complex micro-kernel: four real FMA
chains per element and KC chunk, combined as (rr - ii, ir + ri), scaled by
alpha and merged with beta (src/gemm_kernel-inl.h:226-428). Cases: all nine
op pairs (N, T, C), shapes with partial tiles and several KC chunks, alpha
and beta special values (beta 0 with C poisoned), padding, host and device
arrays, row-major CBLAS and the argument checks.
"""
import numpy as np
import pytest

from tests.oracle_lib import creal, same_bits

pytestmark = pytest.mark.gpu

OPS = ["N", "T", "C"]


def crand(rng, rows, cols, dtype):
    return np.asfortranarray((rng.uniform(-1, 1, (rows, cols))
                              + 1j * rng.uniform(-1, 1, (rows, cols))).astype(dtype))


def run(hb, orc, p, ta, tb, m, n, k, alpha, beta, pad=0, seed=0):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(seed)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    lda, ldb, ldc = max(1, ra + pad), max(1, rb + pad), max(1, m + pad)
    a = crand(rng, lda, max(ca, 1), dtype)
    b = crand(rng, ldb, max(cb, 1), dtype)
    c = crand(rng, ldc, max(n, 1), dtype)
    if beta == 0:
        c[:] = np.nan + 1j * np.nan
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    hb.zgemm(p, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c1, ldc)
    assert orc.zgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c2, ldc) == 0
    assert same_bits(creal(c1), creal(c2)), (ta, tb, m, n, k, alpha, beta)


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("ta", OPS)
@pytest.mark.parametrize("tb", OPS)
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 13, 9), (37, 23, 300), (64, 50, 513),
                                   (130, 70, 256)])
def test_zgemm_bitexact(hb, orc, p, ta, tb, m, n, k):
    run(hb, orc, p, ta, tb, m, n, k, 1.5 - 0.5j, 0.25 + 0.75j, pad=2, seed=m + n + k)


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (1.0, 1.0), (-1.0 + 2j, 1.0),
                                        (0.0, 0.5 - 0.5j), (0.0, 1.0), (0.5j, 0.0)])
def test_zgemm_alpha_beta(hb, orc, p, alpha, beta):
    run(hb, orc, p, "N", "C", 45, 33, 270, alpha, beta, seed=5)


def test_zgemm_large_and_device(hb, orc):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(7)
    m, n, k = 300, 260, 700
    a, b, c = (crand(rng, m, k, np.complex128), crand(rng, k, n, np.complex128),
               crand(rng, m, n, np.complex128))
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).T.cuda()  # noqa: E731
    tc = dev(c)
    hb.zgemm("z", "N", "N", m, n, k, 0.75 + 0.25j, dev(a), m, dev(b), k, -0.5j, tc, m)
    c2 = c.copy(order="F")
    assert orc.zgemm("N", "N", m, n, k, 0.75 + 0.25j, a, m, b, k, -0.5j, c2, m) == 0
    assert same_bits(creal(tc.cpu().numpy()), creal(c2))


def test_cblas_zgemm_row_major_and_errors(hb, orc):
    rng = np.random.default_rng(8)
    L = hb.lib()
    m, n, k = 33, 21, 300
    a = rng.uniform(-1, 1, (m, k)) + 1j * rng.uniform(-1, 1, (m, k))  # row-major storage
    b = rng.uniform(-1, 1, (k, n)) + 1j * rng.uniform(-1, 1, (k, n))
    c = rng.uniform(-1, 1, (m, n)) + 1j * rng.uniform(-1, 1, (m, n))
    al = np.array([1.5, -0.25])
    be = np.array([0.5, 0.5])
    got = np.ascontiguousarray(c)
    ac, bc = np.ascontiguousarray(a), np.ascontiguousarray(b)
    L.cblas_zgemm(hb.CblasRowMajor, hb.CblasNoTrans, hb.CblasNoTrans, m, n, k, al.ctypes.data,
                  ac.ctypes.data, k, bc.ctypes.data, n, be.ctypes.data, got.ctypes.data, n)
    # Row-major C^T = B^T A^T as a column-major product (src/cblas.cc:529-535).
    want = np.asfortranarray(c.T)
    assert orc.zgemm("N", "N", n, m, k, 1.5 - 0.25j, np.asfortranarray(b.T), n,
                     np.asfortranarray(a.T), k, 0.5 + 0.5j, want, n) == 0
    assert same_bits(creal(got.T), creal(want))
    z = np.zeros(64, np.complex128)
    with hb.ErrorCapture() as cap:
        L.cblas_zgemm(hb.CblasRowMajor, hb.CblasNoTrans, hb.CblasNoTrans, -1, n, k,
                      al.ctypes.data, z.ctypes.data, k, z.ctypes.data, n, be.ctypes.data,
                      z.ctypes.data, n)
        L.cblas_cgemm(7, hb.CblasNoTrans, hb.CblasNoTrans, m, n, k, al.ctypes.data,
                      z.ctypes.data, k, z.ctypes.data, n, be.ctypes.data, z.ctypes.data, n)
        hb.zgemm("z", "X", "N", 2, 2, 2, 1.0, z, 2, z, 2, 0.0, z, 2)
        hb.zgemm("c", "N", "N", 2, 2, 2, 1.0, z.astype(np.complex64), 1,
                 z.astype(np.complex64), 2, 0.0, z.astype(np.complex64), 2)
    assert cap.errors == [("cblas_zgemm", 4), ("cblas_cgemm", 1), ("ZGEMM", 1),
                          ("CGEMM", 8)]


def test_zgemm_misaligned_device_operand(hb, orc):
    """A device operand whose complex elements start 8 bytes off a 16-byte
    boundary is copied to an aligned buffer before the asynchronous copies."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(9)
    m, n, k = 70, 50, 300
    a, b, c = (crand(rng, m, k, np.complex128), crand(rng, k, n, np.complex128),
               crand(rng, m, n, np.complex128))
    flat = np.zeros(2 * m * k + 1)
    flat[1:] = a.ravel(order="F").view(np.float64)
    ta = torch.from_numpy(flat).cuda()
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).T.cuda()  # noqa: E731
    tc = dev(c)
    hb.zgemm("z", "N", "N", m, n, k, 1.25 - 0.5j, ta.data_ptr() + 8, m, dev(b), k, 0.5, tc, m)
    c2 = c.copy(order="F")
    assert orc.zgemm("N", "N", m, n, k, 1.25 - 0.5j, a, m, b, k, 0.5, c2, m) == 0
    assert same_bits(creal(tc.cpu().numpy()), creal(c2))


CTRI = [(s, u, t, d) for s in "LR" for u in "LU" for t in "NTC" for d in "NU"]


def ctriangle(rng, ka, uplo, diag, dtype):
    """Triangular complex matrix with NaN wherever TRSM must not read."""
    a = np.full((ka, ka), np.nan + 1j * np.nan, dtype=dtype, order="F")
    t = (rng.uniform(-1, 1, (ka, ka)) + 1j * rng.uniform(-1, 1, (ka, ka))) / max(ka, 1)
    keep = np.tril(np.ones((ka, ka), bool), -1)
    if uplo == "U":
        keep = keep.T
    a[keep] = t[keep]
    if diag == "N":
        idx = np.arange(ka)
        a[idx, idx] = (1.5 + rng.uniform(0, 0.5, ka)) * np.exp(1j * rng.uniform(0, 6.28, ka))
    return a


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("side,uplo,trans,diag", CTRI)
def test_ztrsm_bitexact(hb, orc, p, side, uplo, trans, diag):
    dtype = np.complex128 if p == "z" else np.complex64
    for m, n in [(1, 3), (5, 7), (33, 17), (100, 40), (300, 70)]:
        if side == "R":
            m, n = n, m
        rng = np.random.default_rng(m * 31 + n)
        ka = m if side == "L" else n
        a = ctriangle(rng, ka, uplo, diag, dtype)
        b = crand(rng, m + 1, n, dtype)
        for alpha in (1.0, 0.5 - 0.75j):
            b1, b2 = b.copy(order="F"), b.copy(order="F")
            hb.ztrsm(p, side, uplo, trans, diag, m, n, alpha, a, ka, b1, m + 1)
            assert orc.ztrsm(side, uplo, trans, diag, m, n, alpha, a, ka, b2, m + 1) == 0
            assert same_bits(creal(b1), creal(b2)), (m, n, alpha)


@pytest.mark.parametrize("p", ["z", "c"])
def test_ztrsm_diagonal_reciprocals(hb, orc, p):
    """The device's 1/t(j, j) against the C++ runtime's complex quotient (the
    reference's), through diagonal triangles: magnitudes 2^-40..2^40 and
    purely real or imaginary diagonals."""
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(11)
    for trial in range(8):
        r = 32
        d = (rng.uniform(-1, 1, r) * 2.0 ** rng.integers(-40, 40, r)
             + 1j * rng.uniform(-1, 1, r) * 2.0 ** rng.integers(-40, 40, r))
        d[trial % r] = d[trial % r].real
        d[(trial + 5) % r] = 1j * d[(trial + 5) % r].imag
        a = np.asfortranarray(np.diag(d).astype(dtype))
        b = np.asfortranarray(np.ones((50, r), dtype))
        b1, b2 = b.copy(order="F"), b.copy(order="F")
        hb.ztrsm(p, "R", "U", "N", "N", 50, r, 1.0, a, r, b1, 50)
        assert orc.ztrsm("R", "U", "N", "N", 50, r, 1.0, a, r, b2, 50) == 0
        assert same_bits(creal(b1), creal(b2)), trial


def test_ztrsm_device_misaligned_and_cblas(hb, orc):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(13)
    m, n = 90, 40
    a = ctriangle(rng, m, "L", "N", np.complex128)
    b = crand(rng, m, n, np.complex128)
    flat = np.zeros(2 * m * n + 1)
    flat[1:] = b.ravel(order="F").view(np.float64)
    tb = torch.from_numpy(flat).cuda()
    ta = torch.from_numpy(np.ascontiguousarray(a.T)).T.cuda()
    hb.ztrsm("z", "L", "L", "C", "N", m, n, 1.0 - 1.0j, ta, m, tb.data_ptr() + 8, m)
    want = b.copy(order="F")
    assert orc.ztrsm("L", "L", "C", "N", m, n, 1.0 - 1.0j, a, m, want, m) == 0
    got = tb.cpu().numpy()[1:].view(np.complex128).reshape(n, m).T
    assert same_bits(creal(got), creal(want))
    # Row-major CBLAS: B^T := alpha B^T op(A)^T with the other side and triangle.
    L = hb.lib()
    al = np.array([0.5, 0.25])
    brow = np.ascontiguousarray(b)
    arow = np.ascontiguousarray(a)
    L.cblas_ztrsm(hb.CblasRowMajor, hb.CblasLeft, hb.CblasLower, hb.CblasNoTrans,
                  hb.CblasNonUnit, m, n, al.ctypes.data, arow.ctypes.data, m,
                  brow.ctypes.data, n)
    want = np.asfortranarray(b.T)
    assert orc.ztrsm("R", "U", "N", "N", n, m, 0.5 + 0.25j, np.asfortranarray(a.T), m, want,
                     n) == 0
    assert same_bits(creal(brow.T), creal(want))
    with hb.ErrorCapture() as cap:
        hb.ztrsm("z", "X", "L", "N", "N", 2, 2, 1.0, a, 2, b, 2)
        hb.ztrsm("c", "L", "L", "N", "N", 2, 2, 1.0, a.astype(np.complex64), 1,
                 b.astype(np.complex64), 2)
        L.cblas_ztrsm(hb.CblasRowMajor, hb.CblasLeft, hb.CblasLower, hb.CblasNoTrans,
                      hb.CblasNonUnit, -1, n, al.ctypes.data, arow.ctypes.data, m,
                      brow.ctypes.data, n)
    assert cap.errors == [("ZTRSM", 1), ("CTRSM", 9), ("cblas_ztrsm", 6)]


# --------------------------------------------------------------------------
# Complex LU family (zgetrf_, cgetrf_, ...2_, ?laswp_, ?getrs_, ?gesv_)
# against the oracle's restatement of the reference's drivers and leaf, bit
# for bit: shapes around the leaf (16) and the block (64), panels split over
# several CTAs (m > 512), padding, both recursions.

ZLU_SHAPES = [(1, 1), (1, 6), (6, 1), (3, 7), (16, 40), (40, 16), (17, 17), (33, 17),
              (17, 33), (64, 64), (65, 70), (90, 150), (150, 90), (200, 200), (513, 300),
              (1100, 260)]


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("m,n", ZLU_SHAPES)
def test_zgetrf_bitexact(hb, orc, p, recursive, m, n):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(m * 31 + n)
    lda = m + 3
    a = crand(rng, lda, n, dtype)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1 = np.zeros(min(m, n), np.int32)
    p2 = np.zeros(min(m, n), np.int32)
    i1 = hb.zgetrf(p, m, n, a1, lda, p1, recursive=recursive)
    i2 = orc.zgetrf(m, n, a2, lda, p2, recursive=recursive)
    assert i1 == i2 == 0
    assert np.array_equal(p1, p2)
    assert same_bits(creal(a1), creal(a2))
    assert np.array_equal(a1[m:, :], a[m:, :])


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("k", [1, 9, 17, 30])
def test_zgetrf_singular_info(hb, orc, p, recursive, k):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(100 + k)
    m, n = 40, 30
    a = crand(rng, m, n, dtype)
    a[:, k - 1] = 0
    if k < n:
        a[:, n - 1] = 0
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    assert hb.zgetrf(p, m, n, a1, m, p1, recursive=recursive) == k
    assert orc.zgetrf(m, n, a2, m, p2, recursive=recursive) == k
    assert np.array_equal(p1, p2)
    assert same_bits(creal(a1), creal(a2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("n", [5, 40])
def test_zgetrf_tiny_pivots(hb, p, recursive, n):
    """Golden from the reference's TinyPivots test: pivots below the safe
    minimum divide the column (the runtime's complex quotient), L(i, 0) =
    2^-min(i, 20) exactly, no interchanges."""
    dtype = np.complex128 if p == "z" else np.complex64
    rt = np.float64 if p == "z" else np.float32
    tiny = np.finfo(rt).tiny / 4
    a = np.zeros((n, n), dtype, order="F")
    for i in range(n):
        a[i, 0] = np.ldexp(tiny, -min(i, 20))
    for k in range(1, n):
        a[0, k] = 1
        a[k, k] = 4
    ipiv = np.zeros(n, np.int32)
    assert hb.zgetrf(p, n, n, a, n, ipiv, recursive=recursive) == 0
    assert np.array_equal(ipiv, np.arange(1, n + 1))
    for i in range(1, n):
        assert a[i, 0] == np.ldexp(rt(1), -min(i, 20)), i


def test_zgetrf_mixed_magnitudes_and_ties(hb, orc):
    """Pivots decided by |re| + |im| with ties (first index wins), parts of
    very different sizes and tiny complex pivots with both parts nonzero."""
    rng = np.random.default_rng(3)
    n = 48
    a = crand(rng, n, n, np.complex128)
    a[5:12, 0] = 0.5 + 0.5j       # equal magnitudes, several rows
    a[20, 0] = 1.0 + 0j
    a[21, 0] = 0 - 1.0j           # the same |re| + |im|
    a[:, 3] *= 1e-310             # subnormal column: tiny pivots, both parts
    a[:, 7] = a[:, 7].real * 1e200 + 1j * a[:, 7].imag * 1e-200
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    i1 = hb.zgetrf("z", n, n, a1, n, p1)
    i2 = orc.zgetrf(n, n, a2, n, p2)
    assert i1 == i2
    assert np.array_equal(p1, p2)
    assert same_bits(creal(a1), creal(a2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
def test_zgetrs_zgesv_bitexact(hb, orc, p, trans):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(7)
    n, nrhs = 300, 5
    a = crand(rng, n, n, dtype)
    lu = a.copy(order="F")
    ipiv = np.zeros(n, np.int32)
    assert orc.zgetrf(n, n, lu, n, ipiv) == 0
    b = crand(rng, n, nrhs, dtype)
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    assert hb.zgetrs(p, trans, n, nrhs, lu, n, ipiv, b1, n) == 0
    assert orc.zgetrs(trans, n, nrhs, lu, n, ipiv, b2, n) == 0
    assert same_bits(creal(b1), creal(b2))
    if trans == "N":
        a1, a2 = a.copy(order="F"), a.copy(order="F")
        b1, b2 = b.copy(order="F"), b.copy(order="F")
        q1, q2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
        assert hb.zgesv(p, n, nrhs, a1, n, q1, b1, n) == 0
        assert orc.zgesv(n, nrhs, a2, n, q2, b2, n) == 0
        assert np.array_equal(q1, q2)
        assert same_bits(creal(a1), creal(a2)) and same_bits(creal(b1), creal(b2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("incx", [1, -1, 2, -2])
def test_zlaswp(hb, orc, p, incx):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(9)
    lda, n = 50, 37
    a = crand(rng, lda, n, dtype)
    k1, k2 = 3, 20
    ipiv = rng.integers(1, lda + 1, k1 + (k2 - k1) * abs(incx)).astype(np.int32)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    hb.zlaswp(p, n, a1, lda, k1, k2, ipiv, incx)
    orc.zlaswp(n, a2, lda, k1, k2, ipiv, incx)
    assert np.array_equal(a1, a2)


def test_zgetrf_device_arrays_misaligned_and_errors(hb, orc):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(21)
    m, n = 600, 250
    a = crand(rng, m, n, np.complex128)
    want = a.copy(order="F")
    pw = np.zeros(n, np.int32)
    assert orc.zgetrf(m, n, want, m, pw) == 0
    # A device array whose address is 8 bytes past a complex element.
    flat = np.zeros(2 * m * n + 1)
    flat[1:] = a.ravel(order="F").view(np.float64)
    ta = torch.from_numpy(flat).cuda()
    tp = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert hb.zgetrf("z", m, n, ta.data_ptr() + 8, m, tp) == 0
    got = ta.cpu().numpy()[1:].view(np.complex128).reshape(n, m).T
    assert np.array_equal(tp.cpu().numpy(), pw)
    assert same_bits(creal(got), creal(want))
    # Aligned device arrays (complex64) and the solve on them.
    a32 = crand(rng, 200, 200, np.complex64)
    b32 = crand(rng, 200, 2, np.complex64)
    wa, wb, wp = a32.copy(order="F"), b32.copy(order="F"), np.zeros(200, np.int32)
    assert orc.zgesv(200, 2, wa, 200, wp, wb, 200) == 0
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).T.cuda()  # noqa: E731
    da, db = dev(a32), dev(b32)
    dp = torch.zeros(200, dtype=torch.int32, device="cuda")
    assert hb.zgesv("c", 200, 2, da, 200, dp, db, 200) == 0
    assert same_bits(creal(np.asfortranarray(da.cpu().numpy())), creal(wa))
    assert same_bits(creal(np.asfortranarray(db.cpu().numpy())), creal(wb))
    z = np.zeros((4, 4), np.complex128, order="F")
    ip = np.zeros(4, np.int32)
    assert hb.zgetrf("z", 0, 4, z, 1, ip) == 0
    with hb.ErrorCapture() as cap:
        assert hb.zgetrf("z", -1, 4, z, 4, ip) == -1
        assert hb.zgetrf("c", 4, -2, z.astype(np.complex64), 4, ip) == -2
        assert hb.zgetrf("z", 4, 4, z, 3, ip, recursive=True) == -4
        assert hb.zgetrs("z", "X", 4, 1, z, 4, ip, z, 4) == -1
        assert hb.zgetrs("c", "N", 4, 1, z.astype(np.complex64), 4, ip,
                         z.astype(np.complex64), 3) == -8
        assert hb.zgesv("z", 4, -1, z, 4, ip, z, 4) == -2
    assert cap.errors == [("ZGETRF", 1), ("CGETRF", 2), ("ZGETRF2", 4), ("ZGETRS", 1),
                          ("CGETRS", 8), ("ZGESV", 2)]


# --------------------------------------------------------------------------
# Complex Cholesky family (zpotrf_, cpotrf_, ...2_, ?potrs_, ?posv_) and the
# complex HERK it updates with, against the oracle bit for bit.

def _hpd(rng, n, dtype):
    g = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = g @ g.conj().T / n + 1e-3 * np.eye(n)
    h += 1j * np.diag(rng.uniform(-1, 1, n))  # an imaginary diagonal is ignored
    return np.asfortranarray(h.astype(dtype))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("n", [1, 7, 32, 33, 64, 65, 130, 257, 600])
def test_zpotrf_bitexact(hb, orc, p, uplo, recursive, n):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(n * 3 + (uplo == "U"))
    lda = n + 2
    a = crand(rng, lda, n, dtype)  # the other triangle and the padding are garbage
    a[:n, :] = np.where(np.tril(np.ones((n, n), bool)) if uplo == "L"
                        else np.triu(np.ones((n, n), bool)), _hpd(rng, n, dtype), a[:n, :])
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    i1 = hb.zpotrf(p, uplo, n, a1, lda, recursive=recursive)
    i2 = orc.zpotrf(uplo, n, a2, lda, recursive=recursive)
    assert i1 == i2 == 0
    assert same_bits(creal(a1), creal(a2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("uplo", ["U", "L"])
def test_zpotrf_not_positive_definite(hb, orc, p, uplo):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(17)
    n = 200
    for bad in (1, 33, 70, 200):
        a = _hpd(rng, n, dtype)
        a[bad - 1, bad - 1] = -1.0
        a1, a2 = a.copy(order="F"), a.copy(order="F")
        i1 = hb.zpotrf(p, uplo, n, a1, n)
        i2 = orc.zpotrf(uplo, n, a2, n)
        assert i1 == i2 and 0 < i1 <= bad
        assert same_bits(creal(a1), creal(a2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "C"])
@pytest.mark.parametrize("n,k,alpha,beta", [(45, 300, -0.75, 0.5), (70, 600, 1.0, 1.0),
                                            (33, 20, -1.0, 0.0), (64, 0, 2.0, 0.25),
                                            (40, 10, 0.0, -2.0)])
def test_zherk_bitexact(hb, orc, p, uplo, trans, n, k, alpha, beta):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(n + k)
    rows = n if trans == "N" else k
    a = crand(rng, max(rows, 1), max(k if trans == "N" else n, 1), dtype)
    c = crand(rng, n, n, dtype)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    hb.zherk(p, uplo, trans, n, k, alpha, a, max(rows, 1), beta, c1, n)
    assert orc.zherk(uplo, trans, n, k, alpha, a, max(rows, 1), beta, c2, n) == 0
    assert same_bits(creal(c1), creal(c2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("uplo", ["U", "L"])
def test_zpotrs_zposv_bitexact(hb, orc, p, uplo):
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(23)
    n, nrhs = 300, 4
    a = _hpd(rng, n, dtype)
    b = crand(rng, n, nrhs, dtype)
    f = a.copy(order="F")
    assert orc.zpotrf(uplo, n, f, n) == 0
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    assert hb.zpotrs(p, uplo, n, nrhs, f, n, b1, n) == 0
    assert orc.zpotrs(uplo, n, nrhs, f, n, b2, n) == 0
    assert same_bits(creal(b1), creal(b2))
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    assert hb.zposv(p, uplo, n, nrhs, a1, n, b1, n) == 0
    assert orc.zposv(uplo, n, nrhs, a2, n, b2, n) == 0
    assert same_bits(creal(a1), creal(a2)) and same_bits(creal(b1), creal(b2))


def test_zpotrf_device_misaligned_and_errors(hb, orc):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(29)
    n = 400
    a = _hpd(rng, n, np.complex128)
    want = a.copy(order="F")
    assert orc.zpotrf("L", n, want, n) == 0
    flat = np.zeros(2 * n * n + 1)
    flat[1:] = a.ravel(order="F").view(np.float64)
    ta = torch.from_numpy(flat).cuda()
    assert hb.zpotrf("z", "L", n, ta.data_ptr() + 8, n) == 0
    got = ta.cpu().numpy()[1:].view(np.complex128).reshape(n, n).T
    assert same_bits(creal(got), creal(want))
    z = np.zeros((4, 4), np.complex128, order="F")
    assert hb.zpotrf("z", "L", 0, z, 1) == 0
    with hb.ErrorCapture() as cap:
        assert hb.zpotrf("z", "X", 4, z, 4) == -1
        assert hb.zpotrf("c", "U", 4, z.astype(np.complex64), 3, recursive=True) == -4
        assert hb.zposv("z", "L", 4, -1, z, 4, z, 4) == -3
        assert hb.zpotrs("c", "U", 4, 1, z.astype(np.complex64), 4,
                         z.astype(np.complex64), 2) == -7
        hb.zherk("z", "L", "T", 4, 4, 1.0, z, 4, 1.0, z, 4)
        hb.zherk("c", "U", "N", 4, 4, 1.0, z.astype(np.complex64), 3, 1.0,
                 z.astype(np.complex64), 4)
    assert cap.errors == [("ZPOTRF", 1), ("CPOTRF2", 4), ("ZPOSV", 3), ("CPOTRS", 7),
                          ("ZHERK", 2), ("CHERK", 7)]


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.3 - 0.2j])
def test_complex_split_chunks_bitexact(hb, orc, p, beta):
    """Few output tiles and many KC chunks: the chunks run in parallel and
    merge in order, which must give the sequential result. The first chunk's
    merge stores (beta 0), adds (beta 1) or applies a general beta."""
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(41)
    m, n, k = 100, 70, 3000
    a, b, c = crand(rng, m, k, dtype), crand(rng, k, n, dtype), crand(rng, m, n, dtype)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    hb.zgemm(p, "N", "N", m, n, k, 0.5 - 1.0j, a, m, b, k, beta, c1, m)
    assert orc.zgemm("N", "N", m, n, k, 0.5 - 1.0j, a, m, b, k, beta, c2, m) == 0
    assert same_bits(creal(c1), creal(c2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "C"])
@pytest.mark.parametrize("beta", [0.0, 0.5, 1.0])
def test_complex_split_chunks_herk_bitexact(hb, orc, p, uplo, trans, beta):
    """HERK on a 64 x 64 triangle with k = 4096: the split's first chunk
    applies beta on the crossing tiles, the later chunks add with beta 1."""
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(42)
    n, k = 64, 4096
    h = crand(rng, n, k, dtype) if trans == "N" else crand(rng, k, n, dtype)
    ldh = h.shape[0]
    d = crand(rng, n, n, dtype)
    d1, d2 = d.copy(order="F"), d.copy(order="F")
    hb.zherk(p, uplo, trans, n, k, -1.0, h, ldh, beta, d1, n)
    assert orc.zherk(uplo, trans, n, k, -1.0, h, ldh, beta, d2, n) == 0
    assert same_bits(creal(d1), creal(d2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("m", [7000, 8700])
def test_zgetrf_tall_panels_bitexact(hb, orc, p, recursive, m):
    """Narrow panels over many CTAs of 512 rows: m = 7000 runs the cluster
    variant with 14 CTAs exchanging candidates through distributed shared
    memory, m = 8700 (17 CTAs, beyond the 16-CTA cluster) the cooperative
    variant with polled global slots."""
    dtype = np.complex128 if p == "z" else np.complex64
    n = 20
    rng = np.random.default_rng(m + n)
    a = crand(rng, m, n, dtype)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    i1 = hb.zgetrf(p, m, n, a1, m, p1, recursive=recursive)
    i2 = orc.zgetrf(m, n, a2, m, p2, recursive=recursive)
    assert i1 == i2 == 0
    assert np.array_equal(p1, p2)
    assert same_bits(creal(a1), creal(a2))


@pytest.mark.parametrize("p", ["z", "c"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "C"])
def test_cblas_zherk_layouts(hb, orc, p, uplo, trans):
    """Row-major CBLAS HERK is the column-major HERK of the transposed
    storage with the other triangle and N <-> C (src/cblas.cc:610-630)."""
    dtype = np.complex128 if p == "z" else np.complex64
    rng = np.random.default_rng(51)
    n, k = 70, 300
    L = hb.lib()
    fn = L.cblas_zherk if p == "z" else L.cblas_cherk
    cu = hb.CblasUpper if uplo == "U" else hb.CblasLower
    ct = hb.CblasNoTrans if trans == "N" else hb.CblasConjTrans
    rows, cols = (n, k) if trans == "N" else (k, n)
    a = crand(rng, rows, cols, dtype)
    c = crand(rng, n, n, dtype)
    # Column-major.
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    fn(hb.CblasColMajor, cu, ct, n, k, -0.5, a.ctypes.data, rows, 0.25, c1.ctypes.data, n)
    assert orc.zherk(uplo, trans, n, k, -0.5, a, rows, 0.25, c2, n) == 0
    assert same_bits(creal(c1), creal(c2))
    # Row-major: the same storage read as the transpose.
    arow = np.ascontiguousarray(a)
    crow = np.ascontiguousarray(c)
    fn(hb.CblasRowMajor, cu, ct, n, k, -0.5, arow.ctypes.data, cols, 0.25, crow.ctypes.data, n)
    want = np.asfortranarray(c.T)
    other = "L" if uplo == "U" else "U"
    flip = "C" if trans == "N" else "N"
    assert orc.zherk(other, flip, n, k, -0.5, np.asfortranarray(a.T), cols, 0.25, want, n) == 0
    assert same_bits(creal(crow.T), creal(want))
    with hb.ErrorCapture() as cap:
        fn(hb.CblasColMajor, cu, hb.CblasTrans, n, k, 1.0, a.ctypes.data, rows, 1.0,
           c1.ctypes.data, n)
        fn(hb.CblasRowMajor, cu, ct, n, k, 1.0, arow.ctypes.data, cols, 1.0,
           crow.ctypes.data, n - 1)
    name = "cblas_zherk" if p == "z" else "cblas_cherk"
    assert cap.errors == [(name, 3), (name, 11)]
