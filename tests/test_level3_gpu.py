"""GPU parity of SYMM, SYR2K, GEMMTR (and its alias GEMMT) and TRMM, double
and single precision, through the C ABI against the oracle.

The bar is bit-exact (NaN payloads aside). Inputs follow the reference's
level-3 tests (tests/level3_test.cc:33-475): NaN wherever the routine must
not read (the other triangle of a structured matrix, a unit diagonal, C when
beta = 0), all side/uplo/trans/diag cases, sizes across partial micro-tiles,
KC chunks (256 double, 384 float) and, for TRMM, a triangular operand wider
than one NC block (4080) of the reference's column tiles. Shapes above
m*n*k = 2^22 with m, n >= 32 run on the DMMA tensor-core kernel; smaller ones
on the element-wise kernels.
"""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits, first_diff

pytestmark = pytest.mark.gpu

TRI_CASES = [(s, u, t, d) for s in "LR" for u in "LU" for t in "NT" for d in "NU"]


def structured(rng, n, ld, uplo, dtype, diag="G"):
    """n x n (leading dimension ld): random stored triangle, NaN elsewhere;
    diag "N": |d| near 1.5, "U": NaN (not read), "G": random."""
    a = np.full((ld, max(n, 1)), np.nan, dtype=dtype, order="F")
    r = rng.uniform(-1, 1, (n, n))
    keep = np.tril(np.ones((n, n), bool), -1)
    if uplo == "U":
        keep = keep.T
    a[:n, :n][keep] = r[keep]
    idx = np.arange(n)
    if diag == "N":
        a[idx, idx] = np.where(rng.uniform(size=n) >= 0.5, 1.5, -1.5) + 0.5 * rng.uniform(-1, 1, n)
    elif diag == "G":
        a[idx, idx] = rng.uniform(-1, 1, n)
    return a


def both(hb, orc, p, call_hb, call_orc, out):
    o1, o2 = out.copy(order="F"), out.copy(order="F")
    call_hb(o1)
    assert call_orc(o2) == 0
    assert same_bits(o1, o2), first_diff(o1, o2)


@pytest.mark.parametrize("p", ["d", "s"])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("m,n", [(1, 7), (13, 40), (100, 7), (300, 40), (600, 520)])
def test_symm_bitexact(hb, orc, p, side, uplo, m, n):
    dtype = np.float32 if p == "s" else np.float64
    rng = np.random.default_rng(m * 13 + n)
    ka = m if side == "L" else n
    lda, ldb, ldc = ka + 2, m + 1, m + 3
    a = structured(rng, ka, lda, uplo, dtype)
    b = rand(rng, ldb, n, dtype)
    for alpha, beta in [(1.5, 0.5), (-1.0, 0.0), (0.7, 0.3)]:
        c = rand(rng, ldc, n, dtype)
        if beta == 0.0:
            c[:] = np.nan
        both(hb, orc, p,
             lambda o: hb.symm(p, side, uplo, m, n, alpha, a, lda, b, ldb, beta, o, ldc),
             lambda o: orc.symm(p, side, uplo, m, n, dtype(alpha), a, lda, b, ldb,
                                dtype(beta), o, ldc), c)


@pytest.mark.parametrize("p", ["d", "s"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,k", [(1, 3), (37, 13), (100, 300), (520, 300), (300, 800)])
def test_syr2k_gemmtr_bitexact(hb, orc, p, uplo, trans, n, k):
    dtype = np.float32 if p == "s" else np.float64
    rng = np.random.default_rng(n * 7 + k)
    rows, cols = (n, k) if trans == "N" else (k, n)
    lda = ldb = rows + 1
    ldc = n + 2
    a, b = rand(rng, lda, cols, dtype), rand(rng, ldb, cols, dtype)
    tri = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    for alpha, beta in [(0.75, -0.5), (-1.25, 0.0), (1.0, 0.3), (0.5, 1.0)]:
        c = rand(rng, ldc, n, dtype)
        if beta == 0.0:
            c[:n][tri] = np.nan
        both(hb, orc, p,
             lambda o: hb.syr2k(p, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, o, ldc),
             lambda o: orc.syr2k(p, uplo, trans, n, k, dtype(alpha), a, lda, b, ldb,
                                 dtype(beta), o, ldc), c)
        for ta, tb in [(trans, "T" if trans == "N" else "N"), ("N", "N"), ("T", "T")]:
            ra = n if ta == "N" else k
            rb = k if tb == "N" else n
            aa = rand(rng, ra + 1, k if ta == "N" else n, dtype)
            bb = rand(rng, rb + 1, n if tb == "N" else k, dtype)
            for name in ("gemmtr", "gemmt"):
                both(hb, orc, p,
                     lambda o: hb.gemmtr(p, uplo, ta, tb, n, k, alpha, aa, ra + 1, bb, rb + 1,
                                         beta, o, ldc, name=name),
                     lambda o: orc.gemmtr(p, uplo, ta, tb, n, k, dtype(alpha), aa, ra + 1, bb,
                                          rb + 1, dtype(beta), o, ldc), c)


def run_trmm(hb, orc, p, side, uplo, trans, diag, m, n, alpha, seed, poison=None):
    dtype = np.float32 if p == "s" else np.float64
    rng = np.random.default_rng(seed)
    ka = m if side == "L" else n
    lda, ldb = ka + 1, m + 2
    a = structured(rng, ka, lda, uplo, dtype, diag)
    b = rand(rng, ldb, n, dtype)
    if poison is not None:
        poison(b)
    both(hb, orc, p,
         lambda o: hb.trmm(p, side, uplo, trans, diag, m, n, alpha, a, lda, o, ldb),
         lambda o: orc.trmm(p, side, uplo, trans, diag, m, n, dtype(alpha), a, lda, o, ldb),
         b)


@pytest.mark.parametrize("p", ["d", "s"])
@pytest.mark.parametrize("side,uplo,trans,diag", TRI_CASES)
def test_trmm_bitexact(hb, orc, p, side, uplo, trans, diag):
    shapes = [(1, 19), (37, 19), (300, 19), (11, 300)]
    shapes += [(700, 300)] if side == "L" else [(300, 700)]
    for i, (m, n) in enumerate(shapes):
        run_trmm(hb, orc, p, side, uplo, trans, diag, m, n, (1.5, -1.0)[i % 2], m * 100 + n)


@pytest.mark.parametrize("side,uplo", [("R", "L"), ("R", "U"), ("L", "L"), ("L", "U")])
def test_trmm_wide_triangle(hb, orc, side, uplo):
    """A triangular operand of order 4200 (> NC = 4080): the reference's column
    micro-tiles restart at 4080, so the right-side k ranges change pattern."""
    if side == "R":
        run_trmm(hb, orc, "d", side, uplo, "N", "N", 40, 4200, 0.5, 77)
    else:
        run_trmm(hb, orc, "d", side, uplo, "T", "U", 4200, 40, 0.5, 78)


@pytest.mark.parametrize("p", ["d", "s"])
@pytest.mark.parametrize("side,uplo", [("L", "L"), ("L", "U"), ("R", "L"), ("R", "U")])
@pytest.mark.parametrize("m,n", [(40, 3), (200, 64), (64, 200)])
def test_trmm_nonfinite_micro_tile_ranges(hb, orc, p, side, uplo, m, n):
    """Inf in B meets structural zeros only inside the reference's micro-tile
    k ranges: which elements turn NaN follows src/gemm-inl.h:62-85 exactly."""
    def poison(b):
        if side == "L":
            b[min(m - 1, 20), :] = np.inf
            b[m // 2, : n // 2] = -np.inf
        else:
            b[:, min(n - 1, 5)] = np.inf
            b[: m // 2, n // 2] = np.nan
    run_trmm(hb, orc, p, side, uplo, "N", "N", m, n, 1.0, m + n, poison)


def test_level3_device_pointers(hb, orc):
    """Device (torch CUDA) buffers are used in place."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    m, n = 300, 260
    a = structured(rng, m, m, "L", np.float64, "N")
    b = rand(rng, m, n)
    b_orc = b.copy(order="F")
    ta = torch.from_numpy(a.T.copy()).T.cuda()
    tb = torch.from_numpy(b.T.copy()).T.cuda()
    hb.trmm("d", "L", "L", "N", "N", m, n, -0.5, ta, m, tb, m)
    assert orc.trmm("d", "L", "L", "N", "N", m, n, -0.5, a, m, b_orc, m) == 0
    got = np.asfortranarray(tb.cpu().numpy())
    assert same_bits(got, b_orc), first_diff(got, b_orc)
    c = rand(rng, m, n)
    tc = torch.from_numpy(c.T.copy()).T.cuda()
    hb.symm("d", "L", "L", m, n, 0.5, ta, m, torch.from_numpy(b.T.copy()).T.cuda(), m, 0.3,
            tc, m)
    c_orc = c.copy(order="F")
    assert orc.symm("d", "L", "L", m, n, 0.5, a, m, b, m, 0.3, c_orc, m) == 0
    got = np.asfortranarray(tc.cpu().numpy())
    assert same_bits(got, c_orc), first_diff(got, c_orc)


def test_level3_argument_errors(hb):
    z = np.zeros(64)
    c = np.full(64, 7.0)
    with hb.ErrorCapture() as cap:
        hb.symm("d", "X", "U", 4, 4, 1.0, z, 4, z, 4, 0.0, c, 4)
        hb.symm("d", "L", "U", 4, 4, 1.0, z, 4, z, 3, 0.0, c, 4)
        hb.syr2k("d", "U", "X", 4, 4, 1.0, z, 4, z, 4, 0.0, c, 4)
        hb.syr2k("s", "U", "N", 4, 4, 1.0, z, 4, z, 4, 0.0, c, 3)
        hb.gemmtr("d", "U", "N", "X", 4, 4, 1.0, z, 4, z, 4, 0.0, c, 4)
        hb.gemmtr("d", "U", "N", "N", 4, -1, 1.0, z, 4, z, 4, 0.0, c, 4, name="gemmt")
        hb.trmm("d", "L", "U", "N", "X", 4, 4, 1.0, z, 4, c, 4)
        hb.trmm("s", "R", "U", "N", "N", 4, 5, 1.0, z, 4, c, 4)
    assert cap.errors == [("DSYMM", 1), ("DSYMM", 9), ("DSYR2K", 2), ("SSYR2K", 12),
                          ("DGEMMTR", 3), ("DGEMMT", 5), ("DTRMM", 4), ("STRMM", 9)]
    assert np.all(c == 7.0)
    # Quick returns: alpha = 0 with beta = 1 leaves C; TRMM with alpha = 0
    # zeroes B without reading A.
    nan = np.full(16, np.nan)
    cc = np.arange(16.0)
    hb.symm("d", "L", "U", 4, 4, 0.0, nan, 4, nan, 4, 1.0, cc, 4)
    assert np.array_equal(cc, np.arange(16.0))
    hb.trmm("d", "L", "L", "N", "N", 4, 4, 0.0, nan, 4, cc, 4)
    assert np.all(cc == 0.0)


def test_cblas_level3_layouts(hb, orc):
    """Row-major CBLAS calls equal the column-major transposed problems
    (src/cblas.cc:539-700) and report CBLAS argument positions."""
    rng = np.random.default_rng(11)
    RM, CM = hb.CblasRowMajor, hb.CblasColMajor
    m, n = 45, 70
    # TRMM, side L, lower, row-major: B^T := alpha B^T op(A)^T (right, upper).
    a = np.tril(rng.uniform(-1, 1, (m, m))) + 2 * np.eye(m)   # row-major storage
    b = rng.uniform(-1, 1, (m, n))
    got = np.ascontiguousarray(b)
    hb.cblas_level3("dtrmm", RM, hb.CblasLeft, hb.CblasLower, hb.CblasNoTrans,
                    hb.CblasNonUnit, m, n, 1.25, np.ascontiguousarray(a), m, got, n)
    want = np.asfortranarray(b.T)
    orc.trmm("d", "R", "U", "N", "N", n, m, 1.25, np.asfortranarray(a.T), m, want, n)
    assert same_bits(got.T, want), first_diff(got.T, want)
    # SYMM row-major equals column-major on the transposes.
    s = rng.uniform(-1, 1, (m, m))
    s = s + s.T
    c = rng.uniform(-1, 1, (m, n))
    got = np.ascontiguousarray(c)
    hb.cblas_level3("dsymm", RM, hb.CblasLeft, hb.CblasUpper, m, n, 0.5,
                    np.ascontiguousarray(s), m, np.ascontiguousarray(b), n, 0.3, got, n)
    want = np.asfortranarray(c.T)
    orc.symm("d", "R", "L", n, m, 0.5, np.asfortranarray(s.T), m, np.asfortranarray(b.T), n,
             0.3, want, n)
    assert same_bits(got.T, want), first_diff(got.T, want)
    # SYR2K and GEMMT, row-major.
    k = 33
    x, y = rng.uniform(-1, 1, (m, k)), rng.uniform(-1, 1, (m, k))
    cc = rng.uniform(-1, 1, (m, m))
    got32 = np.ascontiguousarray(cc, np.float32)
    hb.cblas_level3("ssyr2k", RM, hb.CblasLower, hb.CblasNoTrans, m, k, 0.5,
                    np.ascontiguousarray(x, np.float32), k, np.ascontiguousarray(y, np.float32),
                    k, 0.3, got32, m)
    want = np.asfortranarray(cc.T, np.float32)
    orc.syr2k("s", "U", "T", m, k, np.float32(0.5), np.asfortranarray(x.T, np.float32), k,
              np.asfortranarray(y.T, np.float32), k, np.float32(0.3), want, m)
    assert same_bits(got32.T, want), first_diff(got32.T, want)
    got = np.ascontiguousarray(cc)
    hb.cblas_level3("dgemmt", RM, hb.CblasUpper, hb.CblasNoTrans, hb.CblasTrans, m, k, 1.5,
                    np.ascontiguousarray(x), k, np.ascontiguousarray(y), k, 0.0, got, m)
    want = np.asfortranarray(cc.T)
    orc.gemmtr("d", "L", "N", "T", m, k, 1.5, np.asfortranarray(y.T), k,
               np.asfortranarray(x.T), k, 0.0, want, m)
    assert same_bits(got.T, want), first_diff(got.T, want)
    with hb.ErrorCapture() as cap:
        hb.cblas_level3("dtrmm", RM, hb.CblasLeft, hb.CblasLower, hb.CblasNoTrans,
                        hb.CblasNonUnit, -1, n, 1.0, a, m, got, n)
        hb.cblas_level3("dsymm", CM, hb.CblasLeft, hb.CblasUpper, m, -1, 1.0, a, m, b, m,
                        0.0, got, m)
        hb.cblas_level3("dgemmtr", 5, hb.CblasUpper, hb.CblasNoTrans, hb.CblasNoTrans, m, k,
                        1.0, x, m, y, k, 0.0, got, m)
    assert cap.errors == [("cblas_dtrmm", 6), ("cblas_dsymm", 5), ("cblas_dgemmtr", 1)]
