"""GPU parity of the inverse routines through the C ABI against the oracle:
?getri_ (src/lapack/getrf.cc:369-483), ?trtri_ and ?trti2_
(src/lapack/triangular.cc:18-166) and their LAPACKE forms, bit for bit.

The oracle's GETRI and TRTRI are pinned against the reference's own driver
sources (tests/test_oracle_pins.py). Cases: the blocked path (lwork = 64 n),
narrowed blocks (lwork = 20 n) and the unblocked path (lwork = n, and every
n <= 64), sizes across the 64-wide blocks and through the DMMA GEMM, NaN
wherever the routine must not read, singular U, workspace queries and
argument errors, host and device arrays.
"""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits, first_diff

pytestmark = pytest.mark.gpu


def lu(orc, rng, n, dtype, lda=None):
    lda = lda or n
    a = rand(rng, lda, n, dtype)
    ipiv = np.zeros(max(n, 1), np.int32)
    f = orc.sgetrf if dtype == np.float32 else orc.dgetrf
    assert f(n, n, a, lda, ipiv) == 0
    return a, ipiv


@pytest.mark.parametrize("p", ["d", "s"])
@pytest.mark.parametrize("n", [1, 2, 5, 33, 64, 65, 100, 200, 300, 1000, 2100])
@pytest.mark.parametrize("lwork_kind", ["opt", "mid", "min"])
def test_getri_bitexact(hb, orc, p, n, lwork_kind):
    if lwork_kind == "min" and n > 1000:
        pytest.skip("the column-by-column path is covered at n <= 1000")
    dtype = np.float32 if p == "s" else np.float64
    rng = np.random.default_rng(n * 7 + len(lwork_kind))
    a, ipiv = lu(orc, rng, n, dtype, lda=n + 3)
    lwork = {"opt": 64 * n, "mid": 20 * n, "min": n}[lwork_kind]
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    w1, w2 = np.zeros(lwork, dtype), np.zeros(lwork, dtype)
    assert hb.getri(p, n, a1, n + 3, ipiv, w1, lwork) == 0
    assert orc.getri(n, a2, n + 3, ipiv, w2, lwork) == 0
    assert same_bits(a1, a2), first_diff(a1, a2)
    assert w1[0] == w2[0]


def test_getri_device_arrays_and_query(hb, orc):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4)
    n = 700
    a, ipiv = lu(orc, rng, n, np.float64)
    ta = torch.from_numpy(a.T.copy()).T.cuda()
    tp = torch.from_numpy(ipiv).cuda()
    tw = torch.zeros(64 * n, dtype=torch.float64, device="cuda")
    assert hb.getri("d", n, ta, n, tp, tw, 64 * n) == 0
    w = np.zeros(64 * n)
    assert orc.getri(n, a, n, ipiv, w, 64 * n) == 0
    got = np.asfortranarray(ta.cpu().numpy())
    assert same_bits(got, a), first_diff(got, a)
    assert tw[0].item() == w[0] == 64 * n
    q = np.zeros(1)
    assert hb.getri("d", n, a, n, ipiv, q, -1) == 0 and q[0] == 64 * n


def test_getri_singular_and_errors(hb, orc):
    n = 70
    a = np.asfortranarray(np.triu(np.ones((n, n))) + np.eye(n))
    a[40, 40] = 0.0
    ipiv = np.arange(1, n + 1, dtype=np.int32)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    w1, w2 = np.full(64 * n, 3.0), np.full(64 * n, 3.0)
    assert hb.getri("d", n, a1, n, ipiv, w1, 64 * n) == 41
    assert orc.getri(n, a2, n, ipiv, w2, 64 * n) == 41
    assert same_bits(a1, a) and same_bits(a2, a)
    assert w1[0] == w2[0] == 64 * n
    w = np.zeros(64 * n)
    with hb.ErrorCapture() as cap:
        assert hb.getri("d", -1, a1, 1, ipiv, w, 1) == -1
        assert hb.getri("d", n, a1, n - 1, ipiv, w, 64 * n) == -3
        assert hb.getri("s", n, a1.astype(np.float32), n, ipiv, w.astype(np.float32),
                        n - 1) == -6
        assert hb.trtri("d", "X", "N", n, a1, n) == -1
        assert hb.trtri("d", "U", "X", n, a1, n) == -2
        assert hb.trtri("s", "U", "N", -2, a1, n) == -3
        assert hb.trtri("d", "L", "N", n, a1, n - 1, unblocked=True) == -5
    assert cap.errors == [("DGETRI", 1), ("DGETRI", 3), ("SGETRI", 6), ("DTRTRI", 1),
                          ("DTRTRI", 2), ("STRTRI", 3), ("DTRTI2", 5)]


def structured(rng, n, lda, uplo, diag, dtype):
    a = np.full((lda, n), np.nan, dtype=dtype, order="F")
    t = rng.uniform(-1, 1, (n, n)) / np.sqrt(max(n, 1))
    keep = np.tril(np.ones((n, n), bool), -1)
    if uplo == "U":
        keep = keep.T
    a[:n][keep] = t[keep]
    if diag == "N":
        a[np.arange(n), np.arange(n)] = 1.0 + rng.uniform(0, 1, n)
    return a


@pytest.mark.parametrize("p", ["d", "s"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("n", [1, 4, 5, 17, 64, 65, 130, 300, 1000])
def test_trtri_bitexact(hb, orc, p, uplo, diag, n):
    dtype = np.float32 if p == "s" else np.float64
    rng = np.random.default_rng(n * 5 + (uplo == "L") * 2 + (diag == "U"))
    lda = n + 2
    a = structured(rng, n, lda, uplo, diag, dtype)
    for unblocked in (False, True):
        if unblocked and n > 300:
            continue
        a1, a2 = a.copy(order="F"), a.copy(order="F")
        assert hb.trtri(p, uplo, diag, n, a1, lda, unblocked=unblocked) == 0
        assert orc.trtri(uplo, diag, n, a2, lda, unblocked=unblocked) == 0
        assert same_bits(a1, a2), (unblocked, first_diff(a1, a2))


def test_trtri_singular(hb):
    n = 100
    a = np.asfortranarray(np.tril(np.ones((n, n))) + np.eye(n))
    a[77, 77] = 0.0
    a1 = a.copy(order="F")
    assert hb.trtri("d", "L", "N", n, a1, n) == 78
    assert same_bits(a1, a)
    # Unit diagonal: the zero is not read.
    assert hb.trtri("d", "L", "U", n, a1, n) == 0


@pytest.mark.parametrize("p", ["d", "s"])
def test_lapacke_getri_trtri_layouts(hb, orc, p):
    """Row-major LAPACKE calls equal the column-major routine on the
    transposed data (lapacke_linear.cc:75-96, 276-298); NaN checks return
    the argument position; LAPACKE_?getri_work answers a query."""
    dtype = np.float32 if p == "s" else np.float64
    L = hb.lib()
    ROW, COL = 101, 102
    rng = np.random.default_rng(9)
    n = 150
    a, ipiv = lu(orc, rng, n, dtype)
    want = a.copy(order="F")
    w = np.zeros(64 * n, dtype)
    assert orc.getri(n, want, n, ipiv, w, 64 * n) == 0
    fn = getattr(L, f"LAPACKE_{p}getri")
    row = np.ascontiguousarray(a)                 # the same matrix, row-major
    assert fn(ROW, n, row.ctypes.data, n, ipiv.ctypes.data) == 0
    assert same_bits(row, want), first_diff(row, want)
    col = a.copy(order="F")
    assert fn(COL, n, col.ctypes.data, n, ipiv.ctypes.data) == 0
    assert same_bits(col, want)
    q = np.zeros(1, dtype)
    fw = getattr(L, f"LAPACKE_{p}getri_work")
    assert fw(ROW, n, row.ctypes.data, n, ipiv.ctypes.data, q.ctypes.data, -1) == 0
    assert q[0] == 64 * n
    bad = a.copy(order="F")
    bad[3, 5] = np.nan
    assert fn(COL, n, bad.ctypes.data, n, ipiv.ctypes.data) == -3
    # TRTRI, upper, row-major: the upper triangle of the row-major matrix.
    t = structured(rng, n, n, "U", "N", dtype)
    trow = np.ascontiguousarray(t[:n])            # the same matrix, row-major
    want = np.asfortranarray(t[:n].copy())
    assert orc.trtri("U", "N", n, want, n) == 0
    ft = getattr(L, f"LAPACKE_{p}trtri")
    assert ft(ROW, b"U", b"N", n, trow.ctypes.data, n) == 0
    tri = np.triu(np.ones((n, n), bool))
    assert same_bits(trow[tri], want[tri]), first_diff(trow[tri], want[tri])
    # A NaN in the unread (lower) part is no error; one on a unit diagonal
    # is not looked at either.
    t2 = np.ascontiguousarray(structured(rng, n, n, "U", "U", dtype)[:n])
    assert ft(ROW, b"U", b"U", n, t2.ctypes.data, n) == 0
    t3 = np.ascontiguousarray(structured(rng, n, n, "U", "N", dtype)[:n])
    t3[2, 7] = np.nan
    assert ft(ROW, b"U", b"N", n, t3.ctypes.data, n) == -5
