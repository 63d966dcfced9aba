"""LAPACKE wrappers of the LU and Cholesky drivers through the C ABI.

The reference's LAPACKE layer (src/lapack/lapacke.cc:37-137,
lapacke_linear.cc:22-73, lapacke_symmetric.cc:22-72, lapacke_util.h:418-480)
calls the column-major routine on the caller's arrays, or on transposed
temporaries for row-major ones, so the results must be those of the oracle's
column-major routine on the same logical matrix, bit for bit, in both layouts
and for host and device arrays; plus the layout, leading-dimension and NaN
checks with their return codes and LAPACKE_xerbla messages
(tests/lapack/getrf_test.cc and potrf_test.cc run the same cases through
LAPACKE in both layouts).
"""
import ctypes

import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits, first_diff
from tests.test_oracle_pins import spd

pytestmark = pytest.mark.gpu

ROW, COL = 101, 102


def ptr(a):
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def store(a, layout, ld):
    """The logical matrix a (rows x cols) in the given layout with leading
    dimension ld (padding filled with a marker)."""
    rows, cols = a.shape
    if layout == COL:
        buf = np.full((cols, ld), -7.25, a.dtype)
        buf[:, :rows] = a.T
    else:
        buf = np.full((rows, ld), -7.25, a.dtype)
        buf[:, :cols] = a
    return buf.reshape(-1).copy()


def load(buf, layout, rows, cols, ld):
    if layout == COL:
        return buf.reshape(cols, ld)[:, :rows].T
    return buf.reshape(rows, ld)[:, :cols]


def padding_kept(buf, layout, rows, cols, ld):
    b = buf.reshape(cols, ld) if layout == COL else buf.reshape(rows, ld)
    inner = rows if layout == COL else cols
    return np.all(b[:, inner:] == -7.25)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("recursive", [False, True])
@pytest.mark.parametrize("layout", [ROW, COL])
@pytest.mark.parametrize("m,n", [(1, 1), (33, 20), (20, 33), (100, 100), (257, 130)])
def test_getrf_layouts(hb, orc, prec, recursive, layout, m, n):
    dt = np.float64 if prec == "d" else np.float32
    rng = np.random.default_rng(m * 7 + n)
    a = rand(rng, m, n, dt)
    ld = (n if layout == ROW else m) + 3
    buf = store(a, layout, ld)
    ipiv = np.zeros(min(m, n), np.int32)
    fn = getattr(hb.lib(), f"LAPACKE_{prec}getrf{'2' if recursive else ''}")
    info = fn(layout, m, n, ptr(buf), ld, ptr(ipiv))
    ref = np.asfortranarray(a.copy())
    p2 = np.zeros(min(m, n), np.int32)
    f = getattr(orc, f"{prec}getrf{'2' if recursive else ''}")
    assert info == f(m, n, ref, m, p2)
    assert np.array_equal(ipiv, p2)
    got = load(buf, layout, m, n, ld)
    assert same_bits(np.ascontiguousarray(got), np.ascontiguousarray(ref)), first_diff(got, ref)
    assert padding_kept(buf, layout, m, n, ld)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("layout", [ROW, COL])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_getrs_gesv_layouts(hb, orc, prec, layout, trans):
    dt = np.float64 if prec == "d" else np.float32
    rng = np.random.default_rng(5)
    n, nrhs = 140, 9
    a = rand(rng, n, n, dt)
    b = rand(rng, n, nrhs, dt)
    lu = np.asfortranarray(a.copy())
    piv = np.zeros(n, np.int32)
    assert getattr(orc, f"{prec}getrf")(n, n, lu, n, piv) == 0
    # getrs with the oracle's factors
    lda = n + 1
    ldb = (nrhs if layout == ROW else n) + 2
    abuf, bbuf = store(lu, layout, lda), store(b, layout, ldb)
    a_before = abuf.copy()
    fn = getattr(hb.lib(), f"LAPACKE_{prec}getrs")
    assert fn(layout, trans.encode(), n, nrhs, ptr(abuf), lda, ptr(piv), ptr(bbuf), ldb) == 0
    x = np.asfortranarray(b.copy())
    assert getattr(orc, f"{prec}getrs")(trans, n, nrhs, lu, n, piv, x, n) == 0
    got = np.ascontiguousarray(load(bbuf, layout, n, nrhs, ldb))
    assert same_bits(got, np.ascontiguousarray(x)), first_diff(got, x)
    assert np.array_equal(abuf, a_before)  # A is input only
    # gesv
    abuf, bbuf = store(a, layout, lda), store(b, layout, ldb)
    p1 = np.zeros(n, np.int32)
    fn = getattr(hb.lib(), f"LAPACKE_{prec}gesv")
    assert fn(layout, n, nrhs, ptr(abuf), lda, ptr(p1), ptr(bbuf), ldb) == 0
    a2, x2 = np.asfortranarray(a.copy()), np.asfortranarray(b.copy())
    p2 = np.zeros(n, np.int32)
    assert getattr(orc, f"{prec}gesv")(n, nrhs, a2, n, p2, x2, n) == 0
    assert np.array_equal(p1, p2)
    assert same_bits(np.ascontiguousarray(load(abuf, layout, n, n, lda)),
                     np.ascontiguousarray(a2))
    assert same_bits(np.ascontiguousarray(load(bbuf, layout, n, nrhs, ldb)),
                     np.ascontiguousarray(x2))


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("layout", [ROW, COL])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("recursive", [False, True])
def test_potrf_potrs_posv_layouts(hb, orc, prec, layout, uplo, recursive):
    dt = np.float64 if prec == "d" else np.float32
    rng = np.random.default_rng(8)
    n, nrhs = 130, 6
    a = (spd(rng, n) + (0.1 * np.eye(n) if prec == "s" else 0)).astype(dt)
    b = rand(rng, n, nrhs, dt)
    lda, ldb = n + 2, (nrhs if layout == ROW else n) + 1
    abuf = store(a, layout, lda)
    fn = getattr(hb.lib(), f"LAPACKE_{prec}potrf2" if recursive else f"LAPACKE_{prec}potrf")
    assert fn(layout, uplo.encode(), n, ptr(abuf), lda) == 0
    f = np.asfortranarray(a.copy())
    assert getattr(orc, f"{prec}potrf2" if recursive else f"{prec}potrf")(uplo, n, f, n) == 0
    got = np.ascontiguousarray(load(abuf, layout, n, n, lda))
    assert same_bits(got, np.ascontiguousarray(f)), first_diff(got, f)
    # potrs with those factors
    bbuf = store(b, layout, ldb)
    assert getattr(hb.lib(), f"LAPACKE_{prec}potrs")(layout, uplo.encode(), n, nrhs, ptr(abuf),
                                                      lda, ptr(bbuf), ldb) == 0
    x = np.asfortranarray(b.copy())
    assert getattr(orc, f"{prec}potrs")(uplo, n, nrhs, f, n, x, n) == 0
    assert same_bits(np.ascontiguousarray(load(bbuf, layout, n, nrhs, ldb)),
                     np.ascontiguousarray(x))
    # posv
    abuf, bbuf = store(a, layout, lda), store(b, layout, ldb)
    assert getattr(hb.lib(), f"LAPACKE_{prec}posv")(layout, uplo.encode(), n, nrhs, ptr(abuf),
                                                     lda, ptr(bbuf), ldb) == 0
    a2, x2 = np.asfortranarray(a.copy()), np.asfortranarray(b.copy())
    assert getattr(orc, f"{prec}posv")(uplo, n, nrhs, a2, n, x2, n) == 0
    assert same_bits(np.ascontiguousarray(load(abuf, layout, n, n, lda)),
                     np.ascontiguousarray(a2))
    assert same_bits(np.ascontiguousarray(load(bbuf, layout, n, nrhs, ldb)),
                     np.ascontiguousarray(x2))


@pytest.mark.parametrize("layout", [ROW, COL])
def test_device_arrays(hb, orc, cuda, layout):
    """Device arrays take device temporaries (row-major) or go straight
    through (column-major); the results are the same bits."""
    torch = cuda
    rng = np.random.default_rng(12)
    n, nrhs = 300, 4
    a = rand(rng, n, n)
    b = rand(rng, n, nrhs)
    lda, ldb = n + 5, (nrhs if layout == ROW else n) + 3
    da = torch.from_numpy(store(a, layout, lda)).cuda()
    db = torch.from_numpy(store(b, layout, ldb)).cuda()
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert hb.lib().LAPACKE_dgesv(layout, n, nrhs, ptr(da), lda, ptr(dp), ptr(db), ldb) == 0
    a2, x2 = np.asfortranarray(a.copy()), np.asfortranarray(b.copy())
    p2 = np.zeros(n, np.int32)
    assert orc.dgesv(n, nrhs, a2, n, p2, x2, n) == 0
    assert np.array_equal(dp.cpu().numpy(), p2)
    assert same_bits(np.ascontiguousarray(load(da.cpu().numpy(), layout, n, n, lda)),
                     np.ascontiguousarray(a2))
    assert same_bits(np.ascontiguousarray(load(db.cpu().numpy(), layout, n, nrhs, ldb)),
                     np.ascontiguousarray(x2))
    # A NaN in a device array is found by the device check.
    da[7] = float("nan")
    torch.cuda.synchronize()
    assert hb.lib().LAPACKE_dgetrf(layout, n, n, ptr(da), lda, ptr(dp)) == -4


def test_nan_checks(hb):
    L = hb.lib()
    n = 6
    a = np.eye(n) * 2.0
    b = np.ones(n)
    p = np.zeros(n, np.int32)
    assert L.LAPACKE_get_nancheck() == 1  # on by default
    bad = a.copy()
    bad[2, 3] = np.nan
    assert L.LAPACKE_dgetrf(COL, n, n, ptr(bad.copy()), n, ptr(p)) == -4
    bb = b.copy()
    bb[1] = np.nan
    assert L.LAPACKE_dgesv(COL, n, 1, ptr(a.copy()), n, ptr(p), ptr(bb.copy()), n) == -7
    assert L.LAPACKE_dgetrs(ROW, b"N", n, 1, ptr(bad.copy()), n, ptr(p), ptr(b.copy()),
                            1) == -5
    # Cholesky checks only the referenced triangle.
    lower_nan = a.copy(order="F")
    lower_nan[4, 1] = np.nan  # column-major: row 4, column 1 is in the lower triangle
    assert L.LAPACKE_dpotrf(COL, b"U", n, ptr(lower_nan), n) == 0
    lower_nan2 = a.copy(order="F")
    lower_nan2[4, 1] = np.nan
    assert L.LAPACKE_dpotrf(COL, b"L", n, ptr(lower_nan2), n) == -4
    assert L.LAPACKE_dposv(COL, b"L", n, 1, ptr(a.copy()), n, ptr(bb.copy()), n) == -7
    # _work functions do not check; switching the checks off skips them.
    L.LAPACKE_set_nancheck(0)
    try:
        assert L.LAPACKE_get_nancheck() == 0
        assert L.LAPACKE_dgetrf(COL, n, n, ptr(bad.copy()), n, ptr(p)) != -4
    finally:
        L.LAPACKE_set_nancheck(1)
    assert L.LAPACKE_dgetrf_work(COL, n, n, ptr(bad.copy()), n, ptr(p)) != -4


def test_argument_errors(hb, capfd):
    L = hb.lib()
    a = np.zeros(16)
    p = np.zeros(4, np.int32)
    assert L.LAPACKE_dgetrf(5, 4, 4, ptr(a), 4, ptr(p)) == -1
    assert L.LAPACKE_sgesv(0, 4, 1, ptr(a), 4, ptr(p), ptr(a), 4) == -1
    # Row-major: a leading dimension below the columns.
    assert L.LAPACKE_dgetrf(ROW, 2, 4, ptr(a), 3, ptr(p)) == -5
    assert L.LAPACKE_dgetrs(ROW, b"N", 4, 2, ptr(a), 4, ptr(p), ptr(a), 1) == -9
    assert L.LAPACKE_dposv(ROW, b"U", 4, 1, ptr(a), 3, ptr(a), 1) == -6
    out = capfd.readouterr().out.splitlines()
    assert out == ["Wrong parameter 1 in LAPACKE_dgetrf",
                   "Wrong parameter 1 in LAPACKE_sgesv",
                   "Wrong parameter 5 in LAPACKE_dgetrf_work",
                   "Wrong parameter 9 in LAPACKE_dgetrs_work",
                   "Wrong parameter 6 in LAPACKE_dposv_work"]
    # Column-major: the LAPACK routine's own check, shifted by one.
    with hb.ErrorCapture() as cap:
        assert L.LAPACKE_dgetrf(COL, 4, 4, ptr(a), 3, ptr(p)) == -5
        assert L.LAPACKE_dpotrf(COL, b"X", 4, ptr(a), 4) == -2
        assert L.LAPACKE_dgetrf(ROW, -1, 4, ptr(a), 4, ptr(p)) == -2
    assert cap.errors == [("DGETRF", 4), ("DPOTRF", 1), ("DGETRF", 1)]
