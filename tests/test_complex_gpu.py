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
