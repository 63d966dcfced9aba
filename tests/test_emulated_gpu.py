"""Emulated FP64 GEMM (Ozaki slices on INT8 tensor cores) through the C ABI.

Exactness pins the tensor-core machinery: integer inputs with |a| <= 63 are
exactly one slice, so every slice count must reproduce the exact integer
product; |a| < 2^20 needs slice pairs up to index 2 each (index sum 4), so
S >= 5 is exact. Accuracy: normwise error against a double-double reference
product, next to the plain FP64 path's error on the same inputs.
"""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits

pytestmark = pytest.mark.gpu


def normwise_err(c, ref, a, b):
    return np.linalg.norm(c - ref) / (np.linalg.norm(a) * np.linalg.norm(b))


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (100, 70, 300), (257, 129, 1000),
                                   (64, 200, 17), (1, 1, 1)])
@pytest.mark.parametrize("slices", [1, 2, 4, 8])
def test_emulated_exact_small_integers(hb, m, n, k, slices):
    rng = np.random.default_rng(m + n + k + slices)
    a = np.asfortranarray(rng.integers(-63, 64, (m, k)).astype(np.float64))
    b = np.asfortranarray(rng.integers(-63, 64, (k, n)).astype(np.float64))
    c = np.zeros((m, n), order="F")
    used = hb.dgemm_emulated("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, slices)
    assert used == slices
    exact = (a.astype(np.int64) @ b.astype(np.int64)).astype(np.float64)
    assert np.array_equal(c, exact)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_emulated_exact_wide_integers(hb, ta, tb):
    rng = np.random.default_rng(3)
    m, n, k = 190, 130, 1000
    A = rng.integers(-(2 ** 20) + 1, 2 ** 20, (m, k)).astype(np.float64)
    B = rng.integers(-(2 ** 20) + 1, 2 ** 20, (k, n)).astype(np.float64)
    a = np.asfortranarray(A if ta == "N" else A.T)
    b = np.asfortranarray(B if tb == "N" else B.T)
    c = np.zeros((m, n), order="F")
    used = hb.dgemm_emulated(ta, tb, m, n, k, 1.0, a, a.shape[0], b, b.shape[0], 0.0, c, m, 5)
    assert used == 5
    exact = A.astype(np.int64) @ B.astype(np.int64)
    assert np.array_equal(c, exact.astype(np.float64))


def dd_reference(hb, a, b, m, n, k):
    cols = np.arange(n, dtype=np.int32)
    out = np.zeros((m, n), order="F")
    hb.dgemm_ddref("N", "N", m, k, a, m, b, k, n, cols, out, m)
    return out


@pytest.mark.parametrize("spread", [0, 8, 30])
def test_emulated_accuracy_vs_plain(hb, spread):
    """Normwise error vs a double-double product: S = 8 is within 2x of the
    plain FP64 path, and the error falls with every added slice."""
    rng = np.random.default_rng(spread)
    m, n, k = 256, 192, 2048
    ea = rng.integers(-spread, spread + 1, (m, k)) if spread else 0
    eb = rng.integers(-spread, spread + 1, (k, n)) if spread else 0
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)) * np.exp2(ea))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)) * np.exp2(eb))
    ref = dd_reference(hb, a, b, m, n, k)
    plain = np.zeros((m, n), order="F")
    hb.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, plain, m)
    err_plain = normwise_err(plain, ref, a, b)
    errs = []
    for s in range(3, 9):
        c = np.zeros((m, n), order="F")
        assert hb.dgemm_emulated("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, s) == s
        errs.append(normwise_err(c, ref, a, b))
    assert all(errs[i + 1] < errs[i] for i in range(len(errs) - 1)), errs
    assert errs[-1] <= 2 * err_plain + 1e-300, (errs, err_plain)


def test_emulated_alpha_beta_and_auto(hb):
    rng = np.random.default_rng(9)
    m, n, k = 150, 90, 700
    a, b, c = rand(rng, m, k), rand(rng, k, n), rand(rng, m, n)
    c0 = c.copy(order="F")
    used = hb.dgemm_emulated("N", "N", m, n, k, 1.5, a, m, b, k, 0.5, c, m, 0)
    assert used in (7, 8)
    exp = 1.5 * (a @ b) + 0.5 * c0
    assert np.abs(c - exp).max() < 1e-12
    # beta == 0 does not read C.
    c[:] = np.nan
    hb.dgemm_emulated("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, 8)
    assert np.isfinite(c).all()


def test_emulated_nonfinite_runs_plain_path(hb):
    rng = np.random.default_rng(1)
    m, n, k = 40, 30, 50
    a, b, c = rand(rng, m, k), rand(rng, k, n), rand(rng, m, n)
    a[3, 4] = np.inf
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    assert hb.dgemm_emulated("N", "N", m, n, k, 1.0, a, m, b, k, 0.5, c1, m, 8) == 0
    hb.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.5, c2, m)
    assert same_bits(c1, c2)


def test_emulated_invalid_arguments(hb):
    a = np.ones(4)
    c = np.full(4, 7.0)
    with hb.ErrorCapture() as cap:
        assert hb.dgemm_emulated("X", "N", 2, 2, 2, 1.0, a, 2, a, 2, 0.0, c, 2, 8) == -1
        assert hb.dgemm_emulated("N", "N", 2, 2, 2, 1.0, a, 2, a, 2, 0.0, c, 2, 9) == -1
    assert cap.errors == [("DGEMM_EMULATED", 1), ("DGEMM_EMULATED", 14)]
    assert np.all(c == 7.0)
