"""Emulated FP64 GEMM (Ozaki slices on INT8 tensor cores) through the C ABI.

Exactness pins the tensor-core machinery: integer inputs with |a| <= 63 are
exactly one slice, so every slice count must reproduce the exact integer
product; |a| < 2^20 needs slice pairs up to index 2 each (index sum 4), so
S >= 5 is exact. Accuracy: normwise error against the exact product rounded
once, computed on the CPU (tests/exact_ref.py) on sampled entries, next to
the plain FP64 path's error on the same inputs; the library's double-double
product, which the benchmark uses as its yardstick, is itself held to 1 ulp
of the exact value.
"""
import math

import numpy as np
import pytest

from tests.exact_ref import exact_gemm_columns
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


# ---------------------------------------------------------------------------
# The yardstick, the S = 8 bound and the automatic slice count, against the
# exact product on the CPU.

def spread_operands(rng, m, n, k, spread):
    ea = rng.integers(-spread, spread + 1, (m, k))
    eb = rng.integers(-spread, spread + 1, (k, n))
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)) * np.exp2(ea))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)) * np.exp2(eb))
    return a, b


def graded_operands(rng, m, n, k, binades=30):
    """Columns of A and rows of B decaying over `binades` binades along k."""
    g = np.exp2(-binades * np.arange(k) / k)
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)) * g[None, :])
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)) * g[:, None])
    return a, b


@pytest.mark.parametrize("spread", [8, 30])
def test_ddref_within_one_ulp_of_exact(hb, spread):
    """The double-double product that grades the benchmark's accuracy claim
    is within 1 ulp of the exact product rounded once (512 entries, K =
    8192)."""
    rng = np.random.default_rng(40 + spread)
    m, n, k = 256, 16, 8192
    a, b = spread_operands(rng, m, n, k, spread)
    cols = np.array([3, 11], dtype=np.int32)
    dd = np.zeros((m, len(cols)), order="F")
    hb.dgemm_ddref("N", "N", m, k, a, m, b, k, n, cols, dd, m)
    exact = exact_gemm_columns(a, b, cols)
    ulp = np.spacing(np.abs(exact))
    assert np.all(np.abs(dd - exact) <= ulp), np.max(np.abs(dd - exact) / ulp)
    # Most entries are the correctly rounded value itself.
    assert np.mean(dd == exact) > 0.9


@pytest.mark.parametrize("spread", [8, 30])
def test_emulated_s8_elementwise_bound(hb, orc, spread):
    """S = 8 meets the reference tests' element-wise GEMM bound
    |C - C_ref| <= 4 (k + 2) eps (|A| |B|) against the oracle's FP64 dgemm
    (the bound form of tests/gemm_test.cc:98-103), and its normwise error
    against the exact product is below the plain FP64 path's."""
    rng = np.random.default_rng(50 + spread)
    m, n, k = 512, 512, 8192
    a, b = spread_operands(rng, m, n, k, spread)
    c = np.zeros((m, n), order="F")
    assert hb.dgemm_emulated("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, 8) == 8
    ref = np.zeros((m, n), order="F")
    orc.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, ref, m)
    absab = np.zeros((m, n), order="F")
    aa, ab = np.asfortranarray(np.abs(a)), np.asfortranarray(np.abs(b))
    orc.dgemm("N", "N", m, n, k, 1.0, aa, m, ab, k, 0.0, absab, m)
    eps = np.finfo(np.float64).eps
    assert np.all(np.abs(c - ref) <= 4 * (k + 2) * eps * absab)
    plain = np.zeros((m, n), order="F")
    hb.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, plain, m)
    assert same_bits(plain, ref)
    rows = np.arange(0, m, 2)
    cols = [7, 300]
    exact = exact_gemm_columns(a, b, cols, rows=rows)
    err_e = np.linalg.norm(c[np.ix_(rows, cols)] - exact) / np.linalg.norm(exact)
    err_p = np.linalg.norm(plain[np.ix_(rows, cols)] - exact) / np.linalg.norm(exact)
    assert err_e <= err_p / 4, (err_e, err_p)


def auto_slices_rule(a, b):
    """CPU restatement of the library's automatic slice count: beta = log2(rho)
    / 2 with rho = K sum_i 4^(e_i - E) sum_j 4^(f_j - F) / sum_p
    (sum_i (a_ip 2^-E)^2)(sum_j (b_pj 2^-F)^2); the smallest S with
    2^(beta + 52.57 - 8 S + max(0, (8 - log2 K) / 2)) + 0.04 <= 1/2, else 0.
    Also returns the distance of the deciding value from the threshold."""
    k = a.shape[1]
    ea = np.frexp(np.abs(a).max(axis=1))[1]
    fb = np.frexp(np.abs(b).max(axis=0))[1]
    E, F = ea.max(), fb.max()
    sa = np.sum(np.exp2(2.0 * (ea - E)))
    sb = np.sum(np.exp2(2.0 * (fb - F)))
    q = np.sum(np.sum((a * np.exp2(-E)) ** 2, axis=0) * np.sum((b * np.exp2(-F)) ** 2, axis=1))
    beta = 0.5 * math.log2(max(1.0, k * sa * sb / q))
    kterm = max(0.0, 0.5 * (8.0 - math.log2(k)))
    margin = math.inf
    for s in range(1, 9):
        r = 2.0 ** (beta + 52.57 - 8.0 * s + kterm) + 0.04
        margin = min(margin, abs(r - 0.5))
        if r <= 0.5:
            return s, beta, margin
    return 0, beta, margin


AUTO_CASES = [("spread", 0, 64), ("spread", 0, 512), ("spread", 0, 8192),
              ("spread", 8, 512), ("spread", 8, 8192), ("spread", 30, 8192),
              ("graded", 30, 64), ("graded", 30, 8192)]


@pytest.mark.parametrize("kind,spread,k", AUTO_CASES)
def test_auto_slices_from_spread(hb, kind, spread, k):
    """slices = 0 picks the count the rule gives for the data, and the result
    is at least as accurate as the plain FP64 path against the exact product
    (normwise, 1024 sampled entries)."""
    rng = np.random.default_rng(60 + spread + k)
    m, n = 256, 160
    if kind == "spread":
        a, b = spread_operands(rng, m, n, k, spread)
    else:
        a, b = graded_operands(rng, m, n, k, spread)
    want, beta, margin = auto_slices_rule(a, b)
    c = np.zeros((m, n), order="F")
    used = hb.dgemm_emulated("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, 0)
    if margin > 1e-9:
        assert used == want, (used, want, beta)
    assert used in (7, 8), (used, beta)
    plain = np.zeros((m, n), order="F")
    hb.dgemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, plain, m)
    rows = np.arange(0, m, 2)
    cols = [0, 50, 101, 159]
    exact = exact_gemm_columns(a, b, cols, rows=rows)
    err_e = np.linalg.norm(c[np.ix_(rows, cols)] - exact) / np.linalg.norm(exact)
    err_p = np.linalg.norm(plain[np.ix_(rows, cols)] - exact) / np.linalg.norm(exact)
    assert err_e <= err_p, (used, beta, err_e, err_p)


def test_auto_slices_transposed_operands_match(hb):
    """The statistic reads op(A) and op(B) through their strides: the
    transposed forms get the same count and the same bits."""
    rng = np.random.default_rng(77)
    m, n, k = 200, 150, 3000
    a, b = spread_operands(rng, m, n, k, 8)
    c1 = np.zeros((m, n), order="F")
    s1 = hb.dgemm_emulated("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c1, m, 0)
    at, bt = np.asfortranarray(a.T), np.asfortranarray(b.T)
    c2 = np.zeros((m, n), order="F")
    s2 = hb.dgemm_emulated("T", "T", m, n, k, 1.0, at, k, bt, n, 0.0, c2, m, 0)
    assert s1 == s2 == auto_slices_rule(a, b)[0]
    assert same_bits(c1, c2)


def test_auto_slices_too_wide_runs_plain(hb):
    """Products 2^40 below the row and column scales (beta = 40) are beyond 8
    slices: the call runs the plain FP64 path, bit for bit."""
    rng = np.random.default_rng(8)
    m, n, k = 96, 80, 500
    a = np.asfortranarray(rng.uniform(0.5, 1, (m, k)) * 2.0 ** -40)
    a[:, 0] = 1.0
    b = np.asfortranarray(rng.uniform(0.5, 1, (k, n)))
    b[0, :] = 2.0 ** -40
    assert auto_slices_rule(a, b)[0] == 0
    c = rand(rng, m, n)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    assert hb.dgemm_emulated("N", "N", m, n, k, 1.5, a, m, b, k, 0.5, c1, m, 0) == 0
    hb.dgemm("N", "N", m, n, k, 1.5, a, m, b, k, 0.5, c2, m)
    assert same_bits(c1, c2)


@pytest.mark.parametrize("slices,beta", [(0, 0.0), (5, 0.5), (8, 1.0)])
def test_host_c_column_blocks_match_device(hb, cuda, slices, beta):
    """A large host C goes back to the host in column blocks while the next
    block is computed; every element must equal the device-pointer call's
    (same slices, same products), including a ragged last block."""
    torch = cuda
    rng = np.random.default_rng(slices + 7)
    m, n, k = 6000, 6150, 512
    a = np.asfortranarray(rng.uniform(-1, 1, (m, k)) * np.exp2(rng.integers(-8, 9, (m, k))))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)) * np.exp2(rng.integers(-8, 9, (k, n))))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    c_host = c0.copy(order="F")
    used_h = hb.dgemm_emulated("N", "N", m, n, k, 1.25, a, m, b, k, beta, c_host, m, slices)
    da = torch.from_numpy(a.T.copy()).cuda()  # column-major m x k as a k x m row-major block
    db = torch.from_numpy(b.T.copy()).cuda()
    dc = torch.from_numpy(c0.T.copy()).cuda()
    torch.cuda.synchronize()
    used_d = hb.dgemm_emulated("N", "N", m, n, k, 1.25, da, m, db, k, beta, dc, m, slices)
    assert used_h == used_d > 0
    assert same_bits(c_host, dc.cpu().numpy().T)
