"""Mixed-precision dgesv / dposv (LAPACK DSGESV / DSPOSV semantics) through
the C ABI.

The reference has no mixed-precision solver, so the checks are stated
against its FP64 routines (the oracle): the refined solution's normwise
forward error is at most that of the oracle's dgesv / dposv solution (within
a factor of 4: both sit at the cond * eps noise level), its residual meets DSGESV's backward criterion, A is left
unchanged, and every path that falls back to FP64 (non-finite A, a singular
or indefinite matrix, no convergence) gives bit for bit the plain path's
factors and solution. Matrices follow the north-star workload: A = H1 diag(s)
H2 with H1, H2 products of 4 Householder reflectors and s geometric from 1 to
1/cond; SPD A = G G^T / n + 1e-3 I.
"""
import numpy as np
import pytest

from tests.oracle_lib import same_bits

pytestmark = pytest.mark.gpu

EPS = 2.0 ** -53


def householder_matrix(rng, n, cond):
    s = np.geomspace(1.0, 1.0 / cond, n)
    a = np.diag(s)
    for side in range(2):
        for _ in range(4):
            v = rng.standard_normal(n)
            v /= np.linalg.norm(v)
            if side == 0:
                a = a - 2.0 * np.outer(v, v @ a)
            else:
                a = a - 2.0 * np.outer(a @ v, v)
    return np.asfortranarray(a)


def spd_matrix(rng, n):
    g = rng.standard_normal((n, n))
    return np.asfortranarray(g @ g.T / n + 1e-3 * np.eye(n))


def fwd_err(x, xt):
    return np.linalg.norm(x - xt) / np.linalg.norm(xt)


def check_backward(a, x, b, n):
    r = b - a @ x
    anrm = np.abs(a).sum(axis=1).max()
    for q in range(x.shape[1]):
        assert np.abs(r[:, q]).max() <= 4 * np.abs(x[:, q]).max() * anrm * EPS * np.sqrt(n)


@pytest.mark.parametrize("n,nrhs", [(300, 1), (700, 3), (1100, 20)])
@pytest.mark.parametrize("cond", [1e2, 1e6])
def test_dgesv_mixed_accuracy(hb, orc, n, nrhs, cond):
    rng = np.random.default_rng(int(n + nrhs + np.log10(cond)))
    a = householder_matrix(rng, n, cond)
    xt = rng.uniform(-1, 1, (n, nrhs))
    b = np.asfortranarray(a @ xt)
    a_in = a.copy(order="F")
    x = np.zeros((n, nrhs), order="F")
    ipiv = np.zeros(n, np.int32)
    info, it = hb.dgesv_mixed(n, nrhs, a_in, n, ipiv, b, n, x, n)
    assert info == 0 and it >= 1, (info, it)
    assert same_bits(a_in, a)  # A untouched when refinement succeeds
    assert ipiv.min() >= 1 and ipiv.max() <= n
    check_backward(a, x, b, n)
    # The FP64 oracle (the reference's dgesv order).
    a2, x2 = a.copy(order="F"), b.copy(order="F")
    p2 = np.zeros(n, np.int32)
    assert orc.dgesv(n, nrhs, a2, n, p2, x2, n) == 0
    assert fwd_err(x, xt) <= 4.0 * fwd_err(x2, xt) + 1e-15, (fwd_err(x, xt), fwd_err(x2, xt))


def test_dgesv_mixed_many_chains(hb):
    """70 right-hand sides (five 16-column chains of the refinement's
    triangular solves, the last one partial) at n = 2100 (33 row blocks, the
    last partial): same forward-error and backward checks, against the known
    solution."""
    n, nrhs = 2100, 70
    rng = np.random.default_rng(21)
    a = householder_matrix(rng, n, 1e6)
    xt = rng.uniform(-1, 1, (n, nrhs))
    b = np.asfortranarray(a @ xt)
    x = np.zeros((n, nrhs), order="F")
    ipiv = np.zeros(n, np.int32)
    info, it = hb.dgesv_mixed(n, nrhs, a.copy(order="F"), n, ipiv, b, n, x, n)
    assert info == 0 and 1 <= it <= 10, (info, it)
    check_backward(a, x, b, n)
    ref = np.linalg.solve(a, b)
    assert fwd_err(x, xt) <= 4.0 * fwd_err(ref, xt) + 1e-15, (fwd_err(x, xt), fwd_err(ref, xt))


def test_dgesv_mixed_tall_panels(hb):
    """n = 9000: the first panels are 9000 rows tall, so their tournament
    leaves run 18 CTAs with two merge levels (16 + 2 candidate sets, then 2);
    forward error and backward criterion as above."""
    n, nrhs = 9000, 2
    rng = np.random.default_rng(90)
    a = householder_matrix(rng, n, 1e6)
    xt = rng.uniform(-1, 1, (n, nrhs))
    b = np.asfortranarray(a @ xt)
    x = np.zeros((n, nrhs), order="F")
    ipiv = np.zeros(n, np.int32)
    info, it = hb.dgesv_mixed(n, nrhs, a.copy(order="F"), n, ipiv, b, n, x, n)
    assert info == 0 and 1 <= it <= 10, (info, it)
    assert ipiv.min() >= 1 and ipiv.max() <= n
    check_backward(a, x, b, n)
    ref = np.linalg.solve(a, b)
    assert fwd_err(x, xt) <= 4.0 * fwd_err(ref, xt) + 1e-15, (fwd_err(x, xt), fwd_err(ref, xt))


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n,nrhs", [(257, 1), (900, 5)])
def test_dposv_mixed_accuracy(hb, orc, uplo, n, nrhs):
    rng = np.random.default_rng(n * 3 + nrhs)
    a = spd_matrix(rng, n)
    xt = rng.uniform(-1, 1, (n, nrhs))
    b = np.asfortranarray(a @ xt)
    # Only the `uplo` triangle is referenced: poison the other one.
    a_in = a.copy(order="F")
    other = np.tril_indices(n, -1) if uplo == "U" else np.triu_indices(n, 1)
    a_in[other] = np.nan
    a_keep = a_in.copy(order="F")
    x = np.zeros((n, nrhs), order="F")
    info, it = hb.dposv_mixed(uplo, n, nrhs, a_in, n, b, n, x, n)
    assert info == 0 and it >= 1, (info, it)
    assert same_bits(a_in, a_keep)
    check_backward(a, x, b, n)
    a2, x2 = a.copy(order="F"), b.copy(order="F")
    assert orc.dposv(uplo, n, nrhs, a2, n, x2, n) == 0
    assert fwd_err(x, xt) <= 4.0 * fwd_err(x2, xt) + 1e-15


@pytest.mark.parametrize("n", [4500, 8200])
def test_dposv_mixed_many_blocks(hb, n):
    """Several diagonal blocks of 512 / 1024 columns with a ragged last one:
    each factored in FP64 by 32-column sub-panels, the blocks below and the
    trailing matrix on INT8. The refined solution must be at least as
    accurate as LAPACK's FP64 solve."""
    rng = np.random.default_rng(n)
    a = spd_matrix(rng, n)
    xt = rng.uniform(-1, 1, (n, 2))
    b = np.asfortranarray(a @ xt)
    x = np.zeros((n, 2), order="F")
    info, it = hb.dposv_mixed("L", n, 2, a.copy(order="F"), n, b, n, x, n)
    assert info == 0 and 1 <= it <= 10, (info, it)
    check_backward(a, x, b, n)
    ref = np.linalg.solve(a, b)
    assert fwd_err(x, xt) <= fwd_err(ref, xt) + 1e-15, (fwd_err(x, xt), fwd_err(ref, xt))


@pytest.mark.parametrize("slices", [3, 4, 5])
def test_dgesv_mixed_slice_counts(hb, slices):
    n = 500
    rng = np.random.default_rng(11)
    a = householder_matrix(rng, n, 1e4)
    xt = rng.uniform(-1, 1, (n, 2))
    b = np.asfortranarray(a @ xt)
    prev = hb.set_mixed_slices(slices)
    try:
        x = np.zeros((n, 2), order="F")
        ipiv = np.zeros(n, np.int32)
        info, it = hb.dgesv_mixed(n, 2, a.copy(order="F"), n, ipiv, b, n, x, n)
    finally:
        hb.set_mixed_slices(prev)
    assert info == 0 and it >= 1
    check_backward(a, x, b, n)


def test_dgesv_mixed_fallbacks_match_plain(hb):
    """Non-finite A (ITER -2) and a singular A (ITER -3): the plain FP64 path
    runs on A itself, so A, IPIV, X and INFO equal dgesv_'s bit for bit."""
    rng = np.random.default_rng(5)
    n, nrhs = 150, 2
    for kind, expect_iter in [("nan", -2), ("singular", -3)]:
        a = rng.uniform(-1, 1, (n, n))
        if kind == "nan":
            a[7, 9] = np.nan
        else:
            a[:, 40] = 0.0
        a = np.asfortranarray(a)
        b = np.asfortranarray(rng.uniform(-1, 1, (n, nrhs)))
        a1, x1 = a.copy(order="F"), np.zeros((n, nrhs), order="F")
        p1 = np.zeros(n, np.int32)
        info1, it = hb.dgesv_mixed(n, nrhs, a1, n, p1, b, n, x1, n)
        a2, x2 = a.copy(order="F"), b.copy(order="F")
        p2 = np.zeros(n, np.int32)
        info2 = hb.dgesv(n, nrhs, a2, n, p2, x2, n)
        assert it == expect_iter and info1 == info2
        assert same_bits(a1, a2) and np.array_equal(p1, p2)
        if info2 == 0:
            assert same_bits(x1, x2)
        else:
            assert info2 == 41


def test_dposv_mixed_indefinite_falls_back(hb):
    rng = np.random.default_rng(6)
    n = 200
    a = spd_matrix(rng, n)
    a[50, 50] = -5.0
    b = np.asfortranarray(rng.uniform(-1, 1, (n, 1)))
    a1, x1 = a.copy(order="F"), np.zeros((n, 1), order="F")
    info1, it = hb.dposv_mixed("L", n, 1, a1, n, b, n, x1, n)
    a2, x2 = a.copy(order="F"), b.copy(order="F")
    info2 = hb.dposv("L", n, 1, a2, n, x2, n)
    assert it == -3 and info1 == info2 > 0
    assert same_bits(a1, a2)


def test_mixed_quick_returns_and_invalid(hb):
    a = np.ones(16)
    x = np.full(16, 7.0)
    ipiv = np.zeros(4, np.int32)
    assert hb.dgesv_mixed(0, 1, a, 1, ipiv, a, 1, x, 1) == (0, 0)
    assert np.all(x == 7.0)
    with hb.ErrorCapture() as cap:
        assert hb.dgesv_mixed(-1, 1, a, 1, ipiv, a, 1, x, 1)[0] == -1
        assert hb.dgesv_mixed(4, -1, a, 4, ipiv, a, 4, x, 4)[0] == -2
        assert hb.dgesv_mixed(4, 1, a, 3, ipiv, a, 4, x, 4)[0] == -4
        assert hb.dgesv_mixed(4, 1, a, 4, ipiv, a, 3, x, 4)[0] == -7
        assert hb.dgesv_mixed(4, 1, a, 4, ipiv, a, 4, x, 3)[0] == -9
        assert hb.dposv_mixed("X", 4, 1, a, 4, a, 4, x, 4)[0] == -1
        assert hb.dposv_mixed("L", 4, 1, a, 3, a, 4, x, 4)[0] == -5
        assert hb.dposv_mixed("L", 4, 1, a, 4, a, 4, x, 3)[0] == -9
    assert cap.errors == [("DGESV_MIXED", 1), ("DGESV_MIXED", 2), ("DGESV_MIXED", 4),
                          ("DGESV_MIXED", 7), ("DGESV_MIXED", 9), ("DPOSV_MIXED", 1),
                          ("DPOSV_MIXED", 5), ("DPOSV_MIXED", 9)]
    assert np.all(x == 7.0)


# ---------------------------------------------------------------------------
# The extra-precise residual and the solvers at the configuration's own size.

@pytest.mark.parametrize("n,nrhs", [(700, 1), (1500, 3), (900, 20)])
def test_dresidual_dd_matches_exact(hb, n, nrhs):
    """b - A x with b = fl(A x): the residual is all cancellation. The
    extra-precise residual is within a few n eps^2 |A||x| of the exact one
    (computed on the CPU, tests/exact_ref.py), far below the n eps |A||x| an
    FP64 residual can reach."""
    from tests.exact_ref import exact_residual
    rng = np.random.default_rng(n + nrhs)
    a = np.asfortranarray(rng.uniform(-1, 1, (n, n)) * np.exp2(rng.integers(-8, 9, (n, n))))
    x = np.asfortranarray(rng.uniform(-1, 1, (n, nrhs)))
    b = np.asfortranarray(a @ x)
    r = np.zeros((n, nrhs), order="F")
    hb.dresidual_dd(n, nrhs, a, n, x, n, b, n, r, n)
    absax = np.abs(a) @ np.abs(x)
    rows = np.arange(0, n, 7)
    for q in range(0, nrhs, max(1, nrhs // 3)):
        exact = exact_residual(a[rows], x[:, q], b[rows, q])
        bound = 8 * n * EPS * EPS * absax[rows, q] + np.spacing(np.abs(exact))
        assert np.all(np.abs(r[rows, q] - exact) <= bound)
        # An FP64 residual misses by far more than this bound.
        assert np.max(np.abs((b[rows, q] - a[rows] @ x[:, q]) - exact) / bound) > 10


def solve_to_last_bit(hb, orc, a, lu, ipiv, b, x0):
    """The solution of A x = b to about the last bit: x0 (the oracle's own
    solution, independent of the solver under test) refined twice with the
    extra-precise residual and the oracle's FP64 LU factors."""
    n, nrhs = b.shape
    x = x0.copy(order="F")
    r = np.zeros((n, nrhs), order="F")
    for _ in range(2):
        hb.dresidual_dd(n, nrhs, a, n, x, n, b, n, r, n)
        d = r.copy(order="F")
        assert orc.dgetrs("N", n, nrhs, lu, n, ipiv, d, n) == 0
        x += d
    return x


def test_dgesv_mixed_config4_n8192(hb, orc):
    """The configuration's case at n = 8192, cond 1e6, nrhs 1 and 64: the
    mixed solver meets DSGESV's backward criterion and its forward error,
    against the solution of A x = b to the last bit, is at most the oracle
    dgesv's (the reference's FP64 LU order) on the same system."""
    import os
    orc.set_threads(os.cpu_count() or 1)
    rng = np.random.default_rng(8192)
    n = 8192
    a = householder_matrix(rng, n, 1e6)
    lu = a.copy(order="F")
    ipiv = np.zeros(n, np.int32)
    assert orc.dgetrf(n, n, lu, n, ipiv) == 0
    anrm = np.abs(a).sum(axis=1).max()
    for nrhs in (1, 64):
        xt = rng.uniform(-1, 1, (n, nrhs))
        b = np.asfortranarray(a @ xt)
        xp = b.copy(order="F")
        assert orc.dgetrs("N", n, nrhs, lu, n, ipiv, xp, n) == 0
        xm = np.zeros((n, nrhs), order="F")
        a_in = a.copy(order="F")
        info, it = hb.dgesv_mixed(n, nrhs, a_in, n, np.zeros(n, np.int32), b, n, xm, n)
        assert info == 0 and it > 0, (info, it)
        assert same_bits(a_in, a)
        xs = solve_to_last_bit(hb, orc, a, lu, ipiv, b, xp)
        e_mixed, e_plain = fwd_err(xm, xs), fwd_err(xp, xs)
        assert e_mixed <= e_plain, (nrhs, e_mixed, e_plain)
        r = np.zeros((n, nrhs), order="F")
        hb.dresidual_dd(n, nrhs, a, n, xm, n, b, n, r, n)
        for q in range(nrhs):
            assert np.abs(r[:, q]).max() <= np.abs(xm[:, q]).max() * anrm * EPS * np.sqrt(n)
