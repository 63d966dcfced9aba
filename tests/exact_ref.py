"""Correctly rounded dot products on the CPU (test infrastructure).

The error yardstick of the emulated GEMM and of the mixed solvers. Every
product a*b is split exactly into p + e with p = fl(a*b) and e = a*b - p
(Dekker's TwoProduct over Veltkamp's split, T. J. Dekker, "A floating-point
technique for extending the available precision", Numer. Math. 18, 1971),
and the 2K doubles are summed by math.fsum, which returns the correctly
rounded value of their exact sum (Shewchuk's adaptive summation). The result
is therefore the exact dot product rounded once to double. The split is exact
while no intermediate overflows and no product falls below 2^-969; the entry
points check both.
"""
import math

import numpy as np

_SPLIT = 134217729.0  # 2^27 + 1
_TINY = 2.0 ** -969
_HUGE = 2.0 ** 995


def _split(x):
    c = _SPLIT * x
    hi = c - (c - x)
    return hi, x - hi


def two_product(a, b):
    """Elementwise p = fl(a b) and e with a b = p + e exactly."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    p = a * b
    ah, al = _split(a)
    bh, bl = _split(b)
    e = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    return p, e


def _check(a, b):
    if not (np.isfinite(a).all() and np.isfinite(b).all()):
        raise ValueError("exact dot products need finite inputs")
    if np.abs(a).max(initial=0.0) >= _HUGE or np.abs(b).max(initial=0.0) >= _HUGE:
        raise ValueError("inputs too large for an exact split")


def _check_products(nz_a, nz_b, p):
    both = nz_a & nz_b
    if both.any() and np.abs(p[both]).min() < _TINY:
        raise ValueError("a product is too small for an exact split")


def exact_dot(x, y):
    """The exact dot product of two float64 vectors, rounded once."""
    x = np.asarray(x, dtype=np.float64).ravel()
    y = np.asarray(y, dtype=np.float64).ravel()
    _check(x, y)
    p, e = two_product(x, y)
    _check_products(x != 0.0, y != 0.0, p)
    return math.fsum(np.concatenate([p, e]).tolist())


def exact_gemm_columns(a, b, cols, rows=None):
    """Columns `cols` of A B (A m x k, B k x n, float64 arrays in any order),
    each entry the exact value rounded once; restricted to `rows` if given.
    Returns an array of shape (len(rows), len(cols))."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    _check(a, b)
    rows = np.arange(a.shape[0]) if rows is None else np.asarray(rows)
    out = np.empty((len(rows), len(cols)))
    ar = a[rows]
    for jj, j in enumerate(cols):
        p, e = two_product(ar, b[:, j][None, :])
        _check_products(ar != 0.0, (b[:, j] != 0.0)[None, :], p)
        pe = np.concatenate([p, e], axis=1)
        for ii in range(len(rows)):
            out[ii, jj] = math.fsum(pe[ii].tolist())
    return out


def exact_residual(a, x, b):
    """b - A x for one right-hand side, each entry the exact value rounded
    once (A n x n, x and b vectors)."""
    a = np.asarray(a, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    _check(a, x)
    p, e = two_product(a, x[None, :])
    _check_products(a != 0.0, (x != 0.0)[None, :], p)
    out = np.empty(a.shape[0])
    for i in range(a.shape[0]):
        out[i] = math.fsum([b[i]] + (-p[i]).tolist() + (-e[i]).tolist())
    return out
