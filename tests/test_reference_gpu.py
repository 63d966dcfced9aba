"""The GPU path against the reference library itself (GPU).

oracle/_ref/libhwyblas_ref.so is the reference's own source tree compiled
unmodified against the Highway-API shim (oracle/hwy_shim). The GPU results
of the configurations' routines must equal its results bit for bit, pivots
included: dgemm_ (configuration 1's NN 1024^3 with alpha 1.5, beta 0.5, and
transposed and ragged cases), dtrsm_ (configuration 2's L/L/N/U 4096 x 512,
scaled to stay finite), dgetrf_ (configuration 2's n = 4096), dpotrf_ and
idamax_. Skipped where the library could not be built.
"""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ta,tb,m,n,k", [("N", "N", 1024, 1024, 1024), ("T", "N", 300, 200, 700),
                                         ("N", "T", 129, 65, 257), ("T", "T", 33, 517, 90)])
def test_dgemm_is_the_reference(hb, refblas, ta, tb, m, n, k):
    rng = np.random.default_rng(m + n + k)
    a = rand(rng, m if ta == "N" else k, k if ta == "N" else m)
    b = rand(rng, k if tb == "N" else n, n if tb == "N" else k)
    c = rand(rng, m, n)
    c1, c2 = c.copy(order="F"), c.copy(order="F")
    hb.dgemm(ta, tb, m, n, k, 1.5, a, a.shape[0], b, b.shape[0], 0.5, c1, m)
    refblas.dgemm(ta, tb, m, n, k, 1.5, a, a.shape[0], b, b.shape[0], 0.5, c2, m)
    assert same_bits(c1, c2)


def test_dtrsm_config2_is_the_reference(hb, refblas):
    rng = np.random.default_rng(4096)
    m, n = 4096, 512
    a = np.asfortranarray(rng.uniform(-1, 1, (m, m)) / m)
    b = rand(rng, m, n)
    b1, b2 = b.copy(order="F"), b.copy(order="F")
    hb.dtrsm("L", "L", "N", "U", m, n, 1.0, a, m, b1, m)
    refblas.dtrsm("L", "L", "N", "U", m, n, 1.0, a, m, b2, m)
    assert same_bits(b1, b2)


def test_dgetrf_config2_is_the_reference(hb, refblas):
    rng = np.random.default_rng(17)
    n = 4096
    a = rand(rng, n, n)
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    p1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    assert hb.dgetrf(n, n, a1, n, p1) == refblas.dgetrf(n, n, a2, n, p2) == 0
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2)


@pytest.mark.parametrize("uplo", ["L", "U"])
def test_dpotrf_is_the_reference(hb, refblas, uplo):
    rng = np.random.default_rng(ord(uplo))
    n = 1500
    g = rng.standard_normal((n, n))
    a = np.asfortranarray(g @ g.T / n + np.eye(n))
    a1, a2 = a.copy(order="F"), a.copy(order="F")
    assert hb.dpotrf(uplo, n, a1, n) == refblas.dpotrf(uplo, n, a2, n) == 0
    assert same_bits(a1, a2)


@pytest.mark.parametrize("mode", ["rand", "ties", "nan_inside"])
def test_idamax_is_the_reference(hb, refblas, mode):
    rng = np.random.default_rng(5)
    n = 100000
    x = rng.uniform(-1, 1, n)
    if mode == "ties":
        x = np.round(x * 5) / 5
    elif mode == "nan_inside":
        x[n // 2] = np.nan
    assert hb.idamax(n, x, 1) == refblas.idamax(n, x, 1)
