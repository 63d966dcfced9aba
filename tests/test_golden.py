"""Golden LU / Cholesky fixtures produced by the reference's own LAPACK
drivers (tests/golden/make_golden.py): the oracle must reproduce them bit for
bit on the CPU, and the library on the GPU."""
import os

import numpy as np
import pytest

from tests.oracle_lib import same_bits, first_diff

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "lapack_ref.npz")


def cases(prefix):
    data = np.load(GOLDEN)
    keys = sorted({k.rsplit("_", 1)[0] for k in data.files if k.startswith(prefix)})
    return data, keys


def getrf_case(key):
    _, m, rec = key.split("_")[0], *key.split("_")[1:]
    mm, nn = (int(v) for v in m.split("x"))
    return mm, nn, rec == "rec"


def test_golden_getrf_oracle(orc):
    data, keys = cases("getrf_")
    assert len(keys) >= 8
    for key in keys:
        m, n, rec = getrf_case(key)
        info_ref, lda = data[key + "_info"]
        a = data[key + "_a"].copy(order="F")
        piv = np.zeros(min(m, n), np.int32)
        info = (orc.dgetrf2 if rec else orc.dgetrf)(m, n, a, lda, piv)
        assert info == info_ref, key
        assert np.array_equal(piv, data[key + "_ipiv"]), key
        assert same_bits(a, data[key + "_lu"]), (key, first_diff(a, data[key + "_lu"]))


def test_golden_potrf_oracle(orc):
    data, keys = cases("potrf_")
    for key in keys:
        _, n, uplo, rec = key.split("_")
        n = int(n)
        a = data[key + "_a"].copy(order="F")
        info = (orc.dpotrf2 if rec == "rec" else orc.dpotrf)(uplo, n, a, n)
        assert info == data[key + "_info"][0], key
        assert same_bits(a, data[key + "_l"]), key


@pytest.mark.gpu
def test_golden_getrf_gpu(hb):
    data, keys = cases("getrf_")
    for key in keys:
        m, n, rec = getrf_case(key)
        info_ref, lda = data[key + "_info"]
        a = data[key + "_a"].copy(order="F")
        piv = np.zeros(min(m, n), np.int32)
        info = (hb.dgetrf2 if rec else hb.dgetrf)(m, n, a, lda, piv)
        assert info == info_ref, key
        assert np.array_equal(piv, data[key + "_ipiv"]), key
        assert same_bits(a, data[key + "_lu"]), (key, first_diff(a, data[key + "_lu"]))


@pytest.mark.gpu
def test_golden_potrf_gpu(hb):
    data, keys = cases("potrf_")
    for key in keys:
        _, n, uplo, rec = key.split("_")
        n = int(n)
        a = data[key + "_a"].copy(order="F")
        info = (hb.dpotrf2 if rec == "rec" else hb.dpotrf)(uplo, n, a, n)
        assert info == data[key + "_info"][0], key
        assert same_bits(a, data[key + "_l"]), key
