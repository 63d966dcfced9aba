"""A bounded device wait that runs out (GPU): the LU panel's cooperative pivot
exchange, whose CTAs poll global tags for their peers' candidates, is given a
poll limit of 1 through the test hook, so its waits give up. The call must
return, report the timeout (cudaErrorLaunchTimeout through
hwyblas_last_cuda_error), leave the context usable, and, with the default
limit restored, the next factorization must be bit-identical to the oracle
again. The failure is made on purpose only through the limit: no fault, trap
or endless wait. The panel's loads are plain loads (no TMA or asynchronous
copies are in flight when a wait gives up)."""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits

pytestmark = pytest.mark.gpu

CUDA_ERROR_LAUNCH_TIMEOUT = 702  # cudaErrorLaunchTimeout
DEFAULT_POLLS = 1 << 26


def test_leaf_wait_times_out_reports_and_recovers(hb, orc):
    lib = hb.lib()
    rng = np.random.default_rng(12)
    # 59 CTAs of 1024 rows: beyond the 16-CTA cluster, so the cooperative
    # variant with polled global slots runs.
    m, n = 60000, 16
    a0 = rand(rng, m, n)
    lib.hwyblas_last_cuda_error()  # clear
    prev = lib.hwyblas_set_leaf_wait_limit(1)
    try:
        assert prev == DEFAULT_POLLS
        a = a0.copy(order="F")
        ipiv = np.zeros(n, np.int32)
        hb.dgetrf2(m, n, a, m, ipiv)
        assert lib.hwyblas_last_cuda_error() == CUDA_ERROR_LAUNCH_TIMEOUT
    finally:
        assert lib.hwyblas_set_leaf_wait_limit(0) == 1
    a1, a2 = a0.copy(order="F"), a0.copy(order="F")
    p1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32)
    info1 = hb.dgetrf2(m, n, a1, m, p1)
    assert lib.hwyblas_last_cuda_error() == 0
    info2 = orc.dgetrf2(m, n, a2, m, p2)
    assert info1 == info2 == 0
    assert np.array_equal(p1, p2)
    assert same_bits(a1, a2)


def test_leaf_wait_limit_default_is_restored(hb):
    lib = hb.lib()
    assert lib.hwyblas_set_leaf_wait_limit(0) == DEFAULT_POLLS
