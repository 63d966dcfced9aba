import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (CUDA device)")


@pytest.fixture(scope="session")
def orc():
    from tests import oracle_lib
    return oracle_lib.Oracle()


@pytest.fixture(scope="session")
def ref_drivers():
    """The reference's own getrf.cc/potrf.cc drivers (oracle/_ref), if built."""
    from tests import oracle_lib
    lib = oracle_lib.load_ref()
    if lib is None:
        pytest.skip("oracle/_ref/libhwyref.so not built (needs the reference sources)")
    return lib


@pytest.fixture(scope="session")
def refblas():
    """The reference library itself, compiled against the Highway-API shim
    (oracle/_ref/libhwyblas_ref.so), if built."""
    from tests import oracle_lib
    lib = oracle_lib.load_refblas()
    if lib is None:
        pytest.skip("oracle/_ref/libhwyblas_ref.so not built (needs the reference sources)")
    return lib


@pytest.fixture(scope="session")
def hb():
    import hwyblas_b200
    hwyblas_b200.lib()
    return hwyblas_b200


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
