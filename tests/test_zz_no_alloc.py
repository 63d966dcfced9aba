"""hwyblas_idamax_noalloc: the IDAMAX reduction with its scratch in a fixed
device array instead of allocated memory, called through the C ABI and
compared with idamax_ on the same device vectors (the index must be equal).

The file is named to be collected last, so that the shared scratch has been
set up by an earlier call in some runs and not in others (it also passes
alone).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 1024 * 16384


def _vector(torch, rng, n, incx, mode):
    span = (n - 1) * incx + 1
    x = rng.uniform(-1.0, 1.0, span)
    if mode == "ties":
        x = np.round(x * 4) / 4  # many equal magnitudes: first index wins
    elif mode == "nan_first":
        x[0] = np.nan
    elif mode == "nan_inside":
        x[(n // 2) * incx] = np.nan
    return torch.from_numpy(x).cuda()


@pytest.mark.parametrize("n,incx,mode", [
    (1, 1, "rand"), (2, 1, "ties"), (1000, 1, "rand"), (1000, 3, "ties"),
    (16384, 1, "rand"), (16385, 2, "nan_inside"), (1_000_003, 1, "ties"),
    (50_000, 1, "nan_first"), (MAX_N, 1, "rand"),
])
def test_noalloc_matches_idamax_two_calls(hb, cuda, n, incx, mode):
    torch = cuda
    rng = np.random.default_rng(n + incx)
    x1 = _vector(torch, rng, n, incx, mode)
    x2 = _vector(torch, rng, n, incx, "ties")
    r1 = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    r2 = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    # Two calls in a row on one stream, then both results.
    assert hb.idamax_noalloc(n, x1, incx, r1, stream) == 0
    assert hb.idamax_noalloc(n, x2, incx, r2, stream) == 0
    torch.cuda.synchronize()
    assert int(r1.item()) == hb.idamax(n, x1, incx)
    assert int(r2.item()) == hb.idamax(n, x2, incx)
    if mode == "nan_first":
        assert int(r1.item()) == 1


def test_noalloc_allocates_nothing(hb, cuda):
    torch = cuda
    n = 300_000
    x = torch.rand(n, dtype=torch.float64, device="cuda")
    r = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert hb.idamax_noalloc(n, x, 1, r, stream) == 0  # set-up, if not yet done
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        assert hb.idamax_noalloc(n, x, 1, r, stream) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert int(r.item()) == int(torch.argmax(x.abs()).item()) + 1


def test_noalloc_quick_return_and_rejections(hb, cuda):
    torch = cuda
    x = torch.rand(10, dtype=torch.float64, device="cuda")
    r = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert hb.idamax_noalloc(0, x, 1, r, stream) == 0
    torch.cuda.synchronize()
    assert int(r.item()) == 0
    r.fill_(-7)
    assert hb.idamax_noalloc(10, x, 0, r, stream) == 0
    torch.cuda.synchronize()
    assert int(r.item()) == 0
    r.fill_(-7)
    torch.cuda.synchronize()
    host_x = np.ones(10)
    with hb.ErrorCapture() as cap:
        assert hb.idamax_noalloc(MAX_N + 1, x, 1, r, stream) == -1
        assert hb.idamax_noalloc(10, host_x, 1, r, stream) == -2
        assert hb.idamax_noalloc(10, x, 1, np.zeros(1, np.int32), stream) == -4
    assert cap.errors == [("IDAMAX_NOALLOC", 1), ("IDAMAX_NOALLOC", 2),
                          ("IDAMAX_NOALLOC", 4)]
    torch.cuda.synchronize()
    assert int(r.item()) == -7
