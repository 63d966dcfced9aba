"""GPU parity of ?gerfs_ (iterative refinement with error bounds,
src/lapack/gesvx.cc:319-456, and its LACN2 estimate, src/lapack/trsen.cc:
2243-2366) through the C ABI against the oracle, bit for bit: the refined X,
FERR, BERR and the final WORK/IWORK contents.

The oracle's GERFS is pinned against the reference's own gesvx.cc and
trsen.cc (tests/test_oracle_pins.py). Cases: op N, T and C, one to three
right-hand sides, a starting X perturbed so that the refinement iterates,
well-conditioned and badly scaled A, host and device arrays, the quick
return and the argument checks.
"""
import numpy as np
import pytest

from tests.oracle_lib import rand, same_bits, first_diff

pytestmark = pytest.mark.gpu


def case(orc, rng, n, nrhs, dtype, spread, trans):
    scale = np.exp(np.linspace(0, np.log(spread), n))[None, :]
    a = np.asfortranarray((rand(rng, n, n) * scale).astype(dtype))
    af = a.copy(order="F")
    ipiv = np.zeros(max(n, 1), np.int32)
    getrf = orc.sgetrf if dtype == np.float32 else orc.dgetrf
    getrs = orc.sgetrs if dtype == np.float32 else orc.dgetrs
    assert getrf(n, n, af, n, ipiv) == 0
    b = rand(rng, n, nrhs, dtype)
    x = b.copy(order="F")
    assert getrs(trans, n, nrhs, af, n, ipiv, x, n) == 0
    x = np.asfortranarray((x * (1 + 1e-4 * rng.standard_normal(x.shape))).astype(dtype))
    return a, af, ipiv, b, x


@pytest.mark.parametrize("p", ["d", "s"])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (2, 3), (5, 2), (17, 1), (64, 2), (150, 3),
                                    (700, 2)])
@pytest.mark.parametrize("spread", [1.0, 1e6])
def test_gerfs_bitexact(hb, orc, p, trans, n, nrhs, spread):
    dtype = np.float32 if p == "s" else np.float64
    rng = np.random.default_rng(n * 17 + nrhs + int(spread) % 97)
    a, af, ipiv, b, x = case(orc, rng, n, nrhs, dtype, spread, trans)
    outs = []
    for who in ("hb", "orc"):
        xx = x.copy(order="F")
        ferr, berr = np.zeros(nrhs, dtype), np.zeros(nrhs, dtype)
        work, iwork = np.full(3 * n, 5.0, dtype), np.full(n, 9, np.int32)
        if who == "hb":
            info = hb.gerfs(p, trans, n, nrhs, a, n, af, n, ipiv, b, n, xx, n, ferr, berr,
                            work, iwork)
        else:
            info = orc.gerfs(trans, n, nrhs, a, n, af, n, ipiv, b, n, xx, n, ferr, berr, work,
                             iwork)
        assert info == 0
        outs.append((xx, ferr, berr, work, iwork))
    for name, u, v in zip(("x", "ferr", "berr", "work", "iwork"), outs[0], outs[1]):
        ok = np.array_equal(u, v) if u.dtype == np.int32 else same_bits(u, v)
        assert ok, (name, first_diff(u, v) if u.dtype != np.int32 else None)


def test_gerfs_device_arrays(hb, orc):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(12)
    n, nrhs = 300, 2
    a, af, ipiv, b, x = case(orc, rng, n, nrhs, np.float64, 1e3, "N")
    dev = lambda m: torch.from_numpy(np.ascontiguousarray(m.T)).T.cuda()  # noqa: E731
    tx = dev(x)
    tf, tb = torch.zeros(nrhs, dtype=torch.float64, device="cuda"), torch.zeros(
        nrhs, dtype=torch.float64, device="cuda")
    tw = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    ti = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert hb.gerfs("d", "N", n, nrhs, dev(a), n, dev(af), n, torch.from_numpy(ipiv).cuda(),
                    dev(b), n, tx, n, tf, tb, tw, ti) == 0
    xx = x.copy(order="F")
    ferr, berr = np.zeros(nrhs), np.zeros(nrhs)
    work, iwork = np.zeros(3 * n), np.zeros(n, np.int32)
    assert orc.gerfs("N", n, nrhs, a, n, af, n, ipiv, b, n, xx, n, ferr, berr, work,
                     iwork) == 0
    got = np.asfortranarray(tx.cpu().numpy())
    assert same_bits(got, xx), first_diff(got, xx)
    assert same_bits(tf.cpu().numpy(), ferr) and same_bits(tb.cpu().numpy(), berr)
    assert same_bits(tw.cpu().numpy(), work)


def test_gerfs_quick_return_and_errors(hb):
    z = np.zeros(64)
    ip = np.ones(8, np.int32)
    ferr, berr = np.full(2, 7.0), np.full(2, 7.0)
    assert hb.gerfs("d", "N", 0, 2, z, 1, z, 1, ip, z, 1, z, 1, ferr, berr, z, ip) == 0
    assert np.all(ferr == 0) and np.all(berr == 0)
    with hb.ErrorCapture() as cap:
        assert hb.gerfs("d", "X", 4, 1, z, 4, z, 4, ip, z, 4, z, 4, ferr, berr, z, ip) == -1
        assert hb.gerfs("d", "N", -1, 1, z, 4, z, 4, ip, z, 4, z, 4, ferr, berr, z, ip) == -2
        assert hb.gerfs("s", "N", 4, -1, z, 4, z, 4, ip, z, 4, z, 4, ferr, berr, z, ip) == -3
        assert hb.gerfs("d", "T", 4, 1, z, 3, z, 4, ip, z, 4, z, 4, ferr, berr, z, ip) == -5
        assert hb.gerfs("d", "N", 4, 1, z, 4, z, 3, ip, z, 4, z, 4, ferr, berr, z, ip) == -7
        assert hb.gerfs("d", "N", 4, 1, z, 4, z, 4, ip, z, 3, z, 4, ferr, berr, z, ip) == -10
        assert hb.gerfs("d", "N", 4, 1, z, 4, z, 4, ip, z, 4, z, 3, ferr, berr, z, ip) == -12
    assert cap.errors == [("DGERFS", 1), ("DGERFS", 2), ("SGERFS", 3), ("DGERFS", 5),
                          ("DGERFS", 7), ("DGERFS", 10), ("DGERFS", 12)]
