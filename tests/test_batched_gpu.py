"""Batched LU, LU solve and GEMM through the C ABI.

The reference has no batched API; every problem of a batch must come out bit
for bit as the single-problem routine gives it (dgetrf_, dgetrs_, dgemm_,
sgemm_ - themselves pinned bit-exact to the oracle - and the oracle's sgetrf
for single precision), whatever the mix of sizes. Sizes cover the leaf (<=
16), recursion (<= 64) and blocked (> 64) regimes of the LU and the KC chunk
boundaries of the GEMM.
"""
import numpy as np
import pytest

from tests.oracle_lib import same_bits, first_diff

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 7, 16, 17, 31, 33, 64, 65, 100, 128, 129, 200, 257, 300, 384]


def carve(torch, sizes_elems, dtype):
    """One device allocation carved into per-problem views (contiguous)."""
    total = int(sum(sizes_elems))
    buf = torch.empty(max(total, 1), dtype=dtype, device="cuda")
    views, off = [], 0
    for s in sizes_elems:
        views.append(buf[off:off + s])
        off += s
    return buf, views


def test_dgetrf_batched_matches_single(hb, cuda):
    torch = cuda
    rng = np.random.default_rng(1)
    ns = SIZES + list(rng.integers(1, 260, 40))
    ldas = [n + int(rng.integers(0, 3)) for n in ns]
    _, mats = carve(torch, [l * n for l, n in zip(ldas, ns)], torch.float64)
    _, pivs = carve(torch, ns, torch.int32)
    host = []
    for i, (n, l) in enumerate(zip(ns, ldas)):
        a = rng.uniform(-1, 1, l * n)
        if i == 5:
            a.reshape(n, l)[3, :] = 0.0  # singular: column 3 of problem 5 is zero
        host.append(a)
        mats[i].copy_(torch.from_numpy(a))
    torch.cuda.synchronize()
    info = hb.getrf_batched(ns, mats, ldas, pivs)
    for i, (n, l) in enumerate(zip(ns, ldas)):
        a1 = torch.from_numpy(host[i]).cuda()
        p1 = torch.zeros(n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        info1 = hb.dgetrf(n, n, a1, l, p1)
        got, want = mats[i].cpu().numpy(), a1.cpu().numpy()
        assert info[i] == info1, (i, n, info[i], info1)
        assert np.array_equal(pivs[i].cpu().numpy(), p1.cpu().numpy()), (i, n)
        assert same_bits(got, want), (i, n, first_diff(got, want))
    assert info[5] == 4


def test_sgetrf_batched_matches_oracle(hb, orc, cuda):
    torch = cuda
    rng = np.random.default_rng(2)
    ns = SIZES
    _, mats = carve(torch, [n * n for n in ns], torch.float32)
    _, pivs = carve(torch, ns, torch.int32)
    host = [rng.uniform(-1, 1, n * n).astype(np.float32) for n in ns]
    for i in range(len(ns)):
        mats[i].copy_(torch.from_numpy(host[i]))
    torch.cuda.synchronize()
    info = hb.getrf_batched(ns, mats, ns, pivs, precision="s")
    for i, n in enumerate(ns):
        a = np.asfortranarray(host[i].reshape(n, n).T)
        p = np.zeros(n, np.int32)
        assert orc.sgetrf(n, n, a, n, p) == info[i]
        got = mats[i].cpu().numpy().reshape(n, n).T
        assert np.array_equal(pivs[i].cpu().numpy(), p), (i, n)
        assert same_bits(got, a), (i, n, first_diff(got, a))


@pytest.mark.parametrize("trans", ["N", "T"])
def test_dgetrs_batched_matches_single(hb, cuda, trans):
    torch = cuda
    rng = np.random.default_rng(3)
    ns = SIZES
    nrhs = [int(rng.integers(1, 17)) for _ in ns]
    _, mats = carve(torch, [n * n for n in ns], torch.float64)
    _, pivs = carve(torch, ns, torch.int32)
    _, rhs = carve(torch, [n * r for n, r in zip(ns, nrhs)], torch.float64)
    for i, n in enumerate(ns):
        mats[i].copy_(torch.from_numpy(rng.uniform(-1, 1, n * n) + np.eye(n).ravel() * 2))
        rhs[i].copy_(torch.from_numpy(rng.uniform(-1, 1, n * nrhs[i])))
    torch.cuda.synchronize()
    assert all(v == 0 for v in hb.getrf_batched(ns, mats, ns, pivs))
    b0 = [r.clone() for r in rhs]
    torch.cuda.synchronize()
    assert hb.getrs_batched(trans, ns, nrhs, mats, ns, pivs, rhs, ns) == 0
    for i, n in enumerate(ns):
        x = b0[i].clone()
        torch.cuda.synchronize()
        hb.dgetrs(trans, n, nrhs[i], mats[i], n, pivs[i], x, n)
        got, want = rhs[i].cpu().numpy(), x.cpu().numpy()
        assert same_bits(got, want), (i, n, first_diff(got, want))


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("alpha,beta", [(1.5, 0.5), (-1.0, 1.0), (1.0, 0.0), (0.0, 2.0)])
def test_gemm_batched_matches_single(hb, cuda, ta, tb, alpha, beta):
    torch = cuda
    rng = np.random.default_rng(4)
    dims = [(1, 1, 1), (0, 5, 3), (5, 0, 3), (7, 9, 0), (33, 17, 300), (64, 64, 64),
            (129, 65, 257), (200, 100, 513)] + [tuple(int(v) for v in rng.integers(1, 150, 3))
                                                for _ in range(12)]
    for prec, dtype, single in (("d", torch.float64, hb.dgemm), ("s", torch.float32, hb.sgemm)):
        m = [d[0] for d in dims]
        n = [d[1] for d in dims]
        k = [d[2] for d in dims]
        lda = [max(1, (kk if ta != "N" else mm)) for mm, kk in zip(m, k)]
        ldb = [max(1, (nn if tb != "N" else kk)) for nn, kk in zip(n, k)]
        ldc = [max(1, mm) for mm in m]
        ea = [la * max(1, (mm if ta != "N" else kk)) for la, mm, kk in zip(lda, m, k)]
        eb = [lb * max(1, (kk if tb != "N" else nn)) for lb, nn, kk in zip(ldb, n, k)]
        ec = [lc * max(1, nn) for lc, nn in zip(ldc, n)]
        _, A = carve(torch, ea, dtype)
        _, B = carve(torch, eb, dtype)
        _, C = carve(torch, ec, dtype)
        for v in A + B + C:
            v.copy_(torch.from_numpy(rng.uniform(-1, 1, v.numel())))
        C0 = [v.clone() for v in C]
        torch.cuda.synchronize()
        hb.gemm_batched(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, precision=prec)
        for i in range(len(dims)):
            c1 = C0[i].clone()
            torch.cuda.synchronize()
            single(ta, tb, m[i], n[i], k[i], alpha, A[i], lda[i], B[i], ldb[i], beta, c1, ldc[i])
            got, want = C[i].cpu().numpy(), c1.cpu().numpy()
            assert same_bits(got, want), (prec, i, dims[i], first_diff(got, want))


@pytest.mark.parametrize("config", [64, 256, 1001, 1002])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.5])
def test_dgemm_batched_every_config_matches_single(hb, cuda, config, ta, tb, beta):
    """Each launch configuration the autotuner chooses from (the per-element
    kernel at two thread counts, the FP64 tensor-pipe kernel with 32 x 32 and
    64 x 64 tiles) gives every problem the single dgemm's bits: ragged sizes
    below and across the tiles, k across several 256-deep chunks."""
    torch = cuda
    rng = np.random.default_rng(config + ord(ta) + ord(tb) + int(10 * beta))
    dims = [(16, 16, 8), (17, 31, 5), (15, 40, 9), (64, 64, 256), (65, 63, 257), (96, 130, 600),
            (200, 17, 513), (33, 200, 31), (512, 96, 40)]
    m = [d[0] for d in dims]
    n = [d[1] for d in dims]
    k = [d[2] for d in dims]
    lda = [(kk if ta != "N" else mm) + 1 for mm, kk in zip(m, k)]
    ldb = [(nn if tb != "N" else kk) + 3 for nn, kk in zip(n, k)]
    ldc = [mm + 2 for mm in m]
    ea = [la * (mm if ta != "N" else kk) for la, mm, kk in zip(lda, m, k)]
    eb = [lb * (kk if tb != "N" else nn) for lb, nn, kk in zip(ldb, n, k)]
    ec = [lc * nn for lc, nn in zip(ldc, n)]
    _, A = carve(torch, ea, torch.float64)
    _, B = carve(torch, eb, torch.float64)
    _, C = carve(torch, ec, torch.float64)
    for v in A + B + C:
        v.copy_(torch.from_numpy(rng.uniform(-1, 1, v.numel())))
    C0 = [v.clone() for v in C]
    torch.cuda.synchronize()
    lib = hb.lib()
    prev = lib.hwyblas_batched_set_config(config)
    try:
        hb.gemm_batched(ta, tb, m, n, k, 1.5, A, lda, B, ldb, beta, C, ldc)
    finally:
        lib.hwyblas_batched_set_config(prev)
    for i in range(len(dims)):
        c1 = C0[i].clone()
        torch.cuda.synchronize()
        hb.dgemm(ta, tb, m[i], n[i], k[i], 1.5, A[i], lda[i], B[i], ldb[i], beta, c1, ldc[i])
        got, want = C[i].cpu().numpy(), c1.cpu().numpy()
        assert same_bits(got, want), (config, i, dims[i], first_diff(got, want))


def test_batched_invalid_arguments(hb, cuda):
    torch = cuda
    a = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = torch.zeros(4, dtype=torch.int32, device="cuda")
    host = np.zeros(16)
    with hb.ErrorCapture() as cap:
        hb.getrf_batched([4], [a], [4], [p])  # valid
        hb.getrf_batched([-1], [a], [4], [p])
        hb.getrf_batched([4], [a], [3], [p])
        hb.getrf_batched([4], [host], [4], [p])
        assert hb.getrs_batched("X", [4], [1], [a], [4], [p], [a], [4]) == -1
        assert hb.getrs_batched("N", [4], [1], [a], [4], [p], [a], [3]) == -8
        hb.gemm_batched("N", "N", [2], [2], [2], 1.0, [a], [1], [a], [2], 0.0, [a], [2])
    assert cap.errors == [("DGETRF_BATCHED", 1), ("DGETRF_BATCHED", 3),
                          ("DGETRF_BATCHED", 2),
                          ("DGETRS_BATCHED", 1), ("DGETRS_BATCHED", 8),
                          ("DGEMM_BATCHED", 8)]


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "U"), ("U", "N", "N"),
                                             ("L", "T", "N"), ("U", "T", "U")])
def test_trsm_batched_matches_single(hb, cuda, side, uplo, trans, diag):
    torch = cuda
    rng = np.random.default_rng(5)
    dims = [(1, 1), (5, 33), (33, 5), (64, 17), (100, 70), (129, 40), (40, 129), (300, 3)]
    for prec, dtype in (("d", torch.float64),):
        m = [d[0] for d in dims]
        n = [d[1] for d in dims]
        ka = [mm if side == "L" else nn for mm, nn in zip(m, n)]
        _, A = carve(torch, [k * k for k in ka], dtype)
        _, B = carve(torch, [mm * nn for mm, nn in zip(m, n)], dtype)
        for i, k in enumerate(ka):
            A[i].copy_(torch.from_numpy(rng.uniform(-1, 1, k * k) + np.eye(k).ravel() * k))
            B[i].copy_(torch.from_numpy(rng.uniform(-1, 1, m[i] * n[i])))
        B0 = [v.clone() for v in B]
        torch.cuda.synchronize()
        for alpha in (1.0, -0.5):
            for i in range(len(dims)):
                B[i].copy_(B0[i])
            torch.cuda.synchronize()
            hb.trsm_batched(side, uplo, trans, diag, m, n, alpha, A, ka, B, m, precision=prec)
            for i in range(len(dims)):
                x = B0[i].clone()
                torch.cuda.synchronize()
                hb.dtrsm(side, uplo, trans, diag, m[i], n[i], alpha, A[i], ka[i], x, m[i])
                got, want = B[i].cpu().numpy(), x.cpu().numpy()
                assert same_bits(got, want), (side, uplo, trans, diag, alpha, i,
                                              first_diff(got, want))


def test_batched_repeated_shape_replays(hb, cuda):
    """The same batch shape twice (the second call replays the captured
    graph) with new data: both results bit-identical to single calls."""
    torch = cuda
    rng = np.random.default_rng(6)
    ns = [3, 40, 70, 130, 20]
    _, mats = carve(torch, [n * n for n in ns], torch.float64)
    _, pivs = carve(torch, ns, torch.int32)
    for rep in range(3):
        host = [rng.uniform(-1, 1, n * n) for n in ns]
        for i in range(len(ns)):
            mats[i].copy_(torch.from_numpy(host[i]))
        torch.cuda.synchronize()
        info = hb.getrf_batched(ns, mats, ns, pivs)
        for i, n in enumerate(ns):
            a1 = torch.from_numpy(host[i]).cuda()
            p1 = torch.zeros(n, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            assert hb.dgetrf(n, n, a1, n, p1) == info[i]
            assert same_bits(mats[i].cpu().numpy(), a1.cpu().numpy()), (rep, i)
            assert np.array_equal(pivs[i].cpu().numpy(), p1.cpu().numpy())


@pytest.mark.parametrize("config", [64, 128, 256, 1128, 1001, 1002])
def test_lu_batched_every_config_matches_single(hb, cuda, config):
    """The batched LU, its solve and TRSM under each launch configuration:
    with 1001 and 1002 their trailing updates and TRSM products run on the
    FP64 tensor pipe (32 x 32 and 64 x 64 tiles) and every problem must still
    come out as the single routines give it."""
    torch = cuda
    rng = np.random.default_rng(config)
    ns = [1, 16, 17, 33, 64, 65, 100, 129, 200, 300, 512]
    nrhs = [1, 3, 16, 5, 33, 2, 40, 7, 16, 64, 20]
    _, mats = carve(torch, [n * n for n in ns], torch.float64)
    _, pivs = carve(torch, ns, torch.int32)
    _, rhs = carve(torch, [n * r for n, r in zip(ns, nrhs)], torch.float64)
    host = [rng.uniform(-1, 1, n * n) for n in ns]
    for i, n in enumerate(ns):
        mats[i].copy_(torch.from_numpy(host[i]))
        rhs[i].copy_(torch.from_numpy(rng.uniform(-1, 1, n * nrhs[i])))
    b0 = [r.clone() for r in rhs]
    torch.cuda.synchronize()
    lib = hb.lib()
    prev = lib.hwyblas_batched_set_config(config)
    try:
        info = hb.getrf_batched(ns, mats, ns, pivs)
        for trans in ("N", "T"):
            for i in range(len(ns)):
                rhs[i].copy_(b0[i])
            torch.cuda.synchronize()
            assert hb.getrs_batched(trans, ns, nrhs, mats, ns, pivs, rhs, ns) == 0
            for i, n in enumerate(ns):
                x = b0[i].clone()
                torch.cuda.synchronize()
                hb.dgetrs(trans, n, nrhs[i], mats[i], n, pivs[i], x, n)
                got, want = rhs[i].cpu().numpy(), x.cpu().numpy()
                assert same_bits(got, want), (config, trans, i, n, first_diff(got, want))
        for side, uplo, tr, diag in (("L", "L", "N", "U"), ("R", "U", "T", "N")):
            tri = [m.clone() for m in mats]
            for i in range(len(ns)):
                rhs[i].copy_(b0[i])
            torch.cuda.synchronize()
            mm = ns if side == "L" else nrhs
            nn = nrhs if side == "L" else ns
            # B is n x nrhs (left) or nrhs x n (right), both stored in rhs[i].
            hb.trsm_batched(side, uplo, tr, diag, mm, nn, 0.5, tri, ns, rhs, mm)
            for i, n in enumerate(ns):
                x = b0[i].clone()
                torch.cuda.synchronize()
                hb.dtrsm(side, uplo, tr, diag, mm[i], nn[i], 0.5, tri[i], n, x, mm[i])
                got, want = rhs[i].cpu().numpy(), x.cpu().numpy()
                assert same_bits(got, want), (config, side, i, n, first_diff(got, want))
    finally:
        lib.hwyblas_batched_set_config(prev)
    for i, n in enumerate(ns):
        a1 = torch.from_numpy(host[i]).cuda()
        p1 = torch.zeros(n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert hb.dgetrf(n, n, a1, n, p1) == info[i]
        assert same_bits(mats[i].cpu().numpy(), a1.cpu().numpy()), (config, i, n)
        assert np.array_equal(pivs[i].cpu().numpy(), p1.cpu().numpy())


@pytest.mark.parametrize("config", [64, 128, 256, 1128])
def test_single_precision_batched_every_config(hb, orc, cuda, config):
    """FP32 under each register-tiled configuration: the LU against the
    oracle's sgetrf, the solve against sgetrs and the GEMM against sgemm,
    bit for bit (chains restarted every 384 in single precision)."""
    torch = cuda
    rng = np.random.default_rng(100 + config)
    ns = [1, 16, 17, 64, 65, 130, 257, 400]
    nrhs = [2, 16, 1, 64, 3, 17, 9, 40]
    _, mats = carve(torch, [n * n for n in ns], torch.float32)
    _, pivs = carve(torch, ns, torch.int32)
    _, rhs = carve(torch, [n * r for n, r in zip(ns, nrhs)], torch.float32)
    host = [rng.uniform(-1, 1, n * n).astype(np.float32) for n in ns]
    for i, n in enumerate(ns):
        mats[i].copy_(torch.from_numpy(host[i]))
        rhs[i].copy_(torch.from_numpy(rng.uniform(-1, 1, n * nrhs[i]).astype(np.float32)))
    b0 = [r.clone() for r in rhs]
    dims = [(16, 16, 7), (64, 70, 384), (65, 33, 385), (200, 130, 800), (17, 300, 50)]
    m = [d[0] for d in dims]
    n = [d[1] for d in dims]
    k = [d[2] for d in dims]
    _, A = carve(torch, [mm * kk for mm, kk in zip(m, k)], torch.float32)
    _, B = carve(torch, [kk * nn for kk, nn in zip(k, n)], torch.float32)
    _, C = carve(torch, [mm * nn for mm, nn in zip(m, n)], torch.float32)
    for v in A + B + C:
        v.copy_(torch.from_numpy(rng.uniform(-1, 1, v.numel()).astype(np.float32)))
    C0 = [v.clone() for v in C]
    torch.cuda.synchronize()
    lib = hb.lib()
    prev = lib.hwyblas_batched_set_config(config)
    try:
        info = hb.getrf_batched(ns, mats, ns, pivs, precision="s")
        assert hb.getrs_batched("N", ns, nrhs, mats, ns, pivs, rhs, ns, precision="s") == 0
        hb.gemm_batched("N", "N", m, n, k, 1.25, A, m, B, k, 0.5, C, m, precision="s")
    finally:
        lib.hwyblas_batched_set_config(prev)
    for i, nn in enumerate(ns):
        a = np.asfortranarray(host[i].reshape(nn, nn).T)
        p = np.zeros(nn, np.int32)
        assert orc.sgetrf(nn, nn, a, nn, p) == info[i]
        got = mats[i].cpu().numpy().reshape(nn, nn).T
        assert np.array_equal(pivs[i].cpu().numpy(), p), (config, i, nn)
        assert same_bits(got, a), (config, i, nn, first_diff(got, a))
        x = b0[i].clone()
        torch.cuda.synchronize()
        hb.sgetrs("N", nn, nrhs[i], mats[i], nn, pivs[i], x, nn)
        got, want = rhs[i].cpu().numpy(), x.cpu().numpy()
        assert same_bits(got, want), (config, i, nn, first_diff(got, want))
    for i in range(len(dims)):
        c1 = C0[i].clone()
        torch.cuda.synchronize()
        hb.sgemm("N", "N", m[i], n[i], k[i], 1.25, A[i], m[i], B[i], k[i], 0.5, c1, m[i])
        got, want = C[i].cpu().numpy(), c1.cpu().numpy()
        assert same_bits(got, want), (config, i, dims[i], first_diff(got, want))
