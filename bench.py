#!/usr/bin/env python
"""Benchmark of the level-3 hot path on B200 (one JSON line on rank 0).

Metric: FP64-accurate TFLOP/s, dgemm n=8192 and dgesv n=16384, emulated /
mixed against plain.

Headline (`value`): DGEMM M = N = K = 8192, column-major NN, C = A B, with
A and B entries u * 2^e (u uniform[-1, 1], e uniform in {-8..8}, seeded), on
the emulated-FP64 path (Ozaki INT8 slices on tcgen05, slice count chosen from
the inputs' exponent spread) - 2 * 8192^3 useful FP64 flops per step.
"FP64-accurate": its normwise error against a double-double product of 64
sampled columns must not exceed the plain FP64 path's error on the same
inputs (both are reported; the tests hold the double-double product to 1 ulp
of the exact one).

value  : device-timed, inputs resident in HBM, CUDA events on the library's
         stream, max over ranks; whole-job TFLOP/s (sum over ranks).
e2e    : the same product through the public C ABI with pinned HOST buffers
         (A, B copied in and C copied out inside the timed region).
plain  : the plain FP64 tensor-pipe DGEMM (bit-identical to the reference)
         on the same inputs, and its error.
auto_slices: the automatic slice count at exponent spreads 0, 8 and 30.
config1: dgemm NN 1024^3, alpha 1.5, beta 0.5 (device, C ABI with host
         buffers, and the CPU path single-threaded on the same inputs).
config2: dtrsm L/L/N/U 4096 x 512 and dgetrf 4096, with the LU residual
         ratio and ipiv / bit equality against the CPU path.
batched: 10,000 problems, n log-uniform in [8, 512], dgetrf + dgetrs + dgemm
         each, batched persistent launches against the per-problem loop.
widened: throughput of the routines beyond the hot path (dtrmm, dsymm,
         dsyr2k, dgemmtr, dtrtri, dgetri at n = 8192; zgemm, cgemm at 4096).
dgesv  : n = 16384, A = H1 diag(s) H2 (H1, H2 products of 4 Householder
         reflectors, s geometric from 1 to 1/cond): the plain FP64 dgesv
         (bit-identical to the reference's LU) against the mixed-precision
         solver, forward errors against the known solution, iterations; and
         dposv on SPD A = G G^T / n + 1e-3 I.
Replicas only: every rank runs its own problems (weak scaling).

--impl reference times the reference's CPU implementation of the path on this
host's cores (the oracle port of the reference's DGEMM with its per-element
order, all threads): --warmup untimed and --steps timed steps, each one
bounded column sample of the same workload, plus a single-threaded figure.
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 8192
GESV_N_DEFAULT = 16384
SPREAD = 8
METRIC = "FP64-accurate TFLOP/s: dgemm n=8192, dgesv n=16384; emulated/mixed vs plain"
FALLBACK_BF16_TFLOPS = 1590.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=N_DEFAULT)
    p.add_argument("--gesv-n", type=int, default=GESV_N_DEFAULT)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-dgesv", action="store_true")
    p.add_argument("--no-sweep", action="store_true",
                   help="skip the slice sweep and the automatic slice count per spread")
    p.add_argument("--no-small", action="store_true",
                   help="skip the dgemm 1024 / dtrsm 4096x512 / dgetrf 4096 configurations")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-widened", action="store_true",
                   help="skip the throughput of the routines beyond the hot path")
    p.add_argument("--nrhs", type=int, default=1, help="right-hand sides of --case gesv-mixed")
    p.add_argument("--kernels", action="store_true",
                   help="with --case: per-kernel device time of the call (CUPTI activity "
                        "records through torch.profiler)")
    p.add_argument("--case", default=None,
                   choices=["leaf", "getrf", "gesv", "gesv-mixed", "potrf", "posv-mixed",
                            "trtri", "getri", "trmm", "zgemm", "zgetrf", "zpotrf", "trsm"],
                   help="run one call of a hot-path piece and exit (for profilers): the LU "
                        "leaf on a gesv-n x 16 panel, plain dgetrf / dgesv / dpotrf, or "
                        "mixed dgesv / dposv at gesv-n; dtrtri, dgetri, dtrmm, zgemm, "
                        "zgetrf or zpotrf at n; each after one warm-up call")
    return p.parse_args()


# ---------------------------------------------------------------------------
# Distributed plumbing (replicas only).

def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Dist:
    def __init__(self, world, rank, local, backend):
        self.world, self.rank, self.local = world, rank, local
        self.pg = None
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg is not None:
            import torch
            if torch.cuda.is_available():
                self.pg.barrier(device_ids=[self.local])
            else:
                self.pg.barrier()

    def max(self, x):
        if self.pg is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64,
                         device="cuda" if torch.cuda.is_available() else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.

class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu_id)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append({"sm": float(parts[1]), "max": float(parts[2]),
                             "power": float(parts[3]) if parts[3] not in ("[N/A]", "N/A") else 0.0,
                             "hw": parts[5], "hwt": parts[6], "swt": parts[7], "pcap": parts[8]})
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [r for r in rows if r["power"] > 200] or rows
        reasons = set()
        for r in loaded:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("pcap", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in loaded),
                "sm_max_mhz": max(r["max"] for r in rows),
                "reasons": sorted(reasons), "samples": len(loaded)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's CPU implementation of the path on host cores.

def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def spread_matrix(rng, rows, cols, spread):
    e = rng.integers(-spread, spread + 1, (rows, cols))
    return np.asfortranarray(rng.uniform(-1, 1, (rows, cols)) * np.exp2(e))


class CpuPath:
    """The reference's CPU hot path: the oracle port of its DGEMM / DTRSM /
    DGETRF with the reference's per-element order (kind "port")."""

    def __init__(self):
        from tests.oracle_lib import Oracle
        self.orc = Oracle()
        self.kind = "port"
        self.threads = 1

    def set_threads(self, n):
        self.threads = int(n)
        self.orc.set_threads(self.threads)

    def dgemm(self, *args):
        return self.orc.dgemm(*args)

    def dtrsm(self, *args):
        return self.orc.dtrsm(*args)

    def dgetrf(self, *args):
        return self.orc.dgetrf(*args)


class DgemmSample:
    """One step of the CPU baseline: C = A B with A n x n and B n x cols, the
    first `cols` columns of the n = 8192 workload's product (a bounded sample:
    every column costs the same, so its TFLOP/s is the whole product's)."""

    def __init__(self, cpu, n, cols):
        rng = np.random.default_rng(7)
        self.cpu, self.n, self.cols = cpu, n, cols
        self.a = spread_matrix(rng, n, n, SPREAD)
        self.b = spread_matrix(rng, n, cols, SPREAD)
        self.c = np.zeros((n, cols), order="F")
        self.flops = 2.0 * n * cols * n

    def __call__(self):
        n = self.n
        self.cpu.dgemm("N", "N", n, self.cols, n, 1.0, self.a, n, self.b, n, 0.0, self.c, n)

    def describe(self):
        return (f"dgemm NN {self.n}x{self.cols}x{self.n} (the first {self.cols} of the "
                f"{self.n} output columns) per step")


def cpu_sample_cols(n, threads):
    """Output columns of one CPU step: one 96-column block of C (the CPU
    path's unit of parallel work) per thread."""
    return min(n, 96 * threads)


def cpu_steps(fn, steps, warmup):
    for _ in range(warmup):
        fn()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fn()
        times.append(time.perf_counter() - t0)
    return times


class RefLibrary:
    """The reference library itself (oracle/_ref/libhwyblas_ref.so: its own
    sources compiled against this repository's Highway-API shim), when it
    was built; single-threaded like the reference."""

    def __init__(self):
        from tests.oracle_lib import load_refblas
        self.ref = load_refblas()
        self.kind = "reference"

    def dgemm(self, *args):
        return self.ref.dgemm(*args)


def cpu_single_thread(cpu, n):
    """The single-threaded figure (the reference is single-threaded by
    design): best of 3 on a 32-column sample, with the port and, where it
    was built, with the reference library itself."""
    prev = cpu.threads
    cpu.set_threads(1)
    smp = DgemmSample(cpu, n, 32)
    best = min(cpu_steps(smp, 3, 1))
    cpu.set_threads(prev)
    out = {"value": smp.flops / best / 1e12, "unit": "TFLOP/s", "cores": 1,
           "sample": smp.describe() + ", best of 3", "kind": cpu.kind}
    lib = RefLibrary()
    if lib.ref is not None:
        smp_r = DgemmSample(lib, n, 32)
        best_r = min(cpu_steps(smp_r, 3, 1))
        smp_r()
        smp()
        out["reference_library"] = {
            "value": smp_r.flops / best_r / 1e12, "unit": "TFLOP/s", "cores": 1,
            "bit_identical_to_port": bool(np.array_equal(smp_r.c.view(np.uint64),
                                                         smp.c.view(np.uint64))),
            "note": "the reference's own sources compiled against this repository's "
                    "portable Highway-API shim (slower than a Highway build; the port, "
                    "bit-identical to it, is the timed baseline)"}
    return out


def workload_name(n):
    return (f"dgemm NN M=N=K={n}, C = A B, A and B entries u*2^e (u~U[-1,1], "
            f"e~U{{-{SPREAD}..{SPREAD}}}), FP64-accurate")


def workload_config(n):
    return {"workload": workload_name(n),
            "l2": f"inputs (2 x {8 * n * n >> 20} MiB FP64) larger than L2"}


def run_reference(args):
    """The reference arm: the reference's CPU implementation of the path, all
    host threads, `--warmup` untimed and `--steps` timed steps, each one
    bounded sample of the workload; ms_per_step is the measured step."""
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    cpu = CpuPath()
    threads = cpu_threads()
    cpu.set_threads(threads)
    n = args.n
    smp = DgemmSample(cpu, n, cpu_sample_cols(n, threads))
    times = cpu_steps(smp, args.steps, args.warmup)
    ms = 1e3 * sum(times) / len(times)
    tf = smp.flops / (ms * 1e-3) / 1e12
    single = cpu_single_thread(cpu, n)
    line = {
        "impl": "reference", "metric": METRIC, "value": tf, "unit": "TFLOP/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "ms_per_step": ms, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(n),
        "parallelism": f"{threads} host threads (column blocks of C)",
        "cpu_baseline": {"value": tf, "unit": "TFLOP/s", "cores": threads, "kind": cpu.kind,
                         "sample": smp.describe(), "single_thread": single},
        "e2e": {"value": tf, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference's Highway BLAS does not build here (Highway absent); this "
                "is the oracle port of its hot path with the same per-element order",
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm.

def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"bf16_tflops": FALLBACK_BF16_TFLOPS, "hbm_gbs": 6650.0}, "fallback"


def device_spread(torch, n, spread, gen):
    u = torch.rand(n * n, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
    e = torch.randint(-spread, spread + 1, (n * n,), device="cuda", generator=gen)
    return u * torch.exp2(e.to(torch.float64))


def normwise_error(torch, hb, a, b, c, n, cols):
    """||C[:, cols] - (A B)[:, cols]||_F / (||A||_F ||B[:, cols]||_F) with the
    exact product from the library's double-double reference kernel."""
    ref = torch.empty(n * len(cols), dtype=torch.float64, device="cuda")
    ci = torch.tensor(cols, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    hb.dgemm_ddref("N", "N", n, n, a, n, b, n, n, ci, ref, n)
    cm = c.view(n, n)[cols]        # rows of the row-major view = columns of C
    bm = b.view(n, n)[cols]
    num = torch.linalg.norm(cm.reshape(-1) - ref)
    den = torch.linalg.norm(a) * torch.linalg.norm(bm.reshape(-1))
    return float((num / den).item())


def timed(torch, stream, fn, steps):
    """Average milliseconds of fn() over `steps` calls, CUDA events on the
    library's stream, synchronized on both sides."""
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def int8_products(slices):
    return slices * (slices + 1) // 2


def run_dgemm(args, torch, hb, stream, dist, world, rank, local):
    """The headline: FP64-accurate DGEMM, emulated and plain, same inputs."""
    n = args.n
    flops = 2.0 * n ** 3
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)
    A = device_spread(torch, n, SPREAD, g)
    B = device_spread(torch, n, SPREAD, g)
    C = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    Cp = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # inputs come from torch's stream
    cols = list(range(0, n, max(1, n // 64)))[:64]
    used = [0]

    def emulated():
        used[0] = hb.dgemm_emulated("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, 0)

    def plain():
        hb.dgemm("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, Cp, n)

    for _ in range(args.warmup):
        emulated()
        plain()
    torch.cuda.synchronize()
    err_emul = normwise_error(torch, hb, A, B, C, n, cols)
    err_plain = normwise_error(torch, hb, A, B, Cp, n, cols)

    # Timed region: the emulated path, with the slice-product kernel timed.
    props = torch.cuda.get_device_properties(local)
    clocks = Clocks(f"GPU-{props.uuid}" if hasattr(props, "uuid") else local)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = hb.launch_count()
    hb.kernel_timer(hb.KERNEL_OZAKI_GEMM)
    hb.kernel_timer_read()
    ms = timed(torch, stream, emulated, args.steps)
    oz_ms, oz_launches = hb.kernel_timer_read()
    hb.kernel_timer(0)
    launches = hb.launch_count() - launches0
    dist.barrier()
    clk = clocks.stop()
    ms_max = dist.max(ms)
    value = world * flops / (ms_max * 1e-3) / 1e12

    # Plain FP64 path on the same inputs, DMMA kernel timed.
    hb.kernel_timer(hb.KERNEL_DMMA_GEMM)
    hb.kernel_timer_read()
    ms_plain = dist.max(timed(torch, stream, plain, max(3, args.steps // 2)))
    dm_ms, dm_launches = hb.kernel_timer_read()
    hb.kernel_timer(0)
    S = used[0]
    out = {
        "value": value, "ms": ms_max, "slices": S, "launches": launches, "clocks": clk,
        "err_emulated": err_emul, "err_plain": err_plain,
        "fp64_accurate": bool(err_emul <= err_plain),
        "plain": {"tflops": world * flops / (ms_plain * 1e-3) / 1e12, "ms": ms_plain,
                  "err": err_plain},
        "ozaki_kernel_ms_per_launch": oz_ms / max(1, oz_launches),
        "ozaki_launches_per_step": oz_launches / args.steps,
        "dmma_kernel_ms_per_launch": dm_ms / max(1, dm_launches),
    }

    # Slice sweep S = 3..8 (one warm and one timed call each).
    if not args.no_sweep and rank == 0:
        sweep = {}
        for s in range(3, 9):
            def one(s=s):
                hb.dgemm_emulated("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, s)
            one()
            t = timed(torch, stream, one, 1)
            sweep[str(s)] = {"tflops": flops / (t * 1e-3) / 1e12,
                             "err": normwise_error(torch, hb, A, B, C, n, cols)}
        out["sweep"] = sweep

    # End to end through the C ABI with pinned host buffers: A, B in, C out
    # (beta = 0: C is not read).
    ha = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
    hbuf = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
    hc = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
    ha.copy_(A.cpu())
    hbuf.copy_(B.cpu())
    an, bn, cn = ha.numpy(), hbuf.numpy(), hc.numpy()

    def e2e_call():
        hb.dgemm_emulated("N", "N", n, n, n, 1.0, an, n, bn, n, 0.0, cn, n, 0)

    e2e_call()
    dist.barrier()
    e2e_ms = dist.max(timed(torch, stream, e2e_call, args.e2e_steps))
    out["e2e"] = {"value": world * flops / (e2e_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                  "h2d_bytes_per_step": 2 * 8 * n * n, "d2h_bytes_per_step": 8 * n * n}
    del A, B, C, Cp
    return out


def householder_device(torch, n, cond, seed):
    """A = H1 diag(s) H2 (column-major, flat): H1, H2 products of 4 Householder
    reflectors from seeded Gaussian vectors, s geometric from 1 to 1/cond."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    s = torch.logspace(0.0, -float(np.log10(cond)), n, dtype=torch.float64, device="cuda")
    M = torch.diag(s)  # row-major storage of M; reflectors keep it dense
    for side in range(2):
        for _ in range(4):
            v = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
            v /= torch.linalg.norm(v)
            if side == 0:
                M -= 2.0 * torch.outer(v, v @ M)
            else:
                M -= 2.0 * torch.outer(M @ v, v)
    return M  # M's row-major storage is A^T column-major: solve with A = M^T


def solve_to_last_bit(torch, hb, n, nrhs, A, lu, ipiv, Bm, x0):
    """The solution of A x = b to about the last bit: x0 (the plain FP64
    solution) refined twice with the extra-precise residual
    (hwyblas_dresidual_dd) and the plain FP64 LU factors (bit-identical to the
    reference's). Column-major flat tensors."""
    x = x0.clone()
    r = torch.empty_like(x)
    for _ in range(2):
        hb.dresidual_dd(n, nrhs, A, n, x, n, Bm, n, r, n)
        hb.dgetrs("N", n, nrhs, lu, n, ipiv, r, n)
        x += r
    torch.cuda.synchronize()
    return x


def backward_error(torch, Mt, X, Bm):
    """Normwise backward error max_q ||b - A x||_inf / (||A||_inf ||x||_inf +
    ||b||_inf) of the columns x (rows of X) against b (rows of Bm), A = Mt^T
    given as the column-major data Mt (FP64 torch arithmetic, outside the
    product path)."""
    R = (Mt.t() @ X.t()).t() - Bm
    anorm = Mt.abs().sum(dim=0).max()
    num = R.abs().max(dim=1).values
    den = anorm * X.abs().max(dim=1).values + Bm.abs().max(dim=1).values
    return float((num / den).max().item())


def run_solvers(args, torch, hb, stream):
    """dgesv and dposv at n = args.gesv_n: plain FP64 against mixed. Forward
    errors are stated against the solution of A x = b to the last bit."""
    n = args.gesv_n
    res = {"n": n, "fwd_err": "||x - x*||_F / ||x*||_F, x* = the solution of A x = b to "
                              "the last bit (the plain solution after two steps of "
                              "extra-precise refinement)",
           "bwd_err": "max over columns of ||b - A x||_inf / (||A||_inf ||x||_inf + "
                      "||b||_inf)"}
    gesv_flops = lambda nrhs: 2.0 / 3.0 * n ** 3 + 2.0 * n * n * nrhs
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    cases = [(1e6, 1), (1e6, 64), (1e2, 1), (1e10, 1)]
    mats = {}
    for cond, nrhs in cases:
        if cond not in mats:
            mats[cond] = householder_device(torch, n, cond, 7)
        M = mats[cond]                      # the matrix A is M^T (column-major data of M)
        A = M.reshape(-1)
        g = torch.Generator(device="cuda").manual_seed(3)
        xt = torch.rand(nrhs, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        Bm = (M.t() @ xt.t()).t().contiguous()   # rows of Bm = columns of B = A xt
        torch.cuda.synchronize()
        out = {}
        sols = {}
        lu = None
        for kind in ("plain", "mixed"):
            best = None
            for _ in range(2):  # one warm-up, one timed
                a = A.clone()
                x = Bm.clone() if kind == "plain" else torch.zeros_like(Bm)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                if kind == "plain":
                    info = hb.dgesv(n, nrhs, a, n, ipiv, x, n)
                    it = None
                else:
                    info, it = hb.dgesv_mixed(n, nrhs, a, n, ipiv, Bm, n, x, n)
                torch.cuda.synchronize()
                best = time.perf_counter() - t0
            if kind == "plain":
                lu, piv = a, ipiv.clone()
            sols[kind] = x
            out[kind] = {"ms": best * 1e3, "tflops": gesv_flops(nrhs) / best / 1e12,
                         "solves_per_s": 1.0 / best, "info": info}
            if it is not None:
                out[kind]["iterations"] = it
        xs = solve_to_last_bit(torch, hb, n, nrhs, A, lu, piv, Bm, sols["plain"])
        for kind in ("plain", "mixed"):
            out[kind]["fwd_err"] = float((torch.linalg.norm(sols[kind] - xs) /
                                          torch.linalg.norm(xs)).item())
            out[kind]["bwd_err"] = backward_error(torch, M, sols[kind], Bm)
        out["speedup"] = out["plain"]["ms"] / out["mixed"]["ms"]
        out["mixed_err_le_plain"] = bool(out["mixed"]["fwd_err"] <= out["plain"]["fwd_err"])
        res[f"dgesv_cond{cond:g}_nrhs{nrhs}"] = out
        del lu, sols, xs
    del mats
    # dposv: SPD A = G G^T / n + 1e-3 I.
    g = torch.Generator(device="cuda").manual_seed(11)
    G = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    S = G @ G.t() / n + 1e-3 * torch.eye(n, dtype=torch.float64, device="cuda")
    del G
    xt = torch.rand(1, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    Bm = (S @ xt.t()).t().contiguous()
    A = S.reshape(-1)
    out = {}
    sols = {}
    posv_flops = n ** 3 / 3.0 + 2.0 * n * n
    for kind in ("plain", "mixed"):
        for _ in range(2):
            a = A.clone()
            x = Bm.clone() if kind == "plain" else torch.zeros_like(Bm)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if kind == "plain":
                info, it = hb.dposv("L", n, 1, a, n, x, n), None
            else:
                info, it = hb.dposv_mixed("L", n, 1, a, n, Bm, n, x, n)
            torch.cuda.synchronize()
            best = time.perf_counter() - t0
        sols[kind] = x
        out[kind] = {"ms": best * 1e3, "tflops": posv_flops / best / 1e12, "info": info}
        if it is not None:
            out[kind]["iterations"] = it
    # The last bit for the SPD system: an LU of A (any backward-stable
    # factorization serves the two correction steps).
    lu = A.clone()
    hb.dgetrf(n, n, lu, n, ipiv)
    xs = solve_to_last_bit(torch, hb, n, 1, A, lu, ipiv, Bm, sols["plain"])
    for kind in ("plain", "mixed"):
        out[kind]["fwd_err"] = float((torch.linalg.norm(sols[kind] - xs) /
                                      torch.linalg.norm(xs)).item())
        out[kind]["bwd_err"] = backward_error(torch, S, sols[kind], Bm)
    out["speedup"] = out["plain"]["ms"] / out["mixed"]["ms"]
    out["mixed_err_le_plain"] = bool(out["mixed"]["fwd_err"] <= out["plain"]["fwd_err"])
    res["dposv_spd_nrhs1"] = out
    return res


def run_batched(args, torch, hb, count=10000):
    """Config 5: `count` problems, n log-uniform in [8, 512], each dgetrf +
    dgetrs (nrhs uniform in 1..16) + dgemm (n x n x n), FP64 and FP32: the
    batched persistent launches against a per-problem loop of the
    single-problem routines over the same problems."""
    rng = np.random.default_rng(2024)
    ns = np.exp(rng.uniform(np.log(8), np.log(512), count)).astype(int).clip(8, 512)
    rhs = rng.integers(1, 17, count)
    flops = float(np.sum(2.0 / 3.0 * ns ** 3 + 2.0 * ns ** 2 * rhs + 2.0 * ns ** 3))
    out = {"count": count, "flops": flops}
    for prec, dtype in (("d", torch.float64), ("s", torch.float32)):
        sz_a = [int(n) * int(n) for n in ns]
        sz_b = [int(n) * int(r) for n, r in zip(ns, rhs)]
        A0 = torch.rand(sum(sz_a), dtype=dtype, device="cuda") * 2 - 1
        A = torch.empty_like(A0)
        B = torch.rand(sum(sz_b), dtype=dtype, device="cuda")
        G1 = torch.rand(sum(sz_a), dtype=dtype, device="cuda") * 2 - 1
        G2 = torch.rand(sum(sz_a), dtype=dtype, device="cuda") * 2 - 1
        G3 = torch.zeros(sum(sz_a), dtype=dtype, device="cuda")
        P = torch.zeros(int(ns.sum()), dtype=torch.int32, device="cuda")

        def views(buf, sizes):
            v, o = [], 0
            for s_ in sizes:
                v.append(buf[o:o + s_])
                o += s_
            return v

        va, vb = views(A, sz_a), views(B, sz_b)
        v1, v2, v3 = views(G1, sz_a), views(G2, sz_a), views(G3, sz_a)
        vp = views(P, [int(n) for n in ns])
        nl, rl = [int(n) for n in ns], [int(r) for r in rhs]
        # The C arrays of sizes and device pointers are built once, outside
        # the timed region, as a C caller keeps its arrays; the timed region
        # is the three library calls.
        cn, cr = hb.int_array(nl), hb.int_array(rl)
        ca, cb, cp = hb.ptr_array(va), hb.ptr_array(vb), hb.ptr_array(vp)
        c1, c2, c3 = hb.ptr_array(v1), hb.ptr_array(v2), hb.ptr_array(v3)

        def batched():
            hb.getrf_batched(cn, ca, cn, cp, precision=prec)
            hb.getrs_batched("N", cn, cr, ca, cn, cp, cb, cn, precision=prec)
            hb.gemm_batched("N", "N", cn, cn, cn, 1.0, c1, cn, c2, cn, 0.0, c3, cn,
                            precision=prec)

        times = []
        for _ in range(2):
            A.copy_(A0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            batched()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        t_batched = times[-1]
        entry = {"batched_ms": t_batched * 1e3, "tflops": flops / t_batched / 1e12}
        if prec == "d":
            # The per-problem loop of the single-problem routines over all
            # `count` problems (each call returns when its result is ready).
            def loop(ids):
                for i in ids:
                    n, r = nl[i], rl[i]
                    hb.dgetrf(n, n, va[i], n, vp[i])
                    hb.dgetrs("N", n, r, va[i], n, vp[i], vb[i], n)
                    hb.dgemm("N", "N", n, n, n, 1.0, v1[i], n, v2[i], n, 0.0, v3[i], n)

            loop(range(10))  # warm-up
            A.copy_(A0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            loop(range(count))
            torch.cuda.synchronize()
            t_loop = time.perf_counter() - t0
            entry["loop_ms"] = t_loop * 1e3
            entry["speedup_vs_loop"] = entry["loop_ms"] / entry["batched_ms"]
            # getrf alone, batched against the loop, same problems.
            A.copy_(A0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            hb.getrf_batched(cn, ca, cn, cp)
            torch.cuda.synchronize()
            t_gb = time.perf_counter() - t0
            A.copy_(A0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for i in range(count):
                hb.dgetrf(nl[i], nl[i], va[i], nl[i], vp[i])
            torch.cuda.synchronize()
            t_gl = time.perf_counter() - t0
            entry["getrf_batched_ms"] = t_gb * 1e3
            entry["getrf_loop_ms"] = t_gl * 1e3
            entry["getrf_speedup_vs_loop"] = t_gl / t_gb
        out["fp64" if prec == "d" else "fp32"] = entry
        del A0, A, B, G1, G2, G3, P
    return out


def run_widened(torch, hb, stream):
    """Throughput of the routines beyond the hot path (bit-identical to the
    oracle in the tests), device-resident inputs, CUDA events on the
    library's stream, best of 3 calls after one warm-up."""
    g = torch.Generator(device="cuda").manual_seed(3)

    def colmajor(rows, cols, dtype=torch.float64):
        return (torch.rand(cols, rows, dtype=dtype, device="cuda", generator=g) * 2 - 1).T

    def best(fn, reps=3):
        fn()
        return min(timed(torch, stream, fn, 1) for _ in range(reps))

    out = {}
    n = 8192
    a, b, c = colmajor(n, n), colmajor(n, n), colmajor(n, n)
    rows = [("dtrmm LLNN", lambda: hb.trmm("d", "L", "L", "N", "N", n, n, 1.0, a, n, c, n),
             n ** 3),
            ("dtrmm RUNN", lambda: hb.trmm("d", "R", "U", "N", "N", n, n, 1.0, a, n, c, n),
             n ** 3),
            ("dsymm LU", lambda: hb.symm("d", "L", "U", n, n, 1.0, a, n, b, n, 0.5, c, n),
             2 * n ** 3),
            ("dsyr2k LN", lambda: hb.syr2k("d", "L", "N", n, n, 1.0, a, n, b, n, 0.5, c, n),
             2 * n ** 3),
            ("dgemmtr LNN", lambda: hb.gemmtr("d", "L", "N", "N", n, n, 1.0, a, n, b, n, 0.5,
                                              c, n), n ** 3)]
    for name, fn, flops in rows:
        ms = best(fn)
        out[name] = {"n": n, "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
    # Inverse: LU of a diagonally dominant matrix, then TRTRI of its U and
    # GETRI (each call on a fresh copy; the copy is outside the timed call).
    m = colmajor(n, n)
    m.diagonal().add_(2.0 * n ** 0.5)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    lu = m.clone().T.contiguous().T
    hb.dgetrf(n, n, lu, n, ipiv)
    work = torch.zeros(64 * n, dtype=torch.float64, device="cuda")
    for name, call, flops in (("dtrtri UN", lambda x: hb.trtri("d", "U", "N", n, x, n),
                               n ** 3 / 3),
                              ("dgetri", lambda x: hb.getri("d", n, x, n, ipiv, work, 64 * n),
                               4 * n ** 3 / 3)):
        times = []
        for _ in range(3):
            x = lu.clone().T.contiguous().T
            torch.cuda.synchronize()
            times.append(timed(torch, stream, lambda: call(x), 1))
        ms = min(times[1:])
        out[name] = {"n": n, "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
    del a, b, c, m, lu, work
    nz = 4096
    for p, dt in (("z", torch.complex128), ("c", torch.complex64)):
        za, zb, zc = colmajor(nz, nz, dt), colmajor(nz, nz, dt), colmajor(nz, nz, dt)
        ms = best(lambda: hb.zgemm(p, "N", "N", nz, nz, nz, 1.0, za, nz, zb, nz, 0.0, zc, nz))
        out[p + "gemm NN"] = {"n": nz, "ms": ms, "tflops": 8 * nz ** 3 / (ms * 1e-3) / 1e12}
        # Complex LU of a diagonally dominant matrix and Cholesky of a
        # Hermitian one with a dominant diagonal (fresh copies, copy untimed).
        za.diagonal().add_(2.0 * nz ** 0.5)
        herm = (zb + zb.conj().T) / 2
        herm.diagonal().add_(2.0 * nz ** 0.5)
        herm = herm.T.contiguous().T
        zp = torch.zeros(nz, dtype=torch.int32, device="cuda")
        for name, src, call, flops in (
                (p + "getrf", za, lambda x: hb.zgetrf(p, nz, nz, x, nz, zp), 8 * nz ** 3 / 3),
                (p + "potrf L", herm, lambda x: hb.zpotrf(p, "L", nz, x, nz), 4 * nz ** 3 / 3)):
            times = []
            for _ in range(3):
                x = src.clone().T.contiguous().T
                torch.cuda.synchronize()
                times.append(timed(torch, stream, lambda: call(x), 1))
            ms = min(times[1:])
            out[name] = {"n": nz, "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
        del za, zb, zc, herm
    out["note"] = ("useful flops: trmm n^3, symm/syr2k 2n^3, gemmtr n^3, trtri n^3/3, "
                   "getri 4n^3/3, complex gemm 8n^3, complex getrf 8n^3/3, complex potrf "
                   "4n^3/3")
    return out


def run_auto_slices(torch, hb, stream, n):
    """The automatic slice count on the headline's shape at three exponent
    spreads: the count chosen, its throughput, and its error next to the
    plain FP64 path's (both against the double-double product)."""
    out = {}
    flops = 2.0 * n ** 3
    C = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    Cp = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    cols = list(range(0, n, max(1, n // 64)))[:64]
    for spread in (0, 8, 30):
        g = torch.Generator(device="cuda").manual_seed(99 + spread)
        A = device_spread(torch, n, spread, g)
        B = device_spread(torch, n, spread, g)
        torch.cuda.synchronize()
        used = [0]

        def one():
            used[0] = hb.dgemm_emulated("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, 0)
        one()
        t = timed(torch, stream, one, 2)
        e = normwise_error(torch, hb, A, B, C, n, cols)
        hb.dgemm("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, Cp, n)
        pe = normwise_error(torch, hb, A, B, Cp, n, cols)
        out[f"spread{spread}"] = {"slices": used[0], "tflops": flops / (t * 1e-3) / 1e12,
                                  "err_emulated": e, "err_plain": pe,
                                  "fp64_accurate": bool(e <= pe)}
        del A, B
    return out


def run_small_configs(torch, hb, stream, cpu, fp64_peak):
    """dgemm NN 1024^3 (alpha 1.5, beta 0.5), dtrsm L/L/N/U 4096 x 512 and
    dgetrf 4096, entries U[-1, 1]: device-timed TFLOP/s with the fraction of
    the FP64 tensor-pipe peak, the C-ABI time with host buffers, and the CPU
    path single-threaded on the same inputs with bit equality (and ipiv
    equality and the LU residual ratio ||PA - LU||_1 / (n ||A||_1 eps))."""
    rng = np.random.default_rng(2025)
    res = {}

    def dev(x):
        return torch.from_numpy(np.asfortranarray(x).ravel(order="F").copy()).cuda()

    def host(t, rows, cols):
        return np.asfortranarray(t.cpu().numpy().reshape(cols, rows).T)

    def roof(tflops):
        return {"bound": "tensor", "achieved": tflops, "peak": fp64_peak,
                "unit": "TFLOP/s (FP64)", "frac": tflops / fp64_peak,
                "peak_source": "measured DMMA issue rate (hwyblas_fp64_peak_tflops)"}

    def cpu_time(fn, reps):
        cpu.set_threads(1)
        best = min(cpu_steps(fn, reps, 0))
        cpu.set_threads(cpu_threads())
        return best

    # Config 1: dgemm.
    n = 1024
    a, b, c = (rng.uniform(-1, 1, (n, n)) for _ in range(3))
    a, b, c = np.asfortranarray(a), np.asfortranarray(b), np.asfortranarray(c)
    flops = 2.0 * n ** 3
    A, B, C0 = dev(a), dev(b), dev(c)
    Cw = C0.clone()
    gemm = lambda: hb.dgemm("N", "N", n, n, n, 1.5, A, n, B, n, 0.5, Cw, n)
    for _ in range(3):
        gemm()
    ms = timed(torch, stream, gemm, 50)
    Cw.copy_(C0)
    torch.cuda.synchronize()
    gemm()
    c_gpu = host(Cw, n, n)
    hc = c.copy(order="F")
    t0 = time.perf_counter()
    for _ in range(10):
        hc[:] = c
        hb.dgemm("N", "N", n, n, n, 1.5, a, n, b, n, 0.5, hc, n)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / 10
    entry = {"workload": "dgemm NN M=N=K=1024, alpha 1.5, beta 0.5, U[-1,1]",
             "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12,
             "e2e": {"ms": e2e_ms, "tflops": flops / (e2e_ms * 1e-3) / 1e12,
                     "h2d_bytes": 3 * 8 * n * n, "d2h_bytes": 8 * n * n}}
    entry["roofline"] = roof(entry["tflops"])
    if cpu is not None:
        cc = c.copy(order="F")
        cpu.dgemm("N", "N", n, n, n, 1.5, a, n, b, n, 0.5, cc, n)
        entry["bit_identical_to_cpu"] = bool(np.array_equal(cc.view(np.uint64),
                                                            c_gpu.view(np.uint64)))
        cw = c.copy(order="F")

        def cpu_gemm():
            cw[:] = c
            cpu.dgemm("N", "N", n, n, n, 1.5, a, n, b, n, 0.5, cw, n)
        t = cpu_time(cpu_gemm, 3)
        entry["cpu"] = {"ms": t * 1e3, "tflops": flops / t / 1e12, "cores": 1,
                        "kind": cpu.kind}
    res["config1"] = entry

    # Config 2a: dtrsm L/L/N/U, M = 4096, N = 512 (m n ka flops). As
    # configured, the unit lower triangle's entries are U[-1, 1] and the
    # solution overflows; the reference tests' scaled variant (off-diagonal
    # times 1/ka) is the well-posed one that the bits are compared on.
    m, nr = 4096, 512
    t_raw = np.asfortranarray(rng.uniform(-1, 1, (m, m)))
    bb = np.asfortranarray(rng.uniform(-1, 1, (m, nr)))
    t_scaled = np.asfortranarray(t_raw / m)
    flops = float(m) * nr * m
    out2 = {}
    for label, tri in (("configured", t_raw), ("scaled", t_scaled)):
        T, B0 = dev(tri), dev(bb)
        Bw = B0.clone()
        trsm = lambda: hb.dtrsm("L", "L", "N", "U", m, nr, 1.0, T, m, Bw, m)
        for _ in range(2):
            Bw.copy_(B0)
            torch.cuda.synchronize()
            trsm()
        times = []
        for _ in range(5):
            Bw.copy_(B0)
            torch.cuda.synchronize()
            times.append(timed(torch, stream, trsm, 1))
        ms = min(times)
        e = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
        e["roofline"] = roof(e["tflops"])
        if cpu is not None:
            bw = bb.copy(order="F")
            cpu.dtrsm("L", "L", "N", "U", m, nr, 1.0, tri, m, bw, m)
            if label == "scaled":
                e["bit_identical_to_cpu"] = bool(np.array_equal(
                    bw.view(np.uint64), host(Bw, m, nr).view(np.uint64)))
                cw = bb.copy(order="F")

                def cpu_trsm():
                    cw[:] = bb
                    cpu.dtrsm("L", "L", "N", "U", m, nr, 1.0, tri, m, cw, m)
                t = cpu_time(cpu_trsm, 2)
                e["cpu"] = {"ms": t * 1e3, "tflops": flops / t / 1e12, "cores": 1,
                            "kind": cpu.kind}
        out2["dtrsm_" + label] = e
    out2["dtrsm_workload"] = ("dtrsm side=L uplo=L trans=N diag=U, M=4096 N=512; "
                              "configured: off-diagonal U[-1,1]; scaled: times 1/4096")

    # Config 2b: dgetrf n = 4096.
    n = 4096
    a = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    flops = 2.0 / 3.0 * n ** 3
    A0 = dev(a)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    times = []
    for it in range(4):
        Aw = A0.clone()
        torch.cuda.synchronize()
        times.append(timed(torch, stream, lambda: hb.dgetrf(n, n, Aw, n, ipiv), 1))
    ms = min(times[1:])
    lu = Aw.view(n, n).t()  # lu[i, j] = LU(i, j)
    L = torch.tril(lu, -1) + torch.eye(n, dtype=torch.float64, device="cuda")
    U = torch.triu(lu)
    piv = ipiv.cpu().numpy()
    perm = np.arange(n)
    for i in range(n):
        j = piv[i] - 1
        perm[i], perm[j] = perm[j], perm[i]
    Am = A0.view(n, n).t()
    PA = Am[torch.from_numpy(perm).cuda()]
    eps = np.finfo(np.float64).eps / 2
    norm1 = lambda x: float(x.abs().sum(dim=0).max().item())
    ratio = norm1(L @ U - PA) / n / norm1(Am) / eps
    e = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12, "lu_residual_ratio": ratio,
         "ratio_definition": "||P L U - A||_1 / (n ||A||_1 eps), eps = 2^-53 (LAPACK xGET01)"}
    e["roofline"] = roof(e["tflops"])
    if cpu is not None:
        aw = a.copy(order="F")
        pw = np.zeros(n, np.int32)
        cpu.set_threads(1)
        t0 = time.perf_counter()
        cpu.dgetrf(n, n, aw, n, pw)
        t = time.perf_counter() - t0
        cpu.set_threads(cpu_threads())
        e["ipiv_equal_to_cpu"] = bool(np.array_equal(pw, piv))
        e["bit_identical_to_cpu"] = bool(np.array_equal(
            aw.view(np.uint64), host(Aw, n, n).view(np.uint64)))
        e["cpu"] = {"ms": t * 1e3, "tflops": flops / t / 1e12, "cores": 1, "kind": cpu.kind}
    out2["dgetrf"] = e
    out2["dgetrf_workload"] = "dgetrf n=4096, U[-1,1], partial pivoting (2/3 n^3 flops)"
    res["config2"] = out2
    return res


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = Dist(world, rank, local, "nccl")
    import hwyblas_b200 as hb
    lib = hb.lib()
    stream = torch.cuda.Stream()
    hb.set_stream(stream)
    n = args.n
    d = run_dgemm(args, torch, hb, stream, dist, world, rank, local)

    peaks, peak_kind = measured_peaks()
    int8_inferred = 2.0 * float(peaks.get("bf16_tflops", FALLBACK_BF16_TFLOPS))
    fp64_peak = float(lib.hwyblas_fp64_peak_tflops())
    int8_peak = float(lib.hwyblas_int8_peak_tops())
    S = d["slices"]
    # Dominant kernel: the slice-product GEMM. Algorithmic work = INT8
    # multiply-adds of all S(S+1)/2 slice products, 2 n^3 ops each, spread
    # over the launches of one step.
    per_step_ops = int8_products(S) * 2.0 * n ** 3 if S > 0 else 0.0
    per_launch_ops = per_step_ops / max(1.0, d["ozaki_launches_per_step"])
    oz_ms = d["ozaki_kernel_ms_per_launch"]
    achieved = per_launch_ops / (oz_ms * 1e-3) / 1e12 if oz_ms > 0 else None
    # DRAM traffic of the slice-product kernel per launch at n = 8192, S = 8
    # (ncu dram__bytes_read.sum + dram__bytes_write.sum of this workload, a
    # one-pass capture): high pass 7.886e9 B, low pass 4.341e9 B. Other
    # shapes have no measured figure.
    traffic = (7.886e9 + 4.341e9) / 2.0 if (n == 8192 and S == 8) else None
    dm_ms = d["dmma_kernel_ms_per_launch"]
    dm_achieved = 2.0 * n ** 3 / (dm_ms * 1e-3) / 1e12 if dm_ms > 0 else None

    cpu = None
    cpu_path = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_path = CpuPath()
        threads = cpu_threads()
        cpu_path.set_threads(threads)
        smp = DgemmSample(cpu_path, n, cpu_sample_cols(n, threads))
        times = cpu_steps(smp, 3, 1)
        tf = smp.flops / (sum(times) / len(times)) / 1e12
        cpu = {"value": tf, "unit": "TFLOP/s", "cores": threads, "kind": cpu_path.kind,
               "sample": smp.describe() + ", mean of 3",
               "single_thread": cpu_single_thread(cpu_path, n)}

    small = None
    if rank == 0 and world == 1 and not args.no_small:
        small = run_small_configs(torch, hb, stream, cpu_path, fp64_peak)
    auto = None
    if rank == 0 and world == 1 and not args.no_sweep:
        auto = run_auto_slices(torch, hb, stream, n)

    solvers = None
    if rank == 0 and world == 1 and not args.no_dgesv:
        solvers = run_solvers(args, torch, hb, stream)
    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = run_batched(args, torch, hb)
    widened = None
    if rank == 0 and world == 1 and not args.no_widened:
        try:
            widened = run_widened(torch, hb, stream)
        except Exception as exc:  # a side measurement never costs the bench line
            widened = {"error": repr(exc)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": d["value"], "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": d["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int8 slices -> f64", "data": "synthetic (seeded)",
            "config": workload_config(n),
            "path": "emulated FP64 (Ozaki INT8 slices on tcgen05), slice count chosen "
                    "from the inputs' exponent spread",
            "slices": S, "parallelism": f"replicas x{world}",
            "fp64_accurate": d["fp64_accurate"],
            "error": {"emulated": d["err_emulated"], "plain": d["err_plain"],
                      "measure": "normwise ||C - AB||_F / (||A||_F ||B||_F) on 64 columns "
                                 "against a double-double product"},
            "plain": d["plain"],
            "speedup_vs_plain": d["plain"]["ms"] / d["ms"],
            "e2e": d["e2e"],
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": int8_peak,
                         "unit": "TOPS (INT8)",
                         "frac": achieved / int8_peak if achieved else None,
                         "traffic": traffic,
                         "traffic_unit": "bytes per launch (DRAM, ncu)",
                         "kernel": "OzakiGemmKernel (slice products, "
                                   f"{d['ozaki_launches_per_step']:.0f} launches per step)",
                         "peak_source": "measured tcgen05.mma kind::i8 issue rate "
                                        "(hwyblas_int8_peak_tops)",
                         "peak_inferred": int8_inferred,
                         "peak_inferred_source": f"2 x bf16_tflops of {peak_kind} "
                                                 "MEASURED_PEAKS"},
            "roofline_plain": {"bound": "tensor", "achieved": dm_achieved,
                               "peak": fp64_peak, "unit": "TFLOP/s (FP64)",
                               "frac": dm_achieved / fp64_peak if dm_achieved else None,
                               "kernel": "DgemmDmmaKernel",
                               "peak_source": "measured DMMA issue rate "
                                              "(hwyblas_fp64_peak_tflops)"},
            "cpu_baseline": cpu,
            "clocks": d["clocks"],
            "gpu_launches": d["launches"],
        }
        if "sweep" in d:
            line["slice_sweep"] = d["sweep"]
        if auto is not None:
            line["auto_slices"] = auto
        if small is not None:
            line["config1"] = small["config1"]
            line["config2"] = small["config2"]
        if solvers is not None:
            line["solvers"] = solvers
        if batched is not None:
            line["batched"] = batched
        if widened is not None:
            line["widened"] = widened
        print(json.dumps(line), flush=True)
    dist.close()
    return 0


def run_case(args):
    """One warm-up and one profiled call of a single hot-path piece."""
    import torch
    import hwyblas_b200 as hb
    torch.cuda.set_device(0)
    n = args.gesv_n
    g = torch.Generator(device="cuda").manual_seed(1)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    if args.case in ("trtri", "getri", "trmm", "zgemm", "zgetrf", "zpotrf"):
        n = args.n
        ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
        dt = torch.complex128 if args.case[0] == "z" else torch.float64
        a0 = torch.rand(n * n, dtype=dt, device="cuda", generator=g) * 2 - 1
        if args.case in ("trtri", "getri", "zgetrf", "zpotrf"):
            a0.view(n, n).diagonal().add_(2.0 * n ** 0.5)
        if args.case == "zpotrf":
            a0 = ((a0.view(n, n) + a0.view(n, n).conj().T) / 2).contiguous().view(-1)
        if args.case in ("trtri", "getri"):
            hb.dgetrf(n, n, a0, n, ipiv)
        other = torch.rand(n * n, dtype=dt, device="cuda", generator=g) * 2 - 1
        work = torch.zeros(64 * n, dtype=torch.float64, device="cuda")
        if args.case == "trtri":
            call = lambda a: hb.trtri("d", "U", "N", n, a, n)
        elif args.case == "getri":
            call = lambda a: hb.getri("d", n, a, n, ipiv, work, 64 * n)
        elif args.case == "trmm":
            call = lambda a: hb.trmm("d", "L", "L", "N", "N", n, n, 1.0, other, n, a, n)
        elif args.case == "zgetrf":
            call = lambda a: hb.zgetrf("z", n, n, a, n, ipiv)
        elif args.case == "zpotrf":
            call = lambda a: hb.zpotrf("z", "L", n, a, n)
        else:
            c = torch.zeros_like(a0)
            call = lambda a: hb.zgemm("z", "N", "N", n, n, n, 1.0, a, n, other, n, 0.0, c, n)
    elif args.case == "trsm":
        # dtrsm L/L/N/U, n x nrhs (the configured 4096 x 512 with --gesv-n 4096
        # --nrhs 512): the triangle is fixed, B is the operand solved in place.
        tri = torch.rand(n * n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        a0 = torch.rand(n * args.nrhs, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        call = lambda x: hb.dtrsm("L", "L", "N", "U", n, args.nrhs, 1.0, tri, n, x, n)
    elif args.case == "leaf":
        a0 = torch.rand(n * 16, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        call = lambda a: hb.dgetrf2(n, 16, a, n, ipiv)
    elif args.case in ("potrf", "posv-mixed"):
        # SPD A = G G^T / n + 1e-3 I, G Gaussian (the dposv configuration).
        gm = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        a0 = torch.addmm(torch.eye(n, dtype=torch.float64, device="cuda"), gm, gm.T,
                         beta=1e-3, alpha=1.0 / n).contiguous().view(-1)
        del gm
        b = torch.rand(n * args.nrhs, dtype=torch.float64, device="cuda", generator=g)
        x = torch.zeros_like(b)
        if args.case == "potrf":
            call = lambda a: hb.dpotrf("L", n, a, n)
        else:
            call = lambda a: hb.dposv_mixed("L", n, args.nrhs, a, n, b, n, x, n)
    else:
        a0 = torch.rand(n * n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        b = torch.rand(n * args.nrhs, dtype=torch.float64, device="cuda", generator=g)
        x = torch.zeros_like(b)
        if args.case == "getrf":
            call = lambda a: hb.dgetrf(n, n, a, n, ipiv)
        elif args.case == "gesv":
            call = lambda a: hb.dgesv(n, args.nrhs, a, n, ipiv, b.clone(), n)
        else:
            call = lambda a: hb.dgesv_mixed(n, args.nrhs, a, n, ipiv, b, n, x, n)
    a = a0.clone()
    call(a)  # warm-up
    a = a0.clone()
    torch.cuda.synchronize()
    prof = None
    if args.kernels:
        from torch.profiler import ProfilerActivity, profile
        prof = profile(activities=[ProfilerActivity.CUDA])
        prof.__enter__()
    t0 = time.perf_counter()
    r = call(a)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    out = {"case": args.case, "n": n, "nrhs": args.nrhs, "ms": ms, "result": r}
    if prof is not None:
        prof.__exit__(None, None, None)
        rows = []
        for e in prof.key_averages():
            t = getattr(e, "device_time_total", 0) or 0
            if t > 0:
                name = e.key.replace("(anonymous namespace)::", "").replace("void ", "")
                rows.append((t, e.count, name.split("(")[0][-70:]))
        rows.sort(reverse=True)
        total = sum(r_[0] for r_ in rows)
        out["kernel_sum_ms"] = total / 1e3
        out["kernels"] = [{"name": k, "launches": c, "ms": t / 1e3,
                           "share": t / total if total else 0.0} for t, c, k in rows[:12]]
    print(json.dumps(out))
    return 0


def main():
    args = parse()
    if args.case is not None:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
