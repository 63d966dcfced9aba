#!/usr/bin/env python
"""Benchmark of the level-3 hot path on B200 (one JSON line on rank 0).

Headline metric: FP64-accurate TFLOP/s of DGEMM at M = N = K = 8192 (column-
major NN, A, B, C uniform[-1, 1] from a seed, alpha 1.5, beta 0.5), i.e.
2*8192^3 useful FP64 flops per step, on the fastest FP64-accurate path of the
library (the plain FP64 tensor-pipe GEMM; the emulated path reports beside
it when available). The dgesv n=16384 part of the metric is reported in the
"dgesv" object when enabled.

value  : device-timed, inputs resident in HBM, CUDA events on the library's
         stream, max over ranks; whole-job TFLOP/s (sum over ranks).
e2e    : the same metric through the public C ABI with pinned HOST buffers:
         every step copies A, B, C in and C out inside the timed region.
Replicas only: every rank runs its own 8192^3 product (weak scaling).

--impl reference times the reference's CPU implementation of the path on this
host's cores (the oracle port of the reference's hot path, all threads) on a
bounded sample of the same workload.
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
ALPHA, BETA = 1.5, 0.5
METRIC = "FP64-accurate TFLOP/s: dgemm n=8192, dgesv n=16384; emulated/mixed vs plain"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=N_DEFAULT)
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--no-cpu-baseline", action="store_true")
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
# CPU baseline: the oracle port of the reference's hot path on host threads.

def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_dgemm_sample(n, cols, steps, threads):
    """TFLOP/s of the reference's DGEMM order (oracle port) on an n x cols x n
    slice of the workload (a bounded sample: cols of the n output columns)."""
    from tests.oracle_lib import Oracle
    orc = Oracle()
    orc.set_threads(threads)
    rng = np.random.default_rng(7)
    a = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    b = np.asfortranarray(rng.uniform(-1, 1, (n, cols)))
    c = np.asfortranarray(rng.uniform(-1, 1, (n, cols)))
    orc.dgemm("N", "N", n, cols, n, ALPHA, a, n, b, n, BETA, c, n)  # warm-up
    best = float("inf")
    for _ in range(steps):
        t0 = time.perf_counter()
        orc.dgemm("N", "N", n, cols, n, ALPHA, a, n, b, n, BETA, c, n)
        best = min(best, time.perf_counter() - t0)
    flops = 2.0 * n * cols * n
    return flops / best / 1e12, f"dgemm NN {n}x{cols}x{n} (1/{n // cols} of the output columns), best of {steps}"


# ---------------------------------------------------------------------------

def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    threads = cpu_threads()
    n = args.n
    cols = max(64, n // 8)
    steps = max(1, args.steps if args.steps < 5 else 3)
    tf, sample = cpu_dgemm_sample(n, cols, steps, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": tf, "unit": "TFLOP/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": 1, "higher_is_better": True,
        "ms_per_step": 2.0 * n ** 3 / (tf * 1e12) * 1e3, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded uniform[-1,1])",
        "config": {"workload": f"dgemm NN M=N=K={n} alpha=1.5 beta=0.5 (column-major)",
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": tf, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": tf, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference's Highway BLAS does not build here (Highway absent); "
                "this is the oracle port of its hot path with the same per-element order",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = Dist(world, rank, local, "nccl")
    import hwyblas_b200 as hb
    lib = hb.lib()
    n = args.n
    flops = 2.0 * n ** 3
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)
    A = torch.rand(n * n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    B = torch.rand(n * n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    C0 = torch.rand(n * n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    C = C0.clone()
    torch.cuda.synchronize()  # inputs come from torch's stream
    stream = torch.cuda.Stream()
    hb.set_stream(stream)
    peak = float(lib.hwyblas_fp64_peak_tflops())

    def step():
        hb.dgemm("N", "N", n, n, n, ALPHA, A, n, B, n, BETA, C, n)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    props = torch.cuda.get_device_properties(local)
    clocks = Clocks(f"GPU-{props.uuid}" if hasattr(props, "uuid") else local)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = hb.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    launches = hb.launch_count() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = dist.max(ms)
    value = world * flops / (ms_max * 1e-3) / 1e12

    # End to end through the C ABI with pinned host buffers.
    ha = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
    hbuf = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
    hc = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
    ha.copy_(A.cpu())
    hbuf.copy_(B.cpu())
    hc.copy_(C0.cpu())
    an, bn, cn = ha.numpy(), hbuf.numpy(), hc.numpy()
    hb.dgemm("N", "N", n, n, n, ALPHA, an, n, bn, n, BETA, cn, n)  # warm-up
    dist.barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.e2e_steps):
        hb.dgemm("N", "N", n, n, n, ALPHA, an, n, bn, n, BETA, cn, n)
    f1.record(stream)
    f1.synchronize()
    e2e_ms = dist.max(f0.elapsed_time(f1) / args.e2e_steps)
    e2e = world * flops / (e2e_ms * 1e-3) / 1e12

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        tf, sample = cpu_dgemm_sample(n, max(64, n // 8), 3, threads)
        cpu = {"value": tf, "unit": "TFLOP/s", "cores": threads, "kind": "port",
               "sample": sample}

    if rank == 0:
        achieved = flops / (ms * 1e-3) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded uniform[-1,1])",
            "config": {"workload": f"dgemm NN M=N=K={n} alpha=1.5 beta=0.5, FP64 DMMA path "
                                   "(bit-identical to the reference)",
                       "path": "plain FP64 tensor pipe", "parallelism": f"replicas x{world}",
                       "l2": "inputs (3 x 512 MiB) larger than L2"},
            "e2e": {"value": e2e, "unit": "TFLOP/s", "h2d_bytes_per_step": 3 * 8 * n * n,
                    "d2h_bytes_per_step": 8 * n * n},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                         "traffic": None,
                         "peak_source": "measured FP64 DMMA issue rate on this GPU "
                                        "(hwyblas_fp64_peak_tflops); no FP64 figure in "
                                        "MEASURED_PEAKS.json",
                         "kernel": "DgemmDmmaKernel<true>"},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    dist.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
