"""Builds libhwyblas_b200.so in-tree with nvcc for sm_100a.

The library is one shared object: the CUDA kernels (csrc/*.cu) and the C++
host layer (csrc/*.cc) behind the C ABI declared in include/hwyblas_b200.h.
The CUDA runtime is linked statically; the driver's cuTensorMapEncodeTiled is
reached through the runtime's entry-point query, so libcuda is only needed at
run time.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhwyblas_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

# -fmad=false: no contraction of a*b + c into an FMA (the reference builds
# with -ffp-contract=off); every FMA in the kernels is an explicit fma().
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "-Wno-deprecated-gpu-targets",
]


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cc")):
            out.append(os.path.join(CSRC, name))
    return out


def _deps():
    deps = sources() + [os.path.join(CSRC, n) for n in os.listdir(CSRC)
                        if n.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "hwyblas_b200.h"))
    deps.append(os.path.abspath(__file__))
    return deps


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def build(force=False, verbose=False, jobs=None):
    """Compiles every source to an object (in parallel) and links the library."""
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    procs = []
    objs = []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj)
                and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in _deps())):
            continue
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"), file=sys.stderr)
    if failed:
        msg = "\n".join(f"{s}:\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
           "-Xcompiler", "-fPIC", "-o", LIB + ".tmp"] + objs + ["-lpthread"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
