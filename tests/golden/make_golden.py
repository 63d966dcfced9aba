"""Generates the golden LU / Cholesky fixtures of tests/golden/ from the
reference's own LAPACK drivers (src/lapack/getrf.cc, potrf.cc,
environment.cc compiled unmodified into oracle/_ref/libhwyref.so by
`make -C oracle ref`, linked to the oracle's BLAS restatement).

Run from the repository root after building oracle/_ref:

    python tests/golden/make_golden.py

Inputs are seeded uniform[-1, 1] matrices (SPD ones G G^T / n + n I for the
Cholesky cases); each case stores the input, the reference's output factors,
pivots and INFO. tests/test_golden.py replays them against the oracle (CPU)
and against the library (GPU).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.oracle_lib import load_ref, ref_call_getrf, ref_call_potrf  # noqa: E402

GETRF = [(1, 1, False), (17, 17, False), (33, 20, True), (20, 33, False),
         (100, 64, True), (65, 65, False), (129, 129, False), (150, 70, True)]
POTRF = [(33, "L", False), (70, "U", False), (100, "L", True), (130, "U", False)]


def main():
    lib = load_ref()
    if lib is None:
        sys.exit("oracle/_ref/libhwyref.so is missing: run `make -C oracle ref` first")
    rng = np.random.default_rng(20261203)
    out = {}
    for i, (m, n, rec) in enumerate(GETRF):
        lda = m + 2
        a = np.asfortranarray(rng.uniform(-1, 1, (lda, n)))
        if i == 3:
            a[:, 5] = 0.0  # a zero column: INFO = 6
        piv = np.zeros(min(m, n), np.int32)
        f = a.copy(order="F")
        info = ref_call_getrf(lib, rec, m, n, f, lda, piv)
        key = f"getrf_{m}x{n}_{'rec' if rec else 'blk'}"
        out[key + "_a"] = a
        out[key + "_lu"] = f
        out[key + "_ipiv"] = piv
        out[key + "_info"] = np.array([info, lda], np.int32)
    for n, uplo, rec in POTRF:
        g = rng.uniform(-1, 1, (n, n))
        a = np.asfortranarray(g @ g.T / n + n * np.eye(n))
        f = a.copy(order="F")
        info = ref_call_potrf(lib, rec, uplo, n, f, n)
        key = f"potrf_{n}_{uplo}_{'rec' if rec else 'blk'}"
        out[key + "_a"] = a
        out[key + "_l"] = f
        out[key + "_info"] = np.array([info], np.int32)
    path = os.path.join(HERE, "lapack_ref.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(GETRF) + len(POTRF)} cases)")


if __name__ == "__main__":
    main()
