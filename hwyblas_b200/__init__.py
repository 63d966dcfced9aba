"""hwyBLAS-B200: hwyBLAS's level-3 hot path on NVIDIA B200 (sm_100a).

The product is the shared library ``libhwyblas_b200.so`` whose C ABI
(``include/hwyblas_b200.h``) replaces the reference's Fortran BLAS/LAPACK and
CBLAS entry points. This package loads it and exposes thin Python wrappers
with the reference's routine names and argument order (Fortran convention:
column-major, 1-based pivots, INFO returned), accepting NumPy arrays (host)
or CUDA tensors (device, used in place). There is no CPU fallback: if the
library is missing or cannot load, every call raises.
"""
import ctypes
import os

from . import _abi

__all__ = [
    "lib", "dgemm", "sgemm", "dtrsm", "strsm", "dsyrk", "idamax", "dlaswp", "dgetrf",
    "dgetrf2", "dgetrs", "dgesv", "slaswp", "sgetrf", "sgetrf2", "sgetrs", "sgesv",
    "dpotrf", "dpotrf2", "dpotrs", "dposv", "ssyrk", "spotrf", "spotrf2", "spotrs",
    "sposv", "cblas_dgemm", "cblas_sgemm", "cblas_dtrsm", "cblas_strsm", "cblas_idamax",
    "ErrorCapture", "launch_count", "set_stream", "dgemm_emulated", "dgemm_ddref", "dresidual_dd",
    "idamax_noalloc", "dgesv_mixed", "dposv_mixed", "set_mixed_slices",
    "kernel_timer", "kernel_timer_read", "KERNEL_DMMA_GEMM", "KERNEL_OZAKI_GEMM",
    "KERNEL_LU_LEAF", "getrf_batched", "getrs_batched", "gemm_batched",
    "trsm_batched", "int_array", "ptr_array", "symm", "syr2k", "gemmtr", "trmm", "cblas_level3", "getri", "trtri", "gerfs", "zgemm", "ztrsm", "zgetrf", "zlaswp", "zgetrs", "zgesv",
    "zpotrf", "zpotrs", "zposv", "zherk",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhwyblas_b200.so")
_lib = None


def lib():
    """The loaded product library (built by hwyblas_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m hwyblas_b200.build`"
                " (there is no CPU fallback)")
        _lib = _abi.declare(ctypes.CDLL(LIB_PATH))
    return _lib


from ._api import (  # noqa: E402  (needs lib())
    dgemm, sgemm, dtrsm, strsm, dsyrk, idamax, dlaswp, dgetrf, dgetrf2, dgetrs,
    dgesv, slaswp, sgetrf, sgetrf2, sgetrs, sgesv, dpotrf, dpotrf2, dpotrs, dposv,
    ssyrk, spotrf, spotrf2, spotrs, sposv,
    cblas_dgemm, cblas_sgemm, cblas_dtrsm, cblas_strsm, cblas_idamax, ErrorCapture, launch_count, set_stream,
    dgemm_emulated, dgemm_ddref, dresidual_dd, idamax_noalloc, dgesv_mixed, dposv_mixed,
    set_mixed_slices, kernel_timer, kernel_timer_read, KERNEL_DMMA_GEMM,
    KERNEL_OZAKI_GEMM, KERNEL_LU_LEAF, getrf_batched, getrs_batched, gemm_batched,
    trsm_batched, int_array, ptr_array, symm, syr2k, gemmtr, trmm, cblas_level3, getri, trtri, gerfs, zgemm, ztrsm, zgetrf, zlaswp, zgetrs, zgesv,
    zpotrf, zpotrs, zposv, zherk,
    CblasRowMajor, CblasColMajor, CblasNoTrans, CblasTrans, CblasConjTrans,
    CblasUpper, CblasLower, CblasNonUnit, CblasUnit, CblasLeft, CblasRight,
)
