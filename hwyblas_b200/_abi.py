"""ctypes prototypes of the C ABI in include/hwyblas_b200.h.

EXPORTED lists every symbol the header declares; the CPU test suite checks
that the built library exports exactly these.
"""
import ctypes

P = ctypes.c_void_p
I = ctypes.c_int
PI = ctypes.POINTER(ctypes.c_int)
D = ctypes.c_double
F = ctypes.c_float
C = ctypes.c_char_p

# name -> (restype, argtypes)
PROTOTYPES = {
    # Fortran BLAS (all arguments by pointer)
    "dgemm_": (None, [C, C, PI, PI, PI, P, P, PI, P, PI, P, P, PI]),
    "sgemm_": (None, [C, C, PI, PI, PI, P, P, PI, P, PI, P, P, PI]),
    "dtrsm_": (None, [C, C, C, C, PI, PI, P, P, PI, P, PI]),
    "strsm_": (None, [C, C, C, C, PI, PI, P, P, PI, P, PI]),
    "dsyrk_": (None, [C, C, PI, PI, P, P, PI, P, P, PI]),
    **{f"{p}gemm_": (None, [C, C, PI, PI, PI, P, P, PI, P, PI, P, P, PI]) for p in "zc"},
    **{f"{p}trsm_": (None, [C, C, C, C, PI, PI, P, P, PI, P, PI]) for p in "zc"},
    **{f"{p}getrf_": (None, [PI, PI, P, PI, P, PI]) for p in "zc"},
    **{f"{p}getrf2_": (None, [PI, PI, P, PI, P, PI]) for p in "zc"},
    **{f"{p}laswp_": (None, [PI, P, PI, PI, PI, P, PI]) for p in "zc"},
    **{f"{p}getrs_": (None, [C, PI, PI, P, PI, P, P, PI, PI]) for p in "zc"},
    **{f"{p}gesv_": (None, [PI, PI, P, PI, P, P, PI, PI]) for p in "zc"},
    **{f"{p}potrf_": (None, [C, PI, P, PI, PI]) for p in "zc"},
    **{f"{p}potrf2_": (None, [C, PI, P, PI, PI]) for p in "zc"},
    **{f"{p}potrs_": (None, [C, PI, PI, P, PI, P, PI, PI]) for p in "zc"},
    **{f"{p}posv_": (None, [C, PI, PI, P, PI, P, PI, PI]) for p in "zc"},
    **{f"{p}herk_": (None, [C, C, PI, PI, P, P, PI, P, P, PI]) for p in "zc"},
    "cblas_zherk": (None, [I, I, I, I, I, ctypes.c_double, P, I, ctypes.c_double, P, I]),
    "cblas_cherk": (None, [I, I, I, I, I, ctypes.c_float, P, I, ctypes.c_float, P, I]),
    **{f"{p}symm_": (None, [C, C, PI, PI, P, P, PI, P, PI, P, P, PI]) for p in "ds"},
    **{f"{p}syr2k_": (None, [C, C, PI, PI, P, P, PI, P, PI, P, P, PI]) for p in "ds"},
    **{f"{p}{r}_": (None, [C, C, C, PI, PI, P, P, PI, P, PI, P, P, PI])
       for p in "ds" for r in ("gemmtr", "gemmt")},
    **{f"{p}trmm_": (None, [C, C, C, C, PI, PI, P, P, PI, P, PI]) for p in "ds"},
    **{f"{p}getri_": (None, [PI, P, PI, P, P, PI, PI]) for p in "ds"},
    **{f"{p}gerfs_": (None, [C, PI, PI, P, PI, P, PI, P, P, PI, P, PI, P, P, P, P, PI])
       for p in "ds"},
    **{f"{p}{r}_": (None, [C, C, PI, P, PI, PI]) for p in "ds" for r in ("trtri", "trti2")},
    "ssyrk_": (None, [C, C, PI, PI, P, P, PI, P, P, PI]),
    "idamax_": (I, [PI, P, PI]),
    "xerbla_": (None, [C, PI, ctypes.c_size_t]),
    "hwyblas_set_error_handler": (P, [P]),
    # LAPACK
    "dgetrf_": (None, [PI, PI, P, PI, P, PI]),
    "dgetrf2_": (None, [PI, PI, P, PI, P, PI]),
    "dlaswp_": (None, [PI, P, PI, PI, PI, P, PI]),
    "dgetrs_": (None, [C, PI, PI, P, PI, P, P, PI, PI]),
    "dgesv_": (None, [PI, PI, P, PI, P, P, PI, PI]),
    "sgetrf_": (None, [PI, PI, P, PI, P, PI]),
    "sgetrf2_": (None, [PI, PI, P, PI, P, PI]),
    "slaswp_": (None, [PI, P, PI, PI, PI, P, PI]),
    "sgetrs_": (None, [C, PI, PI, P, PI, P, P, PI, PI]),
    "sgesv_": (None, [PI, PI, P, PI, P, P, PI, PI]),
    "dpotrf_": (None, [C, PI, P, PI, PI]),
    "dpotrf2_": (None, [C, PI, P, PI, PI]),
    "dpotrs_": (None, [C, PI, PI, P, PI, P, PI, PI]),
    "dposv_": (None, [C, PI, PI, P, PI, P, PI, PI]),
    "spotrf_": (None, [C, PI, P, PI, PI]),
    "spotrf2_": (None, [C, PI, P, PI, PI]),
    "spotrs_": (None, [C, PI, PI, P, PI, P, PI, PI]),
    "sposv_": (None, [C, PI, PI, P, PI, P, PI, PI]),
    # LAPACKE (by value; char arguments as one byte)
    "LAPACKE_xerbla": (None, [C, I]),
    "LAPACKE_set_nancheck": (None, [I]),
    "LAPACKE_get_nancheck": (I, []),
    **{f"LAPACKE_{p}getrf{s}": (I, [I, I, I, P, I, P])
       for p in "ds" for s in ("", "_work")},
    **{f"LAPACKE_{p}getrf2{s}": (I, [I, I, I, P, I, P])
       for p in "ds" for s in ("", "_work")},
    **{f"LAPACKE_{p}getrs{s}": (I, [I, ctypes.c_char, I, I, P, I, P, P, I])
       for p in "ds" for s in ("", "_work")},
    **{f"LAPACKE_{p}gesv{s}": (I, [I, I, I, P, I, P, P, I])
       for p in "ds" for s in ("", "_work")},
    **{f"LAPACKE_{p}potrf{s}": (I, [I, ctypes.c_char, I, P, I])
       for p in "ds" for s in ("", "_work")},
    **{f"LAPACKE_{p}potrf2{s}": (I, [I, ctypes.c_char, I, P, I])
       for p in "ds" for s in ("", "_work")},
    **{f"LAPACKE_{p}potrs{s}": (I, [I, ctypes.c_char, I, I, P, I, P, I])
       for p in "ds" for s in ("", "_work")},
    **{f"LAPACKE_{p}posv{s}": (I, [I, ctypes.c_char, I, I, P, I, P, I])
       for p in "ds" for s in ("", "_work")},
    **{f"LAPACKE_{p}getri": (I, [I, I, P, I, P]) for p in "ds"},
    **{f"LAPACKE_{p}getri_work": (I, [I, I, P, I, P, P, I]) for p in "ds"},
    **{f"LAPACKE_{p}trtri{s}": (I, [I, ctypes.c_char, ctypes.c_char, I, P, I])
       for p in "ds" for s in ("", "_work")},
    # CBLAS (by value)
    "cblas_xerbla": (None, [I, C, C]),
    "cblas_dgemm": (None, [I, I, I, I, I, I, D, P, I, P, I, D, P, I]),
    "cblas_sgemm": (None, [I, I, I, I, I, I, F, P, I, P, I, F, P, I]),
    "cblas_dtrsm": (None, [I, I, I, I, I, I, I, D, P, I, P, I]),
    "cblas_strsm": (None, [I, I, I, I, I, I, I, F, P, I, P, I]),
    "cblas_idamax": (ctypes.c_size_t, [I, P, I]),
    **{f"cblas_{p}gemm": (None, [I, I, I, I, I, I, P, P, I, P, I, P, P, I]) for p in "zc"},
    **{f"cblas_{p}trsm": (None, [I, I, I, I, I, I, I, P, P, I, P, I]) for p in "zc"},
    **{f"cblas_{p}trmm": (None, [I, I, I, I, I, I, I, S, P, I, P, I])
       for p, S in (("d", D), ("s", F))},
    **{f"cblas_{p}symm": (None, [I, I, I, I, I, S, P, I, P, I, S, P, I])
       for p, S in (("d", D), ("s", F))},
    **{f"cblas_{p}syr2k": (None, [I, I, I, I, I, S, P, I, P, I, S, P, I])
       for p, S in (("d", D), ("s", F))},
    **{f"cblas_{p}{r}": (None, [I, I, I, I, I, I, S, P, I, P, I, S, P, I])
       for p, S in (("d", D), ("s", F)) for r in ("gemmtr", "gemmt")},
    # Extensions
    "hwyblas_dgemm_emulated": (I, [C, C, PI, PI, PI, P, P, PI, P, PI, P, P, PI, PI]),
    "hwyblas_dgemm_ddref": (None, [C, C, PI, PI, PI, P, PI, P, PI, PI, P, P, PI]),
    "hwyblas_dgesv_mixed": (None, [PI, PI, P, PI, P, P, PI, P, PI, PI, PI]),
    "hwyblas_dposv_mixed": (None, [C, PI, PI, P, PI, P, PI, P, PI, PI, PI]),
    "hwyblas_set_mixed_slices": (I, [I]),
    "hwyblas_dgetrf_batched": (None, [P, P, P, P, P, I]),
    "hwyblas_sgetrf_batched": (None, [P, P, P, P, P, I]),
    "hwyblas_dgetrs_batched": (None, [ctypes.c_char, P, P, P, P, P, P, P, I, PI]),
    "hwyblas_sgetrs_batched": (None, [ctypes.c_char, P, P, P, P, P, P, P, I, PI]),
    "hwyblas_dtrsm_batched": (None, [ctypes.c_char] * 4 + [P, P, D, P, P, P, P, I]),
    "hwyblas_strsm_batched": (None, [ctypes.c_char] * 4 + [P, P, F, P, P, P, P, I]),
    "hwyblas_dgemm_batched": (None, [ctypes.c_char, ctypes.c_char, P, P, P, D, P, P, P, P,
                                     D, P, P, I]),
    "hwyblas_sgemm_batched": (None, [ctypes.c_char, ctypes.c_char, P, P, P, F, P, P, P, P,
                                     F, P, P, I]),
    "hwyblas_set_stream": (None, [P]),
    "hwyblas_last_cuda_error": (I, []),
    "hwyblas_set_leaf_wait_limit": (ctypes.c_uint, [ctypes.c_uint]),
    "hwyblas_int8_peak_tops": (D, []),
    "hwyblas_dresidual_dd": (None, [PI, PI, P, PI, P, PI, P, PI, P, PI]),
    "hwyblas_batched_set_config": (I, [I]),
    "hwyblas_launch_count": (ctypes.c_uint64, []),
    "hwyblas_kernel_timer": (None, [I]),
    "hwyblas_kernel_timer_read": (D, [PI]),
    "hwyblas_fp64_peak_tflops": (ctypes.c_double, []),
    "hwyblas_idamax_noalloc": (I, [I, P, I, P, P]),
}

EXPORTED = sorted(PROTOTYPES)


def declare(lib):
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
