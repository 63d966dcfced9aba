"""ctypes bindings of the oracle (oracle/liboracle.so) for the tests.

The oracle is the checker: a CPU restatement of the reference's hot path with
its exact rounding. Only the tests, the smoke check and the CPU-baseline legs
of bench.py use it.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libhwyref.so")

P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double
F = ctypes.c_float
CH = ctypes.c_char


def build_oracle():
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return ORACLE_LIB


def load_ref():
    if not os.path.exists(REF_LIB):
        return None
    lib = ctypes.CDLL(REF_LIB)
    lib.dgetrf_.argtypes = [P] * 6
    lib.dgetrf2_.argtypes = [P] * 6
    lib.dpotrf_.argtypes = [P] * 5
    lib.dpotrf2_.argtypes = [P] * 5
    lib.dgetrs_.argtypes = [P] * 9
    lib.dgesv_.argtypes = [P] * 8
    lib.sgetrf_.argtypes = [P] * 6
    lib.sgetrf2_.argtypes = [P] * 6
    lib.sgesv_.argtypes = [P] * 8
    lib.spotrf_.argtypes = [P] * 5
    lib.spotrf2_.argtypes = [P] * 5
    for pre in "zc":
        getattr(lib, f"{pre}potrf_").argtypes = [P] * 5
        getattr(lib, f"{pre}potrf2_").argtypes = [P] * 5
        getattr(lib, f"{pre}herk_").argtypes = [P] * 10
        getattr(lib, f"{pre}getrf_").argtypes = [P] * 6
        getattr(lib, f"{pre}getrf2_").argtypes = [P] * 6
        getattr(lib, f"{pre}getrs_").argtypes = [P] * 9
        getattr(lib, f"{pre}gesv_").argtypes = [P] * 8
    for pre in "ds":
        getattr(lib, f"{pre}gerfs_").argtypes = [P] * 17
        getattr(lib, f"{pre}getri_").argtypes = [P] * 7
        getattr(lib, f"{pre}trtri_").argtypes = [P] * 6
        getattr(lib, f"{pre}trti2_").argtypes = [P] * 6
    return lib


def ptr(a):
    return a.ctypes.data_as(P) if a is not None else None


def _b(s):
    return s.encode() if isinstance(s, str) else s


class Oracle:
    def __init__(self):
        self.lib = ctypes.CDLL(build_oracle())
        L = self.lib
        L.orc_set_lanes.argtypes = [I]
        L.orc_set_threads.argtypes = [I]
        L.orc_dgemm.argtypes = [CH, CH, I, I, I, D, P, I, P, I, D, P, I]
        L.orc_sgemm.argtypes = [CH, CH, I, I, I, F, P, I, P, I, F, P, I]
        L.orc_dtrsm.argtypes = [CH, CH, CH, CH, I, I, D, P, I, P, I]
        L.orc_dsyrk.argtypes = [CH, CH, I, I, D, P, I, D, P, I]
        L.orc_idamax.argtypes = [I, P, I]
        L.orc_dlaswp.argtypes = [I, P, I, I, I, P, I]
        L.orc_dgetrf.argtypes = [I, I, P, I, P]
        L.orc_dgetrf2.argtypes = [I, I, P, I, P]
        L.orc_sgetrf.argtypes = [I, I, P, I, P]
        L.orc_sgetrf2.argtypes = [I, I, P, I, P]
        L.orc_slaswp.argtypes = [I, P, I, I, I, P, I]
        L.orc_sgesv.argtypes = [I, I, P, I, P, P, I]
        L.orc_strsm.argtypes = [CH, CH, CH, CH, I, I, F, P, I, P, I]
        L.orc_dgetrs.argtypes = [CH, I, I, P, I, P, P, I]
        L.orc_sgetrs.argtypes = [CH, I, I, P, I, P, P, I]
        L.orc_dgesv.argtypes = [I, I, P, I, P, P, I]
        L.orc_dpotrf.argtypes = [CH, I, P, I]
        L.orc_dpotrf2.argtypes = [CH, I, P, I]
        L.orc_dpotrs.argtypes = [CH, I, I, P, I, P, I]
        L.orc_dposv.argtypes = [CH, I, I, P, I, P, I]
        L.orc_spotrf.argtypes = [CH, I, P, I]
        L.orc_spotrf2.argtypes = [CH, I, P, I]
        L.orc_spotrs.argtypes = [CH, I, I, P, I, P, I]
        L.orc_sposv.argtypes = [CH, I, I, P, I, P, I]
        L.orc_ssyrk.argtypes = [CH, CH, I, I, F, P, I, F, P, I]
        L.orc_zgemm.argtypes = [CH, CH, I, I, I, P, P, I, P, I, P, P, I]
        L.orc_ztrsm.argtypes = [CH, CH, CH, CH, I, I, P, P, I, P, I]
        L.orc_ctrsm.argtypes = [CH, CH, CH, CH, I, I, P, P, I, P, I]
        L.orc_zrecip.argtypes = [I, P, P]
        L.orc_crecip.argtypes = [I, P, P]
        L.orc_cgemm.argtypes = [CH, CH, I, I, I, P, P, I, P, I, P, P, I]
        L.orc_zherk.argtypes = [CH, CH, I, I, D, P, I, D, P, I]
        L.orc_cherk.argtypes = [CH, CH, I, I, F, P, I, F, P, I]
        for pre in "zc":
            getattr(L, f"orc_{pre}potrf").argtypes = [CH, I, P, I]
            getattr(L, f"orc_{pre}potrf2").argtypes = [CH, I, P, I]
            getattr(L, f"orc_{pre}potrs").argtypes = [CH, I, I, P, I, P, I]
            getattr(L, f"orc_{pre}posv").argtypes = [CH, I, I, P, I, P, I]
            getattr(L, f"orc_{pre}getrf").argtypes = [I, I, P, I, P]
            getattr(L, f"orc_{pre}getrf2").argtypes = [I, I, P, I, P]
            getattr(L, f"orc_{pre}laswp").argtypes = [I, P, I, I, I, P, I]
            getattr(L, f"orc_{pre}getrs").argtypes = [CH, I, I, P, I, P, P, I]
            getattr(L, f"orc_{pre}gesv").argtypes = [I, I, P, I, P, P, I]
        for pre in "ds":
            getattr(L, f"orc_{pre}gerfs").argtypes = [CH, I, I, P, I, P, I, P, P, I, P, I, P,
                                                       P, P, P]
            getattr(L, f"orc_{pre}getri").argtypes = [I, P, I, P, P, I]
            getattr(L, f"orc_{pre}trtri").argtypes = [CH, CH, I, P, I]
            getattr(L, f"orc_{pre}trti2").argtypes = [CH, CH, I, P, I]
        for pre, S in (("d", D), ("s", F)):
            getattr(L, f"orc_{pre}symm").argtypes = [CH, CH, I, I, S, P, I, P, I, S, P, I]
            getattr(L, f"orc_{pre}syr2k").argtypes = [CH, CH, I, I, S, P, I, P, I, S, P, I]
            getattr(L, f"orc_{pre}gemmtr").argtypes = [CH, CH, CH, I, I, S, P, I, P, I, S, P,
                                                        I]
            getattr(L, f"orc_{pre}trmm").argtypes = [CH, CH, CH, CH, I, I, S, P, I, P, I]
        L.orc_set_lanes(8)

    def set_threads(self, n):
        self.lib.orc_set_threads(int(n))

    def dgemm(self, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        return self.lib.orc_dgemm(_b(ta), _b(tb), m, n, k, alpha, ptr(a), lda, ptr(b),
                                  ldb, beta, ptr(c), ldc)

    def sgemm(self, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        return self.lib.orc_sgemm(_b(ta), _b(tb), m, n, k, alpha, ptr(a), lda, ptr(b),
                                  ldb, beta, ptr(c), ldc)

    def dtrsm(self, side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
        return self.lib.orc_dtrsm(_b(side), _b(uplo), _b(trans), _b(diag), m, n, alpha,
                                  ptr(a), lda, ptr(b), ldb)

    def dsyrk(self, uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
        return self.lib.orc_dsyrk(_b(uplo), _b(trans), n, k, alpha, ptr(a), lda, beta,
                                  ptr(c), ldc)

    def idamax(self, n, x, incx):
        return self.lib.orc_idamax(n, ptr(x), incx)

    def dlaswp(self, n, a, lda, k1, k2, ipiv, incx):
        self.lib.orc_dlaswp(n, ptr(a), lda, k1, k2, ptr(ipiv), incx)

    def dgetrf(self, m, n, a, lda, ipiv):
        return self.lib.orc_dgetrf(m, n, ptr(a), lda, ptr(ipiv))

    def dgetrf2(self, m, n, a, lda, ipiv):
        return self.lib.orc_dgetrf2(m, n, ptr(a), lda, ptr(ipiv))

    def sgetrf(self, m, n, a, lda, ipiv):
        return self.lib.orc_sgetrf(m, n, ptr(a), lda, ptr(ipiv))

    def sgetrf2(self, m, n, a, lda, ipiv):
        return self.lib.orc_sgetrf2(m, n, ptr(a), lda, ptr(ipiv))

    def slaswp(self, n, a, lda, k1, k2, ipiv, incx):
        self.lib.orc_slaswp(n, ptr(a), lda, k1, k2, ptr(ipiv), incx)

    def sgetrs(self, trans, n, nrhs, a, lda, ipiv, b, ldb):
        return self.lib.orc_sgetrs(_b(trans), n, nrhs, ptr(a), lda, ptr(ipiv), ptr(b), ldb)

    def sgesv(self, n, nrhs, a, lda, ipiv, b, ldb):
        return self.lib.orc_sgesv(n, nrhs, ptr(a), lda, ptr(ipiv), ptr(b), ldb)

    def strsm(self, side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
        return self.lib.orc_strsm(_b(side), _b(uplo), _b(trans), _b(diag), m, n, alpha,
                                  ptr(a), lda, ptr(b), ldb)

    def dgetrs(self, trans, n, nrhs, a, lda, ipiv, b, ldb):
        return self.lib.orc_dgetrs(_b(trans), n, nrhs, ptr(a), lda, ptr(ipiv), ptr(b), ldb)

    def dgesv(self, n, nrhs, a, lda, ipiv, b, ldb):
        return self.lib.orc_dgesv(n, nrhs, ptr(a), lda, ptr(ipiv), ptr(b), ldb)

    def dpotrf(self, uplo, n, a, lda):
        return self.lib.orc_dpotrf(_b(uplo), n, ptr(a), lda)

    def dpotrf2(self, uplo, n, a, lda):
        return self.lib.orc_dpotrf2(_b(uplo), n, ptr(a), lda)

    def dpotrs(self, uplo, n, nrhs, a, lda, b, ldb):
        return self.lib.orc_dpotrs(_b(uplo), n, nrhs, ptr(a), lda, ptr(b), ldb)

    def spotrf(self, uplo, n, a, lda):
        return self.lib.orc_spotrf(_b(uplo), n, ptr(a), lda)

    def spotrf2(self, uplo, n, a, lda):
        return self.lib.orc_spotrf2(_b(uplo), n, ptr(a), lda)

    def spotrs(self, uplo, n, nrhs, a, lda, b, ldb):
        return self.lib.orc_spotrs(_b(uplo), n, nrhs, ptr(a), lda, ptr(b), ldb)

    def sposv(self, uplo, n, nrhs, a, lda, b, ldb):
        return self.lib.orc_sposv(_b(uplo), n, nrhs, ptr(a), lda, ptr(b), ldb)

    def ssyrk(self, uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
        return self.lib.orc_ssyrk(_b(uplo), _b(trans), n, k, alpha, ptr(a), lda, beta,
                                  ptr(c), ldc)

    # Level 3 through the GEMM problem model; p is "d" or "s".
    def symm(self, p, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
        return getattr(self.lib, f"orc_{p}symm")(_b(side), _b(uplo), m, n, alpha, ptr(a), lda,
                                                 ptr(b), ldb, beta, ptr(c), ldc)

    def syr2k(self, p, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        return getattr(self.lib, f"orc_{p}syr2k")(_b(uplo), _b(trans), n, k, alpha, ptr(a),
                                                  lda, ptr(b), ldb, beta, ptr(c), ldc)

    def gemmtr(self, p, uplo, ta, tb, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        return getattr(self.lib, f"orc_{p}gemmtr")(_b(uplo), _b(ta), _b(tb), n, k, alpha,
                                                   ptr(a), lda, ptr(b), ldb, beta, ptr(c), ldc)

    def trmm(self, p, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
        return getattr(self.lib, f"orc_{p}trmm")(_b(side), _b(uplo), _b(transa), _b(diag), m,
                                                 n, alpha, ptr(a), lda, ptr(b), ldb)

    def gerfs(self, trans, n, nrhs, a, lda, af, ldaf, ipiv, b, ldb, x, ldx, ferr, berr,
              work, iwork):
        p = "s" if a.dtype == np.float32 else "d"
        return getattr(self.lib, f"orc_{p}gerfs")(_b(trans), n, nrhs, ptr(a), lda, ptr(af),
                                                  ldaf, ptr(ipiv), ptr(b), ldb, ptr(x), ldx,
                                                  ptr(ferr), ptr(berr), ptr(work), ptr(iwork))

    def zgemm(self, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        """Complex GEMM on complex128 / complex64 arrays (by c's dtype)."""
        z = c.dtype == np.complex128
        rt = np.float64 if z else np.float32
        al = np.array([complex(alpha).real, complex(alpha).imag], rt)
        be = np.array([complex(beta).real, complex(beta).imag], rt)
        fn = self.lib.orc_zgemm if z else self.lib.orc_cgemm
        return fn(_b(ta), _b(tb), m, n, k, al.ctypes.data, ptr(a), lda, ptr(b), ldb,
                  be.ctypes.data, ptr(c), ldc)

    def ztrsm(self, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb):
        """Complex TRSM on complex128 / complex64 arrays (by b's dtype)."""
        z = b.dtype == np.complex128
        rt = np.float64 if z else np.float32
        al = np.array([complex(alpha).real, complex(alpha).imag], rt)
        fn = self.lib.orc_ztrsm if z else self.lib.orc_ctrsm
        return fn(_b(side), _b(uplo), _b(ta), _b(diag), m, n, al.ctypes.data, ptr(a), lda,
                  ptr(b), ldb)

    # Complex LU family on complex128 / complex64 Fortran-order arrays (by dtype).
    @staticmethod
    def _zp(x):
        return "z" if x.dtype == np.complex128 else "c"

    def zgetrf(self, m, n, a, lda, ipiv, recursive=False):
        fn = getattr(self.lib, f"orc_{self._zp(a)}{'getrf2' if recursive else 'getrf'}")
        return fn(m, n, ptr(a), lda, ptr(ipiv))

    def zlaswp(self, n, a, lda, k1, k2, ipiv, incx):
        getattr(self.lib, f"orc_{self._zp(a)}laswp")(n, ptr(a), lda, k1, k2, ptr(ipiv), incx)

    def zgetrs(self, trans, n, nrhs, a, lda, ipiv, b, ldb):
        return getattr(self.lib, f"orc_{self._zp(a)}getrs")(_b(trans), n, nrhs, ptr(a), lda,
                                                          ptr(ipiv), ptr(b), ldb)

    def zgesv(self, n, nrhs, a, lda, ipiv, b, ldb):
        return getattr(self.lib, f"orc_{self._zp(a)}gesv")(n, nrhs, ptr(a), lda, ptr(ipiv),
                                                         ptr(b), ldb)

    def zpotrf(self, uplo, n, a, lda, recursive=False):
        fn = getattr(self.lib, f"orc_{self._zp(a)}{'potrf2' if recursive else 'potrf'}")
        return fn(_b(uplo), n, ptr(a), lda)

    def zpotrs(self, uplo, n, nrhs, a, lda, b, ldb):
        return getattr(self.lib, f"orc_{self._zp(a)}potrs")(_b(uplo), n, nrhs, ptr(a), lda,
                                                          ptr(b), ldb)

    def zposv(self, uplo, n, nrhs, a, lda, b, ldb):
        return getattr(self.lib, f"orc_{self._zp(a)}posv")(_b(uplo), n, nrhs, ptr(a), lda,
                                                         ptr(b), ldb)

    def zherk(self, uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
        return getattr(self.lib, f"orc_{self._zp(c)}herk")(_b(uplo), _b(trans), n, k, alpha,
                                                         ptr(a), lda, beta, ptr(c), ldc)

    def getri(self, n, a, lda, ipiv, work, lwork):
        p = "s" if a.dtype == np.float32 else "d"
        return getattr(self.lib, f"orc_{p}getri")(n, ptr(a), lda, ptr(ipiv), ptr(work), lwork)

    def trtri(self, uplo, diag, n, a, lda, unblocked=False):
        p = "s" if a.dtype == np.float32 else "d"
        fn = getattr(self.lib, f"orc_{p}{'trti2' if unblocked else 'trtri'}")
        return fn(_b(uplo), _b(diag), n, ptr(a), lda)

    def dposv(self, uplo, n, nrhs, a, lda, b, ldb):
        return self.lib.orc_dposv(_b(uplo), n, nrhs, ptr(a), lda, ptr(b), ldb)


def ref_call_getrf(lib, recursive, m, n, a, lda, ipiv):
    info = ctypes.c_int(0)
    args = [ctypes.byref(ctypes.c_int(m)), ctypes.byref(ctypes.c_int(n)), ptr(a),
            ctypes.byref(ctypes.c_int(lda)), ptr(ipiv), ctypes.byref(info)]
    if a.dtype == np.float32:
        (lib.sgetrf2_ if recursive else lib.sgetrf_)(*args)
    else:
        (lib.dgetrf2_ if recursive else lib.dgetrf_)(*args)
    return info.value


def ref_call_zgetrf(lib, recursive, m, n, a, lda, ipiv):
    """The reference driver's zgetrf_/cgetrf_ (and ...2_), by dtype."""
    info = ctypes.c_int(0)
    pre = "z" if a.dtype == np.complex128 else "c"
    fn = getattr(lib, f"{pre}{'getrf2' if recursive else 'getrf'}_")
    fn(ctypes.byref(ctypes.c_int(m)), ctypes.byref(ctypes.c_int(n)), ptr(a),
       ctypes.byref(ctypes.c_int(lda)), ptr(ipiv), ctypes.byref(info))
    return info.value


def ref_call_zpotrf(lib, recursive, uplo, n, a, lda):
    """The reference driver's zpotrf_/cpotrf_ (and ...2_), by dtype."""
    info = ctypes.c_int(0)
    pre = "z" if a.dtype == np.complex128 else "c"
    fn = getattr(lib, f"{pre}{'potrf2' if recursive else 'potrf'}_")
    fn(ctypes.c_char_p(_b(uplo)), ctypes.byref(ctypes.c_int(n)), ptr(a),
       ctypes.byref(ctypes.c_int(lda)), ctypes.byref(info))
    return info.value


def ref_call_zgetrs(lib, trans, n, nrhs, a, lda, ipiv, b, ldb):
    info = ctypes.c_int(0)
    pre = "z" if a.dtype == np.complex128 else "c"
    I = lambda v: ctypes.byref(ctypes.c_int(v))  # noqa: E731
    getattr(lib, f"{pre}getrs_")(ctypes.c_char_p(_b(trans)), I(n), I(nrhs), ptr(a), I(lda),
                                 ptr(ipiv), ptr(b), I(ldb), ctypes.byref(info))
    return info.value


def ref_call_gesv(lib, n, nrhs, a, lda, ipiv, b, ldb):
    """The reference driver's ?gesv_ (src/lapack/getrf.cc:531), by dtype."""
    info = ctypes.c_int(0)
    fn = lib.sgesv_ if a.dtype == np.float32 else lib.dgesv_
    fn(ctypes.byref(ctypes.c_int(n)), ctypes.byref(ctypes.c_int(nrhs)), ptr(a),
       ctypes.byref(ctypes.c_int(lda)), ptr(ipiv), ptr(b), ctypes.byref(ctypes.c_int(ldb)),
       ctypes.byref(info))
    return info.value


def ref_call_potrf(lib, recursive, uplo, n, a, lda):
    info = ctypes.c_int(0)
    args = [ctypes.c_char_p(_b(uplo)), ctypes.byref(ctypes.c_int(n)), ptr(a),
            ctypes.byref(ctypes.c_int(lda)), ctypes.byref(info)]
    if a.dtype == np.float32:
        (lib.spotrf2_ if recursive else lib.spotrf_)(*args)
    else:
        (lib.dpotrf2_ if recursive else lib.dpotrf_)(*args)
    return info.value


def ref_call_getri(lib, n, a, lda, ipiv, work, lwork):
    """The reference driver's ?getri_ (src/lapack/getrf.cc:538-544), by dtype."""
    info = ctypes.c_int(0)
    fn = lib.sgetri_ if a.dtype == np.float32 else lib.dgetri_
    fn(ctypes.byref(ctypes.c_int(n)), ptr(a), ctypes.byref(ctypes.c_int(lda)), ptr(ipiv),
       ptr(work), ctypes.byref(ctypes.c_int(lwork)), ctypes.byref(info))
    return info.value


def ref_call_gerfs(lib, trans, n, nrhs, a, lda, af, ldaf, ipiv, b, ldb, x, ldx, ferr, berr,
                   work, iwork):
    """The reference's ?gerfs_ (src/lapack/gesvx.cc:796-806), by dtype."""
    info = ctypes.c_int(0)
    fn = lib.sgerfs_ if a.dtype == np.float32 else lib.dgerfs_
    I = lambda v: ctypes.byref(ctypes.c_int(v))  # noqa: E731
    fn(ctypes.c_char_p(_b(trans)), I(n), I(nrhs), ptr(a), I(lda), ptr(af), I(ldaf), ptr(ipiv),
       ptr(b), I(ldb), ptr(x), I(ldx), ptr(ferr), ptr(berr), ptr(work), ptr(iwork),
       ctypes.byref(info))
    return info.value


def ref_call_trtri(lib, unblocked, uplo, diag, n, a, lda):
    """The reference's ?trtri_ / ?trti2_ (src/lapack/triangular.cc:1645-1659)."""
    info = ctypes.c_int(0)
    pre = "s" if a.dtype == np.float32 else "d"
    fn = getattr(lib, f"{pre}{'trti2' if unblocked else 'trtri'}_")
    fn(ctypes.c_char_p(_b(uplo)), ctypes.c_char_p(_b(diag)), ctypes.byref(ctypes.c_int(n)),
       ptr(a), ctypes.byref(ctypes.c_int(lda)), ctypes.byref(info))
    return info.value


def crand(rng, rows, cols, dtype=np.complex128):
    """Column-major complex matrix with parts uniform in [-1, 1]."""
    x = rng.uniform(-1.0, 1.0, (rows, cols)) + 1j * rng.uniform(-1.0, 1.0, (rows, cols))
    return np.asfortranarray(x.astype(dtype))


def hpd(rng, n, dtype=np.complex128):
    """A Hermitian positive definite matrix G G^H / n + 1e-3 I (Fortran order)."""
    g = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return np.asfortranarray((g @ g.conj().T / n + 1e-3 * np.eye(n)).astype(dtype))


def rand(rng, rows, cols, dtype=np.float64):
    """Column-major uniform[-1, 1] matrix (the reference tests' Random<T>)."""
    return np.asfortranarray(rng.uniform(-1.0, 1.0, (rows, cols)).astype(dtype))


def creal(x):
    """The interleaved real view of a complex array (any order)."""
    x = np.ascontiguousarray(np.asarray(x).T)
    return x.view(np.float64 if x.dtype == np.complex128 else np.float32)


def same_bits(x, y):
    """Bitwise equality, treating any two NaNs as equal."""
    x = np.asarray(x)
    y = np.asarray(y)
    if x.shape != y.shape:
        return False
    nx, ny = np.isnan(x), np.isnan(y)
    if not np.array_equal(nx, ny):
        return False
    ix = x.view(np.uint64 if x.dtype == np.float64 else np.uint32)
    iy = y.view(np.uint64 if y.dtype == np.float64 else np.uint32)
    return bool(np.all((ix == iy) | nx))


def first_diff(x, y):
    x = np.asarray(x).ravel(order="F")
    y = np.asarray(y).ravel(order="F")
    bad = ~((x == y) | (np.isnan(x) & np.isnan(y)))
    idx = np.flatnonzero(bad)
    if idx.size == 0:
        return None
    i = idx[0]
    return f"{idx.size} differ; first at flat {i}: {x[i]!r} vs {y[i]!r}"


# ---------------------------------------------------------------------------
# The reference library itself (oracle/_ref/libhwyblas_ref.so): every source
# of the reference compiled unmodified against the Highway-API shim. Built
# only where the reference's sources were present.

REFBLAS_LIB = os.path.join(ORACLE_DIR, "_ref", "libhwyblas_ref.so")


class RefBlas:
    """The reference's own Fortran-convention entry points (all arguments by
    pointer), with the Oracle class's calling style for the tests."""

    def __init__(self):
        self.lib = ctypes.CDLL(REFBLAS_LIB)

    @staticmethod
    def _i(v):
        return ctypes.byref(ctypes.c_int(int(v)))

    @staticmethod
    def _d(v, single=False):
        return ctypes.byref(ctypes.c_float(v) if single else ctypes.c_double(v))

    def _info_call(self, fn, *args):
        info = ctypes.c_int(0)
        fn(*args, ctypes.byref(info))
        return info.value

    def dgemm(self, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, single=False):
        fn = self.lib.sgemm_ if single else self.lib.dgemm_
        i, d = self._i, self._d
        fn(_b(ta), _b(tb), i(m), i(n), i(k), d(alpha, single), ptr(a), i(lda), ptr(b), i(ldb),
           d(beta, single), ptr(c), i(ldc))

    def dtrsm(self, side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
        i, d = self._i, self._d
        self.lib.dtrsm_(_b(side), _b(uplo), _b(trans), _b(diag), i(m), i(n), d(alpha),
                        ptr(a), i(lda), ptr(b), i(ldb))

    def dsyrk(self, uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
        i, d = self._i, self._d
        self.lib.dsyrk_(_b(uplo), _b(trans), i(n), i(k), d(alpha), ptr(a), i(lda), d(beta),
                        ptr(c), i(ldc))

    def dtrmm(self, side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
        i, d = self._i, self._d
        self.lib.dtrmm_(_b(side), _b(uplo), _b(trans), _b(diag), i(m), i(n), d(alpha),
                        ptr(a), i(lda), ptr(b), i(ldb))

    def idamax(self, n, x, incx):
        self.lib.idamax_.restype = ctypes.c_int
        return self.lib.idamax_(self._i(n), ptr(x), self._i(incx))

    def dgetrf(self, m, n, a, lda, ipiv):
        i = self._i
        return self._info_call(self.lib.dgetrf_, i(m), i(n), ptr(a), i(lda), ptr(ipiv))

    def dgetrs(self, trans, n, nrhs, a, lda, ipiv, b, ldb):
        i = self._i
        return self._info_call(self.lib.dgetrs_, _b(trans), i(n), i(nrhs), ptr(a), i(lda),
                               ptr(ipiv), ptr(b), i(ldb))

    def dpotrf(self, uplo, n, a, lda):
        i = self._i
        return self._info_call(self.lib.dpotrf_, _b(uplo), i(n), ptr(a), i(lda))

    def dpotrs(self, uplo, n, nrhs, a, lda, b, ldb):
        i = self._i
        return self._info_call(self.lib.dpotrs_, _b(uplo), i(n), i(nrhs), ptr(a), i(lda),
                               ptr(b), i(ldb))


def load_refblas():
    return RefBlas() if os.path.exists(REFBLAS_LIB) else None
