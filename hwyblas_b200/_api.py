"""Python wrappers with the reference's routine names and argument order.

Each wrapper takes the Fortran arguments by value (characters as str, sizes
as int, scalars as float) and buffers as NumPy arrays (host memory, copied to
the GPU and back by the library) or CUDA tensors (device memory, used in
place), and calls the C ABI. Matrices are column-major: pass
``np.asfortranarray`` data or any buffer with the right leading dimension.
LAPACK wrappers return INFO.
"""
import ctypes
import numbers

from . import lib

CblasRowMajor, CblasColMajor = 101, 102
CblasNoTrans, CblasTrans, CblasConjTrans = 111, 112, 113
CblasUpper, CblasLower = 121, 122
CblasNonUnit, CblasUnit = 131, 132
CblasLeft, CblasRight = 141, 142


def _ptr(x):
    """Address of a NumPy array / torch tensor / integer address."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(f"unsupported buffer {type(x)}")


def _i(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _d(v):
    return ctypes.byref(ctypes.c_double(float(v)))


def _f(v):
    return ctypes.byref(ctypes.c_float(float(v)))


def _c(s):
    return s.encode() if isinstance(s, str) else s


def dgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """C := alpha*op(A)*op(B) + beta*C (reference dgemm_, src/gemm.cc:151)."""
    lib().dgemm_(_c(transa), _c(transb), _i(m), _i(n), _i(k), _d(alpha), _ptr(a),
                 _i(lda), _ptr(b), _i(ldb), _d(beta), _ptr(c), _i(ldc))


def sgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """FP32 GEMM (reference sgemm_, src/gemm.cc:142)."""
    lib().sgemm_(_c(transa), _c(transb), _i(m), _i(n), _i(k), _f(alpha), _ptr(a),
                 _i(lda), _ptr(b), _i(ldb), _f(beta), _ptr(c), _i(ldc))


def dtrsm(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """Triangular solve in place (reference dtrsm_, src/trsm.cc:196)."""
    lib().dtrsm_(_c(side), _c(uplo), _c(transa), _c(diag), _i(m), _i(n),
                 _d(alpha), _ptr(a), _i(lda), _ptr(b), _i(ldb))


def strsm(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """FP32 triangular solve in place (reference strsm_, src/trsm.cc:190)."""
    lib().strsm_(_c(side), _c(uplo), _c(transa), _c(diag), _i(m), _i(n),
                 _f(alpha), _ptr(a), _i(lda), _ptr(b), _i(ldb))


def dsyrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """Symmetric rank-k update (reference dsyrk_, src/level3.cc:416)."""
    lib().dsyrk_(_c(uplo), _c(trans), _i(n), _i(k), _d(alpha), _ptr(a), _i(lda),
                 _d(beta), _ptr(c), _i(ldc))


def ssyrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """FP32 symmetric rank-k update (reference ssyrk_, src/level3.cc:410)."""
    lib().ssyrk_(_c(uplo), _c(trans), _i(n), _i(k), _f(alpha), _ptr(a), _i(lda),
                 _f(beta), _ptr(c), _i(ldc))


def _scal(p):
    return _d if p == "d" else _f


def symm(p, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
    """Symmetric matrix product; p is "d" or "s" (reference dsymm_/ssymm_,
    src/level3.cc:362-375)."""
    sc = _scal(p)
    getattr(lib(), f"{p}symm_")(_c(side), _c(uplo), _i(m), _i(n), sc(alpha), _ptr(a),
                                _i(lda), _ptr(b), _i(ldb), sc(beta), _ptr(c), _i(ldc))


def syr2k(p, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """Symmetric rank-2k update (reference dsyr2k_/ssyr2k_, src/level3.cc:456-469)."""
    sc = _scal(p)
    getattr(lib(), f"{p}syr2k_")(_c(uplo), _c(trans), _i(n), _i(k), sc(alpha), _ptr(a),
                                 _i(lda), _ptr(b), _i(ldb), sc(beta), _ptr(c), _i(ldc))


def gemmtr(p, uplo, transa, transb, n, k, alpha, a, lda, b, ldb, beta, c, ldc, name="gemmtr"):
    """GEMM on one triangle of C (reference ?gemmtr_ and the alias ?gemmt_,
    src/level3.cc:508-575)."""
    sc = _scal(p)
    getattr(lib(), f"{p}{name}_")(_c(uplo), _c(transa), _c(transb), _i(n), _i(k), sc(alpha),
                                  _ptr(a), _i(lda), _ptr(b), _i(ldb), sc(beta), _ptr(c),
                                  _i(ldc))


def trmm(p, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """Triangular matrix product in place (reference dtrmm_/strmm_,
    src/level3.cc:581-592)."""
    getattr(lib(), f"{p}trmm_")(_c(side), _c(uplo), _c(transa), _c(diag), _i(m), _i(n),
                                _scal(p)(alpha), _ptr(a), _i(lda), _ptr(b), _i(ldb))


def getri(p, n, a, lda, ipiv, work, lwork):
    """Inverse from the LU factors; returns INFO (reference ?getri_,
    src/lapack/getrf.cc:538-544). work may be a 1-element array for a
    query (lwork = -1)."""
    info = ctypes.c_int(0)
    getattr(lib(), f"{p}getri_")(_i(n), _ptr(a), _i(lda), _ptr(ipiv), _ptr(work), _i(lwork),
                                 ctypes.byref(info))
    return info.value


def gerfs(p, trans, n, nrhs, a, lda, af, ldaf, ipiv, b, ldb, x, ldx, ferr, berr, work,
          iwork):
    """Iterative refinement with error bounds; returns INFO (reference
    ?gerfs_, src/lapack/gesvx.cc:796-806)."""
    info = ctypes.c_int(0)
    getattr(lib(), f"{p}gerfs_")(_c(trans), _i(n), _i(nrhs), _ptr(a), _i(lda), _ptr(af),
                                 _i(ldaf), _ptr(ipiv), _ptr(b), _i(ldb), _ptr(x), _i(ldx),
                                 _ptr(ferr), _ptr(berr), _ptr(work), _ptr(iwork),
                                 ctypes.byref(info))
    return info.value


def trtri(p, uplo, diag, n, a, lda, unblocked=False):
    """Triangular inverse in place; returns INFO (reference ?trtri_ / ?trti2_,
    src/lapack/triangular.cc:1645-1659)."""
    info = ctypes.c_int(0)
    name = "trti2" if unblocked else "trtri"
    getattr(lib(), f"{p}{name}_")(_c(uplo), _c(diag), _i(n), _ptr(a), _i(lda),
                                  ctypes.byref(info))
    return info.value


def zgemm(p, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """Complex GEMM; p is "z" or "c", arrays complex128 / complex64, alpha and
    beta Python complex (reference zgemm_/cgemm_, src/gemm.cc:160-177)."""
    import numpy as np
    rt = np.float64 if p == "z" else np.float32
    al = np.array([complex(alpha).real, complex(alpha).imag], rt)
    be = np.array([complex(beta).real, complex(beta).imag], rt)
    getattr(lib(), f"{p}gemm_")(_c(transa), _c(transb), _i(m), _i(n), _i(k), al.ctypes.data,
                                _ptr(a), _i(lda), _ptr(b), _i(ldb), be.ctypes.data, _ptr(c),
                                _i(ldc))


def ztrsm(p, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """Complex triangular solve in place; p is "z" or "c" (reference
    ztrsm_/ctrsm_, src/trsm.cc:202-215)."""
    import numpy as np
    rt = np.float64 if p == "z" else np.float32
    al = np.array([complex(alpha).real, complex(alpha).imag], rt)
    getattr(lib(), f"{p}trsm_")(_c(side), _c(uplo), _c(transa), _c(diag), _i(m), _i(n),
                                al.ctypes.data, _ptr(a), _i(lda), _ptr(b), _i(ldb))


def zgetrf(p, m, n, a, lda, ipiv, recursive=False):
    """Complex LU with partial pivoting; p is "z" or "c"; returns INFO
    (reference zgetrf_/cgetrf_ and ...2_, src/lapack/getrf.cc:508-517)."""
    fn = getattr(lib(), f"{p}{'getrf2' if recursive else 'getrf'}_")
    return _info_call(fn, _i(m), _i(n), _ptr(a), _i(lda), _ptr(ipiv))


def zlaswp(p, n, a, lda, k1, k2, ipiv, incx):
    """Complex row interchanges (reference zlaswp_/claswp_, src/lapack/getrf.cc:518)."""
    getattr(lib(), f"{p}laswp_")(_i(n), _ptr(a), _i(lda), _i(k1), _i(k2), _ptr(ipiv), _i(incx))


def zgetrs(p, trans, n, nrhs, a, lda, ipiv, b, ldb):
    """Complex solve with LU factors, trans N/T/C; returns INFO (src/lapack/getrf.cc:524)."""
    return _info_call(getattr(lib(), f"{p}getrs_"), _c(trans), _i(n), _i(nrhs), _ptr(a),
                      _i(lda), _ptr(ipiv), _ptr(b), _i(ldb))


def zgesv(p, n, nrhs, a, lda, ipiv, b, ldb):
    """Complex LU solve of A X = B; returns INFO (src/lapack/getrf.cc:531)."""
    return _info_call(getattr(lib(), f"{p}gesv_"), _i(n), _i(nrhs), _ptr(a), _i(lda),
                      _ptr(ipiv), _ptr(b), _i(ldb))


def zpotrf(p, uplo, n, a, lda, recursive=False):
    """Complex Cholesky; returns INFO (reference zpotrf_/cpotrf_ and ...2_)."""
    fn = getattr(lib(), f"{p}{'potrf2' if recursive else 'potrf'}_")
    return _info_call(fn, _c(uplo), _i(n), _ptr(a), _i(lda))


def zpotrs(p, uplo, n, nrhs, a, lda, b, ldb):
    """Complex solve with Cholesky factors; returns INFO (src/lapack/posv.cc:31)."""
    return _info_call(getattr(lib(), f"{p}potrs_"), _c(uplo), _i(n), _i(nrhs), _ptr(a),
                      _i(lda), _ptr(b), _i(ldb))


def zposv(p, uplo, n, nrhs, a, lda, b, ldb):
    """Complex Cholesky solve of A X = B; returns INFO (src/lapack/posv.cc:85)."""
    return _info_call(getattr(lib(), f"{p}posv_"), _c(uplo), _i(n), _i(nrhs), _ptr(a),
                      _i(lda), _ptr(b), _i(ldb))


def zherk(p, uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """Complex Hermitian rank-k update, alpha and beta real (reference
    zherk_/cherk_, src/level3.cc:439-452)."""
    sc = _d if p == "z" else _f
    getattr(lib(), f"{p}herk_")(_c(uplo), _c(trans), _i(n), _i(k), sc(alpha), _ptr(a),
                                _i(lda), sc(beta), _ptr(c), _i(ldc))


def cblas_level3(name, *args):
    """Calls cblas_<name> (d/s symm, syr2k, gemmtr, gemmt, trmm) with by-value
    scalars, array arguments given as numpy arrays or device pointers."""
    conv = []
    for x in args:
        if isinstance(x, numbers.Integral):
            conv.append(int(x))
        elif isinstance(x, numbers.Real):
            conv.append(float(x))
        else:
            conv.append(_ptr(x))
    getattr(lib(), f"cblas_{name}")(*conv)


def idamax(n, x, incx):
    """1-based index of the first largest |x| (reference idamax_)."""
    return lib().idamax_(_i(n), _ptr(x), _i(incx))


def dlaswp(n, a, lda, k1, k2, ipiv, incx):
    """Row interchanges (reference dlaswp_, src/lapack/getrf.cc:28)."""
    lib().dlaswp_(_i(n), _ptr(a), _i(lda), _i(k1), _i(k2), _ptr(ipiv), _i(incx))


def _info_call(fn, *args):
    info = ctypes.c_int(0)
    fn(*args, ctypes.byref(info))
    return info.value


def dgetrf(m, n, a, lda, ipiv):
    """Blocked LU with partial pivoting; returns INFO (src/lapack/getrf.cc:216)."""
    return _info_call(lib().dgetrf_, _i(m), _i(n), _ptr(a), _i(lda), _ptr(ipiv))


def dgetrf2(m, n, a, lda, ipiv):
    """Recursive LU; returns INFO (src/lapack/getrf.cc:112)."""
    return _info_call(lib().dgetrf2_, _i(m), _i(n), _ptr(a), _i(lda), _ptr(ipiv))


def dgetrs(trans, n, nrhs, a, lda, ipiv, b, ldb):
    """Solve with LU factors; returns INFO (src/lapack/getrf.cc:287)."""
    return _info_call(lib().dgetrs_, _c(trans), _i(n), _i(nrhs), _ptr(a), _i(lda),
                      _ptr(ipiv), _ptr(b), _i(ldb))


def dgesv(n, nrhs, a, lda, ipiv, b, ldb):
    """LU solve of A X = B; returns INFO (src/lapack/getrf.cc:348)."""
    return _info_call(lib().dgesv_, _i(n), _i(nrhs), _ptr(a), _i(lda), _ptr(ipiv),
                      _ptr(b), _i(ldb))


def slaswp(n, a, lda, k1, k2, ipiv, incx):
    """FP32 row interchanges (reference slaswp_, src/lapack/getrf.cc:518)."""
    lib().slaswp_(_i(n), _ptr(a), _i(lda), _i(k1), _i(k2), _ptr(ipiv), _i(incx))


def sgetrf(m, n, a, lda, ipiv):
    """FP32 blocked LU; returns INFO (reference sgetrf_, src/lapack/getrf.cc:508)."""
    return _info_call(lib().sgetrf_, _i(m), _i(n), _ptr(a), _i(lda), _ptr(ipiv))


def sgetrf2(m, n, a, lda, ipiv):
    """FP32 recursive LU; returns INFO (reference sgetrf2_, src/lapack/getrf.cc:513)."""
    return _info_call(lib().sgetrf2_, _i(m), _i(n), _ptr(a), _i(lda), _ptr(ipiv))


def sgetrs(trans, n, nrhs, a, lda, ipiv, b, ldb):
    """FP32 solve with LU factors; returns INFO (src/lapack/getrf.cc:524)."""
    return _info_call(lib().sgetrs_, _c(trans), _i(n), _i(nrhs), _ptr(a), _i(lda),
                      _ptr(ipiv), _ptr(b), _i(ldb))


def sgesv(n, nrhs, a, lda, ipiv, b, ldb):
    """FP32 LU solve of A X = B; returns INFO (src/lapack/getrf.cc:531)."""
    return _info_call(lib().sgesv_, _i(n), _i(nrhs), _ptr(a), _i(lda), _ptr(ipiv),
                      _ptr(b), _i(ldb))


def dpotrf(uplo, n, a, lda):
    """Blocked Cholesky; returns INFO (src/lapack/potrf.cc:128)."""
    return _info_call(lib().dpotrf_, _c(uplo), _i(n), _ptr(a), _i(lda))


def dpotrf2(uplo, n, a, lda):
    """Recursive Cholesky; returns INFO (src/lapack/potrf.cc:48)."""
    return _info_call(lib().dpotrf2_, _c(uplo), _i(n), _ptr(a), _i(lda))


def dpotrs(uplo, n, nrhs, a, lda, b, ldb):
    """Solve with the Cholesky factor; returns INFO (src/lapack/posv.cc:31)."""
    return _info_call(lib().dpotrs_, _c(uplo), _i(n), _i(nrhs), _ptr(a), _i(lda),
                      _ptr(b), _i(ldb))


def dposv(uplo, n, nrhs, a, lda, b, ldb):
    """Cholesky solve of A X = B; returns INFO (src/lapack/posv.cc:78)."""
    return _info_call(lib().dposv_, _c(uplo), _i(n), _i(nrhs), _ptr(a), _i(lda),
                      _ptr(b), _i(ldb))


def spotrf(uplo, n, a, lda):
    """FP32 blocked Cholesky; returns INFO (reference spotrf_, src/lapack/potrf.cc:748)."""
    return _info_call(lib().spotrf_, _c(uplo), _i(n), _ptr(a), _i(lda))


def spotrf2(uplo, n, a, lda):
    """FP32 recursive Cholesky; returns INFO (src/lapack/potrf.cc:753)."""
    return _info_call(lib().spotrf2_, _c(uplo), _i(n), _ptr(a), _i(lda))


def spotrs(uplo, n, nrhs, a, lda, b, ldb):
    """FP32 solve with the Cholesky factor; returns INFO (src/lapack/posv.cc)."""
    return _info_call(lib().spotrs_, _c(uplo), _i(n), _i(nrhs), _ptr(a), _i(lda),
                      _ptr(b), _i(ldb))


def sposv(uplo, n, nrhs, a, lda, b, ldb):
    """FP32 Cholesky solve of A X = B; returns INFO (src/lapack/posv.cc)."""
    return _info_call(lib().sposv_, _c(uplo), _i(n), _i(nrhs), _ptr(a), _i(lda),
                      _ptr(b), _i(ldb))


def dgemm_emulated(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                   slices=0):
    """FP64-accurate GEMM on INT8 tensor cores (Ozaki slices; 0 = auto).
    Returns the slice count used."""
    return lib().hwyblas_dgemm_emulated(_c(transa), _c(transb), _i(m), _i(n), _i(k),
                                        _d(alpha), _ptr(a), _i(lda), _ptr(b), _i(ldb),
                                        _d(beta), _ptr(c), _i(ldc), _i(slices))


def dgemm_ddref(transa, transb, m, k, a, lda, b, ldb, n, cols, out, ldo):
    """out[:, jj] = op(A) op(B)[:, cols[jj]] in double-double (error reference)."""
    lib().hwyblas_dgemm_ddref(_c(transa), _c(transb), _i(m), _i(len(cols)), _i(k),
                              _ptr(a), _i(lda), _ptr(b), _i(ldb), _i(n), _ptr(cols),
                              _ptr(out), _i(ldo))


def dresidual_dd(n, nrhs, a, lda, x, ldx, b, ldb, r, ldr):
    """r = b - A x with extra precision (double-double accumulation)."""
    lib().hwyblas_dresidual_dd(_i(n), _i(nrhs), _ptr(a), _i(lda), _ptr(x), _i(ldx),
                               _ptr(b), _i(ldb), _ptr(r), _i(ldr))


def dgesv_mixed(n, nrhs, a, lda, ipiv, b, ldb, x, ldx):
    """Mixed-precision solve (DSGESV semantics). Returns (info, iter)."""
    info, it = ctypes.c_int(0), ctypes.c_int(0)
    lib().hwyblas_dgesv_mixed(_i(n), _i(nrhs), _ptr(a), _i(lda), _ptr(ipiv), _ptr(b),
                              _i(ldb), _ptr(x), _i(ldx), ctypes.byref(it),
                              ctypes.byref(info))
    return info.value, it.value


def dposv_mixed(uplo, n, nrhs, a, lda, b, ldb, x, ldx):
    """Mixed-precision Cholesky solve (DSPOSV semantics). Returns (info, iter)."""
    info, it = ctypes.c_int(0), ctypes.c_int(0)
    lib().hwyblas_dposv_mixed(_c(uplo), _i(n), _i(nrhs), _ptr(a), _i(lda), _ptr(b),
                              _i(ldb), _ptr(x), _i(ldx), ctypes.byref(it),
                              ctypes.byref(info))
    return info.value, it.value


def set_mixed_slices(slices):
    """Slice count of the mixed solvers' trailing updates; returns the old one."""
    return lib().hwyblas_set_mixed_slices(int(slices))


def _ints(vals):
    if isinstance(vals, ctypes.Array):
        return vals
    return (ctypes.c_int * max(1, len(vals)))(*[int(v) for v in vals])


def _ptrs(objs):
    if isinstance(objs, ctypes.Array):
        return objs
    return (ctypes.c_void_p * max(1, len(objs)))(*[_ptr(o) for o in objs])


def int_array(vals):
    """A C int array for the batched calls (a caller repeating a batch
    builds its arguments once, as a C caller keeps its arrays)."""
    return _ints(list(vals))


def ptr_array(objs):
    """A C array of device pointers for the batched calls."""
    return _ptrs(list(objs))


def getrf_batched(n, a, lda, ipiv, precision="d"):
    """Batched LU: n, lda sequences of ints; a, ipiv sequences of device
    buffers (tensors or addresses). Returns the per-problem INFO list."""
    count = len(n)
    info = (ctypes.c_int * max(1, count))()
    fn = lib().hwyblas_dgetrf_batched if precision == "d" else lib().hwyblas_sgetrf_batched
    fn(_ints(n), _ptrs(a), _ints(lda), _ptrs(ipiv), info, count)
    return list(info)[:count]


def getrs_batched(trans, n, nrhs, a, lda, ipiv, b, ldb, precision="d"):
    """Batched LU solve (per-problem sizes as sequences). Returns INFO."""
    info = ctypes.c_int(0)
    fn = lib().hwyblas_dgetrs_batched if precision == "d" else lib().hwyblas_sgetrs_batched
    fn(_c(trans)[0:1], _ints(n), _ints(nrhs),
       _ptrs(a), _ints(lda), _ptrs(ipiv), _ptrs(b), _ints(ldb), len(n), ctypes.byref(info))
    return info.value


def trsm_batched(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, precision="d"):
    """Batched TRSM (per-problem sizes as sequences, shared alpha)."""
    fn = lib().hwyblas_dtrsm_batched if precision == "d" else lib().hwyblas_strsm_batched
    fn(_c(side)[0:1], _c(uplo)[0:1], _c(transa)[0:1], _c(diag)[0:1], _ints(m), _ints(n),
       float(alpha), _ptrs(a), _ints(lda), _ptrs(b), _ints(ldb), len(m))


def gemm_batched(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                 precision="d"):
    """Batched GEMM (per-problem sizes as sequences, shared alpha and beta)."""
    fn = lib().hwyblas_dgemm_batched if precision == "d" else lib().hwyblas_sgemm_batched
    fn(_c(transa)[0:1], _c(transb)[0:1], _ints(m), _ints(n), _ints(k), float(alpha), _ptrs(a),
       _ints(lda), _ptrs(b), _ints(ldb), float(beta), _ptrs(c), _ints(ldc), len(m))


def idamax_noalloc(n, x, incx, result, stream=None):
    """1-based index of max |x| into the device int `result`, with no
    allocation (x and result in device memory); returns the status code."""
    return lib().hwyblas_idamax_noalloc(int(n), _ptr(x), int(incx), _ptr(result),
                                        stream)


def cblas_dgemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c,
                ldc):
    lib().cblas_dgemm(layout, transa, transb, m, n, k, alpha, _ptr(a), lda,
                      _ptr(b), ldb, beta, _ptr(c), ldc)


def cblas_sgemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c,
                ldc):
    lib().cblas_sgemm(layout, transa, transb, m, n, k, alpha, _ptr(a), lda,
                      _ptr(b), ldb, beta, _ptr(c), ldc)


def cblas_dtrsm(layout, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    lib().cblas_dtrsm(layout, side, uplo, transa, diag, m, n, alpha, _ptr(a), lda,
                      _ptr(b), ldb)


def cblas_strsm(layout, side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb):
    """CBLAS FP32 triangular solve (reference cblas_strsm, src/cblas.cc:1950)."""
    lib().cblas_strsm(layout, side, uplo, transa, diag, m, n, alpha, _ptr(a), lda,
                      _ptr(b), ldb)


def cblas_idamax(n, x, incx):
    return lib().cblas_idamax(n, _ptr(x), incx)


_HANDLER_T = ctypes.CFUNCTYPE(None, ctypes.c_char_p, ctypes.c_int)


class ErrorCapture:
    """Installs an error handler that records (name, position) instead of
    printing, as the reference's tests do (tests/lapack/lapack_test_util.h:99)."""

    def __init__(self):
        self.errors = []
        self._cb = _HANDLER_T(self._record)
        self._prev = None

    def _record(self, name, pos):
        self.errors.append((name.decode(), pos))

    def __enter__(self):
        self._prev = lib().hwyblas_set_error_handler(
            ctypes.cast(self._cb, ctypes.c_void_p))
        return self

    def __exit__(self, *exc):
        lib().hwyblas_set_error_handler(self._prev)
        return False


KERNEL_DMMA_GEMM, KERNEL_OZAKI_GEMM, KERNEL_LU_LEAF = 1, 2, 3


def kernel_timer(family):
    """Time every launch of a kernel family with CUDA events (0 = off)."""
    lib().hwyblas_kernel_timer(int(family))


def kernel_timer_read():
    """(total milliseconds, launches) of the timed kernel since the last read."""
    n = ctypes.c_int(0)
    ms = lib().hwyblas_kernel_timer_read(ctypes.byref(n))
    return float(ms), n.value


def launch_count():
    """Kernels launched by the library so far (all threads)."""
    return int(lib().hwyblas_launch_count())


def set_stream(stream):
    """Issue the calling thread's work on `stream` (cudaStream_t as int, or a
    torch.cuda.Stream); None restores the library's stream."""
    if stream is not None and hasattr(stream, "cuda_stream"):
        stream = stream.cuda_stream
    lib().hwyblas_set_stream(stream)
