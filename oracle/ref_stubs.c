/* Fortran BLAS symbols that the reference's LU/Cholesky sources reference but
 * that the checked path never calls (complex types, xGETRI). TEST
 * INFRASTRUCTURE ONLY: they abort if reached. */
#include <stdio.h>
#include <stdlib.h>
#define ORC_STUB(name)                                                  \
  void name(void) {                                                     \
    fprintf(stderr, "oracle/_ref: " #name " is not part of the checked path\n"); \
    abort();                                                            \
  }
ORC_STUB(dswap_) ORC_STUB(sswap_) ORC_STUB(ddot_) ORC_STUB(sdot_)
ORC_STUB(dgemv_) ORC_STUB(sgemv_) ORC_STUB(cdotc_)
ORC_STUB(cgemm_) ORC_STUB(cgemv_) ORC_STUB(cherk_) ORC_STUB(cscal_)
ORC_STUB(csscal_) ORC_STUB(cswap_) ORC_STUB(ctrsm_) ORC_STUB(icamax_)
ORC_STUB(izamax_) ORC_STUB(zdotc_) ORC_STUB(zdscal_) ORC_STUB(zgemm_)
ORC_STUB(zgemv_) ORC_STUB(zherk_) ORC_STUB(zscal_) ORC_STUB(zswap_)
ORC_STUB(ztrsm_)
