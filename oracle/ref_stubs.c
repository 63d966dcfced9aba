/* Fortran BLAS symbols that the reference's LU, Cholesky and triangular
 * sources reference but that the checked path never calls (complex types,
 * condition numbers and refinement of triangular systems). TEST
 * INFRASTRUCTURE ONLY: they abort if reached. */
#include <stdio.h>
#include <stdlib.h>
#define ORC_STUB(name)                                                  \
  void name(void) {                                                     \
    fprintf(stderr, "oracle/_ref: " #name " is not part of the checked path\n"); \
    abort();                                                            \
  }
ORC_STUB(ddot_) ORC_STUB(sdot_) ORC_STUB(cdotc_)
ORC_STUB(dtrsv_) ORC_STUB(strsv_) ORC_STUB(drot_) ORC_STUB(srot_)
ORC_STUB(caxpy_) ORC_STUB(ccopy_) ORC_STUB(cdotu_) ORC_STUB(ctrmm_)
ORC_STUB(ctrmv_) ORC_STUB(ctrsv_) ORC_STUB(dzasum_) ORC_STUB(scasum_)
ORC_STUB(zaxpy_) ORC_STUB(zcopy_) ORC_STUB(zdotu_) ORC_STUB(ztrmm_)
ORC_STUB(ztrmv_) ORC_STUB(ztrsv_)
ORC_STUB(cgemv_) ORC_STUB(cscal_)
ORC_STUB(csscal_) ORC_STUB(cswap_) ORC_STUB(icamax_)
ORC_STUB(izamax_) ORC_STUB(zdotc_) ORC_STUB(zdscal_)
ORC_STUB(zgemv_) ORC_STUB(zscal_) ORC_STUB(zswap_)
