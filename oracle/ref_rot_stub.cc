// The one reference kernel the Highway-API shim does not restate: xLASR's
// rotation sequences (src/lapack/rotation_kernels.cc), which use x86 block
// shuffles and serve only the SVD and eigenvalue drivers. TEST
// INFRASTRUCTURE ONLY: it aborts if reached; nothing on the checked path
// (GEMM, TRSM, LU, Cholesky and their solvers) calls it.
#include <cstdio>
#include <cstdlib>
#include <complex>

#include "src/lapack/rotation_kernels.h"

namespace hwyblas {
namespace lapack {

template <typename T>
void LasrVariable(bool, bool, blasint, blasint, const RealT<T>*, const RealT<T>*, T*, blasint) {
  std::fprintf(stderr, "oracle/_ref: xLASR is not part of the checked path\n");
  std::abort();
}
template void LasrVariable<float>(bool, bool, blasint, blasint, const float*, const float*,
                                  float*, blasint);
template void LasrVariable<double>(bool, bool, blasint, blasint, const double*,
                                   const double*, double*, blasint);
template void LasrVariable<std::complex<float>>(bool, bool, blasint, blasint, const float*,
                                                const float*, std::complex<float>*, blasint);
template void LasrVariable<std::complex<double>>(bool, bool, blasint, blasint,
                                                 const double*, const double*,
                                                 std::complex<double>*, blasint);

}  // namespace lapack
}  // namespace hwyblas
