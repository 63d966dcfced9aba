// Highway-API shim (TEST INFRASTRUCTURE ONLY): with one static target, the
// including file is compiled once, so there is nothing to re-include. The
// per-target include guards of the "-inl.h" files work unchanged because
// HWY_TARGET_TOGGLE is never defined.
#include "hwy/base.h"
