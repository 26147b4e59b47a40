/* refshim/cblas.h -- CBLAS names used by the reference CORE kernels, bound to
 * scipy's OpenBLAS.  TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_REFSHIM_CBLAS_H
#define ORACLE_REFSHIM_CBLAS_H
#include "../blas_shim.h"
#endif
