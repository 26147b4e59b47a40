/* refshim/lapacke.h -- LAPACKE names used by the reference CORE kernels,
 * bound to scipy's OpenBLAS.  TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_REFSHIM_LAPACKE_H
#define ORACLE_REFSHIM_LAPACKE_H
#include "../blas_shim.h"
#endif
