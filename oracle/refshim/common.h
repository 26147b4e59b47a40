/*
 * refshim/common.h -- minimal stand-in for the dplasma core-kernel build
 * environment, so that the reference's own CORE_d* sources (after its
 * precision generator) compile against scipy's OpenBLAS without PaRSEC or a
 * CMake-generated tree.  TEST INFRASTRUCTURE ONLY (oracle/_ref build).
 * Written for this project; it declares only what those six files use.
 */
#ifndef ORACLE_REFSHIM_COMMON_H
#define ORACLE_REFSHIM_COMMON_H
#include <stdint.h>
#include <stdlib.h>
#include "cblas.h"
#include "lapacke.h"
typedef int PLASMA_enum;
/* dplasma enum -> LAPACK character (values: src/include/dplasma/constants.h:78-99) */
#define lapack_const(x) ((x) == 121 ? 'U' : (x) == 122 ? 'L' : (x) == 123 ? 'A' : \
                         (x) == 111 ? 'N' : (x) == 112 ? 'T' : (x) == 113 ? 'C' : \
                         (x) == 131 ? 'N' : (x) == 132 ? 'U' : (x) == 141 ? 'L' : 'R')
#endif
