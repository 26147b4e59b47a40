/*
 * blas_shim.h -- declarations of the CBLAS / LAPACKE entry points the CPU
 * oracle calls, bound to the OpenBLAS build that ships inside the scipy
 * wheel (its exported symbols carry a "scipy_" prefix).
 *
 * TEST INFRASTRUCTURE ONLY: nothing in the product library includes this.
 *
 * The enum values follow the CBLAS standard, which is also what dplasma uses
 * for its own constants (src/include/dplasma/constants.h:78-99), so a
 * dplasma_enum_t can be passed straight through, as the reference's
 * src/cores/core_ztrsm.c:86 does.
 */
#ifndef ORACLE_BLAS_SHIM_H
#define ORACLE_BLAS_SHIM_H

#ifndef ORACLE_CBLAS_ENUMS_DEFINED
#define ORACLE_CBLAS_ENUMS_DEFINED
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;
#endif

#define LAPACK_COL_MAJOR 102
typedef int lapack_int;

void scipy_cblas_dgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int,
                       double, const double *, int, const double *, int, double, double *, int);
void scipy_cblas_dsyrk(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, int, int,
                       double, const double *, int, double, double *, int);
void scipy_cblas_dtrsm(CBLAS_ORDER, CBLAS_SIDE, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG,
                       int, int, double, const double *, int, double *, int);
void scipy_cblas_dtrmm(CBLAS_ORDER, CBLAS_SIDE, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG,
                       int, int, double, const double *, int, double *, int);
void scipy_cblas_dsymm(CBLAS_ORDER, CBLAS_SIDE, CBLAS_UPLO, int, int,
                       double, const double *, int, const double *, int, double, double *, int);
lapack_int scipy_LAPACKE_dpotrf_work(int, char, lapack_int, double *, lapack_int);
void scipy_openblas_set_num_threads(int);
int scipy_openblas_get_num_threads(void);

#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dsyrk scipy_cblas_dsyrk
#define cblas_dtrsm scipy_cblas_dtrsm
#define cblas_dtrmm scipy_cblas_dtrmm
#define cblas_dsymm scipy_cblas_dsymm
#define LAPACKE_dpotrf_work scipy_LAPACKE_dpotrf_work

#endif
