/*
 * ref_driver.c -- drives the reference's own tile kernels (CORE_dplgsy,
 * CORE_dplrnt, CORE_dpotrf, CORE_dtrsm, CORE_dsyrk, CORE_dgemm, compiled from
 * the dplasma sources by oracle/Makefile into oracle/_ref/) through the tile
 * loops of src/zpotrf_L.jdf / src/zpotrf_U.jdf.  PaRSEC (the reference's
 * runtime) is not vendored, so the DAG itself is restated: sequentially
 * (ref_dpotrf) and as OpenMP dependent tasks (ref_dpotrf_parallel, used as
 * the reference CPU timing arm).
 *
 * TEST INFRASTRUCTURE ONLY: validates oracle.c and times the CPU baseline.
 */
#include <stdint.h>
#include <stddef.h>
#include "refshim/common.h"

void CORE_dplgsy(double bump, int m, int n, double *A, int lda, int gM, int m0, int n0,
                 unsigned long long int seed);
void CORE_dplrnt(int m, int n, double *A, int lda, int gM, int m0, int n0, unsigned long long int seed);
void CORE_dpotrf(PLASMA_enum uplo, int N, double *A, int LDA, int *info);
void CORE_dtrsm(PLASMA_enum side, PLASMA_enum uplo, PLASMA_enum transA, PLASMA_enum diag, int M, int N,
                double alpha, const double *A, int LDA, double *B, int LDB);
void CORE_dsyrk(PLASMA_enum uplo, PLASMA_enum trans, int N, int K, double alpha, const double *A, int LDA,
                double beta, double *C, int LDC);
void CORE_dgemm(PLASMA_enum transA, int transB, int M, int N, int K, double alpha, const double *A, int LDA,
                const double *B, int LDB, double beta, double *C, int LDC);

/* Exported wrappers so the tests can call the reference generators tile by tile. */
void ref_dplgsy_tile(double bump, int m, int n, double *A, int lda, int gM, int m0, int n0, uint64_t seed)
{
    CORE_dplgsy(bump, m, n, A, lda, gM, m0, n0, seed);
}
void ref_dplrnt_tile(int m, int n, double *A, int lda, int gM, int m0, int n0, uint64_t seed)
{
    CORE_dplrnt(m, n, A, lda, gM, m0, n0, seed);
}

/* Sequential tile Cholesky over the reference kernels (src/zpotrf_L.jdf,
 * src/zpotrf_U.jdf task bodies in k order). */
int ref_dpotrf(int uplo, int N, int NB, double *A, int lda)
{
    int MT = (N + NB - 1) / NB, info = 0;
#define T(m, n) (A + (size_t)(m) * NB + (size_t)(n) * NB * (size_t)lda)
#define CL(k) (((k) == MT - 1) ? N - (k) * NB : NB)
    for (int k = 0; k < MT; k++) {
        int iinfo = 0;
        CORE_dpotrf(uplo, CL(k), T(k, k), lda, &iinfo);
        if (iinfo != 0 && info == 0) info = k * NB + iinfo;
        for (int m = k + 1; m < MT; m++) {
            if (uplo == 122) CORE_dtrsm(142, 122, 112, 131, CL(m), NB, 1.0, T(k, k), lda, T(m, k), lda);
            else             CORE_dtrsm(141, 121, 112, 131, NB, CL(m), 1.0, T(k, k), lda, T(k, m), lda);
        }
        for (int m = k + 1; m < MT; m++) {
            if (uplo == 122) {
                CORE_dsyrk(122, 111, CL(m), NB, -1.0, T(m, k), lda, 1.0, T(m, m), lda);
                for (int n = k + 1; n < m; n++)
                    CORE_dgemm(111, 112, CL(m), NB, NB, -1.0, T(m, k), lda, T(n, k), lda, 1.0, T(m, n), lda);
            } else {
                CORE_dsyrk(121, 112, CL(m), NB, -1.0, T(k, m), lda, 1.0, T(m, m), lda);
                for (int n = k + 1; n < m; n++)
                    CORE_dgemm(112, 111, NB, CL(m), NB, -1.0, T(k, n), lda, T(k, m), lda, 1.0, T(n, m), lda);
            }
        }
    }
#undef T
#undef CL
    return info;
}

#define TD_NAME ref_dag_dpotrf
#define TD_POTRF(uplo, n, T, ld, iinfo) CORE_dpotrf((uplo), (n), (T), (ld), (iinfo))
#define TD_TRSM(side, uplo, trans, m, n, T, ldt, C, ldc) \
    CORE_dtrsm((side), (uplo), (trans), 131, (m), (n), 1.0, (T), (ldt), (C), (ldc))
#define TD_SYRK(uplo, trans, n, k, A, lda, C, ldc) CORE_dsyrk((uplo), (trans), (n), (k), -1.0, (A), (lda), 1.0, (C), (ldc))
#define TD_GEMM(ta, tb, m, n, k, A, lda, B, ldb, C, ldc) \
    CORE_dgemm((ta), (tb), (m), (n), (k), -1.0, (A), (lda), (B), (ldb), 1.0, (C), (ldc))
#include "tile_dag.h"

int ref_dpotrf_parallel(int uplo, int N, int NB, double *A, int lda, int nthreads)
{
    if (uplo != 121 && uplo != 122) return -1;
    int saved = scipy_openblas_get_num_threads();
    scipy_openblas_set_num_threads(1);
    int info = ref_dag_dpotrf(uplo, N, NB, A, lda, nthreads);
    scipy_openblas_set_num_threads(saved);
    return info;
}
