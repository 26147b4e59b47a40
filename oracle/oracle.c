/*
 * oracle.c -- CPU restatement of DPLASMA's tile Cholesky factor-and-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the
 * B200 library: only the tests, the smoke entry and the CPU-baseline leg of
 * the benchmark load it.  The product library never links or calls it.
 *
 * Every routine restates the reference algorithm and cites the reference file
 * and lines it follows (paths are relative to the dplasma source tree).
 * Arithmetic that the reference delegates to BLAS/LAPACK goes to the OpenBLAS
 * build shipped in the scipy wheel (see blas_shim.h).
 *
 * Storage used here: one dense column-major array with leading dimension lda
 * (the LAPACK layout).  Tile (m,n) of an NB-blocked matrix starts at
 * A + m*NB + n*NB*lda and has CLEAN_MB x CLEAN_NB valid entries
 * (src/floputils.h:6-7).  The tile algorithms issue exactly the BLAS calls of
 * the reference task bodies, each tile updated in increasing k as PaRSEC
 * serialises them (src/zpotrf_L.jdf:486-491), so with one BLAS thread the
 * result is the reference CPU result for the same BLAS.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include "blas_shim.h"

#define ORC_UPPER 121
#define ORC_LOWER 122
#define ORC_UPPERLOWER 123
#define ORC_NOTRANS 111
#define ORC_TRANS 112
#define ORC_CONJTRANS 113
#define ORC_NONUNIT 131
#define ORC_UNIT 132

/* ------------------------------------------------------------------------ */
/* Random generator: 64-bit LCG with O(log n) jump-ahead.                    */
/* src/cores/random.h:19-41 (constants at random.h:19-22).                   */
/* ------------------------------------------------------------------------ */
static const uint64_t ORC_LCG_A = 6364136223846793005ULL;
static const uint64_t ORC_LCG_C = 1ULL;
static const float ORC_RNDF_MUL = 5.4210108624275222e-20f;

uint64_t orc_rnd64_jump(uint64_t n, uint64_t seed)
{
    uint64_t a_k = ORC_LCG_A, c_k = ORC_LCG_C, ran = seed;
    /* binary powering of the affine map x -> a*x + c */
    while (n) {
        if (n & 1ULL) ran = a_k * ran + c_k;
        c_k *= (a_k + 1ULL);
        a_k *= a_k;
        n >>= 1;
    }
    return ran;
}

/* One generated value: single-precision arithmetic stored in double
 * (src/cores/core_zplgsy.c:89 `0.5f - ran * RndF_Mul`).  The file is
 * compiled with -ffp-contract=off so the multiply and subtract round
 * separately, as a plain x86-64 build of the reference does. */
static inline double orc_value(uint64_t ran)
{
    float r = (float)ran;
    float p = r * ORC_RNDF_MUL;
    float v = 0.5f - p;
    return (double)v;
}

/* CORE_dplgsy restated: src/cores/core_zplgsy.c:72-150 (REAL, NBELEM=1).
 * Entry (i,j) of the global matrix, i>=j, is the LCG value at jump index
 * i + j*gM; the upper part mirrors the lower; `bump` is added on the
 * diagonal of diagonal tiles. */
void orc_dplgsy_tile(double bump, int m, int n, double *A, int lda,
                     int gM, int m0, int n0, uint64_t seed)
{
    int64_t i, j;
    if (m0 == n0) {
        for (j = 0; j < n; j++) {
            uint64_t ran = orc_rnd64_jump((uint64_t)(m0 + j) + (uint64_t)(n0 + j) * (uint64_t)gM, seed);
            for (i = j; i < m; i++) {
                A[i + j * (int64_t)lda] = orc_value(ran);
                ran = ORC_LCG_A * ran + ORC_LCG_C;
            }
        }
        for (j = 0; j < n; j++) {
            A[j + j * (int64_t)lda] += bump;
            for (i = 0; i < j; i++)
                A[i + j * (int64_t)lda] = A[j + i * (int64_t)lda];
        }
    } else if (m0 > n0) {
        for (j = 0; j < n; j++) {
            uint64_t ran = orc_rnd64_jump((uint64_t)m0 + (uint64_t)(n0 + j) * (uint64_t)gM, seed);
            for (i = 0; i < m; i++) {
                A[i + j * (int64_t)lda] = orc_value(ran);
                ran = ORC_LCG_A * ran + ORC_LCG_C;
            }
        }
    } else {
        for (i = 0; i < m; i++) {
            uint64_t ran = orc_rnd64_jump((uint64_t)n0 + (uint64_t)(m0 + i) * (uint64_t)gM, seed);
            for (j = 0; j < n; j++) {
                A[i + j * (int64_t)lda] = orc_value(ran);
                ran = ORC_LCG_A * ran + ORC_LCG_C;
            }
        }
    }
}

/* CORE_dplrnt restated: src/cores/core_zplrnt.c:68-91. */
void orc_dplrnt_tile(int m, int n, double *A, int lda, int gM, int m0, int n0, uint64_t seed)
{
    for (int64_t j = 0; j < n; j++) {
        uint64_t ran = orc_rnd64_jump((uint64_t)m0 + (uint64_t)(n0 + j) * (uint64_t)gM, seed);
        for (int64_t i = 0; i < m; i++) {
            A[i + j * (int64_t)lda] = orc_value(ran);
            ran = ORC_LCG_A * ran + ORC_LCG_C;
        }
    }
}

static inline int orc_clean(int k, int kt, int n, int nb) { return (k == kt - 1) ? n - k * nb : nb; }
static inline double *orc_tile(double *A, int lda, int nb, int m, int n)
{
    return A + (size_t)m * nb + (size_t)n * nb * (size_t)lda;
}

/* dplasma_dplgsy over a dense array: the apply operator of
 * src/zplgsy_wrapper.c:23-43 run on every tile of the `uplo` region
 * (dplasmaLower: m>=n, dplasmaUpper: m<=n, dplasmaUpperLower: all). */
void orc_dplgsy(double bump, int uplo, int N, int NB, double *A, int lda, uint64_t seed)
{
    int MT = (N + NB - 1) / NB;
    for (int n = 0; n < MT; n++)
        for (int m = 0; m < MT; m++) {
            if (uplo == ORC_LOWER && m < n) continue;
            if (uplo == ORC_UPPER && m > n) continue;
            orc_dplgsy_tile(bump, orc_clean(m, MT, N, NB), orc_clean(n, MT, N, NB),
                            orc_tile(A, lda, NB, m, n), lda, N, m * NB, n * NB, seed);
        }
}

/* dplasma_dplrnt over a dense M x N array: src/zplrnt_wrapper.c:24-64. */
void orc_dplrnt(int diagdom, int M, int N, int MB, int NB, double *A, int lda, uint64_t seed)
{
    int MT = (M + MB - 1) / MB, NT = (N + NB - 1) / NB;
    for (int n = 0; n < NT; n++)
        for (int m = 0; m < MT; m++) {
            int tm = orc_clean(m, MT, M, MB), tn = orc_clean(n, NT, N, NB);
            double *T = A + (size_t)m * MB + (size_t)n * NB * (size_t)lda;
            orc_dplrnt_tile(tm, tn, T, lda, M, m * MB, n * NB, seed);
            if (diagdom && m == n) {
                double alpha = (double)(M > N ? M : N);
                int mn = tm < tn ? tm : tn;
                for (int i = 0; i < mn; i++) T[i + (size_t)i * lda] += alpha;
            }
        }
}

/* ------------------------------------------------------------------------ */
/* Tile Cholesky.                                                            */
/* Lower: src/zpotrf_L.jdf task bodies potrf (:194-206), trsm (:324-343),    */
/*        herk->syrk (:447-464), gemm (:612-633).                            */
/* Upper: src/zpotrf_U.jdf potrf (:194-206), trsm (:326-345),                */
/*        herk->syrk (:450-468), gemm (:626-648).                            */
/* INFO = k*NB + iinfo of the first failing diagonal tile                    */
/* (src/zpotrf_L.jdf:200-202); the DAG keeps running, as in the reference.   */
/* ------------------------------------------------------------------------ */
int orc_dpotrf(int uplo, int N, int NB, double *A, int lda)
{
    int MT = (N + NB - 1) / NB;
    int info = 0;
    if (uplo != ORC_LOWER && uplo != ORC_UPPER) return -1;
    for (int k = 0; k < MT; k++) {
        int tk = orc_clean(k, MT, N, NB);
        double *Tkk = orc_tile(A, lda, NB, k, k);
        int iinfo = LAPACKE_dpotrf_work(LAPACK_COL_MAJOR, uplo == ORC_LOWER ? 'L' : 'U', tk, Tkk, lda);
        if (iinfo != 0 && info == 0) info = k * NB + iinfo;
        if (uplo == ORC_LOWER) {
            for (int m = k + 1; m < MT; m++)
                cblas_dtrsm(CblasColMajor, CblasRight, CblasLower, CblasTrans, CblasNonUnit,
                            orc_clean(m, MT, N, NB), NB, 1.0, Tkk, lda, orc_tile(A, lda, NB, m, k), lda);
            for (int m = k + 1; m < MT; m++) {
                int tm = orc_clean(m, MT, N, NB);
                double *Amk = orc_tile(A, lda, NB, m, k);
                cblas_dsyrk(CblasColMajor, CblasLower, CblasNoTrans, tm, NB,
                            -1.0, Amk, lda, 1.0, orc_tile(A, lda, NB, m, m), lda);
                for (int n = k + 1; n < m; n++)
                    cblas_dgemm(CblasColMajor, CblasNoTrans, CblasTrans, tm, NB, NB,
                                -1.0, Amk, lda, orc_tile(A, lda, NB, n, k), lda,
                                1.0, orc_tile(A, lda, NB, m, n), lda);
            }
        } else {
            for (int n = k + 1; n < MT; n++)
                cblas_dtrsm(CblasColMajor, CblasLeft, CblasUpper, CblasTrans, CblasNonUnit,
                            NB, orc_clean(n, MT, N, NB), 1.0, Tkk, lda, orc_tile(A, lda, NB, k, n), lda);
            for (int n = k + 1; n < MT; n++) {
                int tn = orc_clean(n, MT, N, NB);
                double *Akn = orc_tile(A, lda, NB, k, n);
                cblas_dsyrk(CblasColMajor, CblasUpper, CblasTrans, tn, NB,
                            -1.0, Akn, lda, 1.0, orc_tile(A, lda, NB, n, n), lda);
                for (int m = k + 1; m < n; m++)
                    cblas_dgemm(CblasColMajor, CblasTrans, CblasNoTrans, NB, tn, NB,
                                -1.0, orc_tile(A, lda, NB, k, m), lda, Akn, lda,
                                1.0, orc_tile(A, lda, NB, m, n), lda);
            }
        }
    }
    return info;
}

/* ------------------------------------------------------------------------ */
/* Left triangular solves, tile by tile.                                     */
/*   LLN: src/ztrsm_LLN.jdf:29-191   forward,  B_m -= A(m,k) B_k            */
/*   LLT: src/ztrsm_LLT.jdf:29-190   backward, B_m -= A(k,m)^T B_k          */
/*   LUN: src/ztrsm_LUN.jdf:29-187   backward, B_m -= A(m,k) B_k            */
/*   LUT: src/ztrsm_LUT.jdf:29-187   forward,  B_m -= A(k,m)^T B_k          */
/* alpha is applied with the first touch of each tile (lalpha, e.g.          */
/* src/ztrsm_LLN.jdf:47,155).  B is N x NRHS, blocked NB x NB.               */
/* ------------------------------------------------------------------------ */
int orc_dtrsm_left(int uplo, int trans, int diag, double alpha, int N, int NRHS, int NB,
                   const double *A, int lda, double *B, int ldb)
{
    int MT = (N + NB - 1) / NB, NT = (NRHS + NB - 1) / NB;
    int notrans = (trans == ORC_NOTRANS);
    int forward = (uplo == ORC_LOWER) ? notrans : !notrans;
    CBLAS_TRANSPOSE tA = notrans ? CblasNoTrans : CblasTrans;
    for (int kk = 0; kk < MT; kk++) {
        int k = forward ? kk : MT - 1 - kk;
        int tk = orc_clean(k, MT, N, NB);
        const double *Akk = A + (size_t)k * NB + (size_t)k * NB * lda;
        double lalpha = (kk == 0) ? alpha : 1.0;
        for (int n = 0; n < NT; n++) {
            int tn = orc_clean(n, NT, NRHS, NB);
            cblas_dtrsm(CblasColMajor, CblasLeft, (CBLAS_UPLO)uplo, tA, (CBLAS_DIAG)diag,
                        tk, tn, lalpha, Akk, lda, B + (size_t)k * NB + (size_t)n * NB * ldb, ldb);
        }
        for (int mm = kk + 1; mm < MT; mm++) {
            int m = forward ? mm : MT - 1 - mm;
            int tm = orc_clean(m, MT, N, NB);
            /* op(A) block that couples unknown block k into equation block m */
            const double *Amk;
            if ((uplo == ORC_LOWER && notrans) || (uplo == ORC_UPPER && notrans))
                Amk = A + (size_t)m * NB + (size_t)k * NB * lda;      /* A(m,k) */
            else
                Amk = A + (size_t)k * NB + (size_t)m * NB * lda;      /* A(k,m), used transposed */
            for (int n = 0; n < NT; n++) {
                int tn = orc_clean(n, NT, NRHS, NB);
                if (notrans)
                    cblas_dgemm(CblasColMajor, CblasNoTrans, CblasNoTrans, tm, tn, tk,
                                -1.0, Amk, lda, B + (size_t)k * NB + (size_t)n * NB * ldb, ldb,
                                lalpha, B + (size_t)m * NB + (size_t)n * NB * ldb, ldb);
                else
                    cblas_dgemm(CblasColMajor, CblasTrans, CblasNoTrans, tm, tn, tk,
                                -1.0, Amk, lda, B + (size_t)k * NB + (size_t)n * NB * ldb, ldb,
                                lalpha, B + (size_t)m * NB + (size_t)n * NB * ldb, ldb);
            }
        }
    }
    return 0;
}

/* dplasma_dpotrs: src/zpotrs_wrapper.c:56-97 (the non-composed branch
 * :87-95).  Lower: LLN then LLT.  Upper: LUT then LUN. */
int orc_dpotrs(int uplo, int N, int NRHS, int NB, const double *A, int lda, double *B, int ldb)
{
    if (uplo != ORC_UPPER && uplo != ORC_LOWER) return -1;
    if (uplo == ORC_UPPER) {
        orc_dtrsm_left(uplo, ORC_TRANS, ORC_NONUNIT, 1.0, N, NRHS, NB, A, lda, B, ldb);
        orc_dtrsm_left(uplo, ORC_NOTRANS, ORC_NONUNIT, 1.0, N, NRHS, NB, A, lda, B, ldb);
    } else {
        orc_dtrsm_left(uplo, ORC_NOTRANS, ORC_NONUNIT, 1.0, N, NRHS, NB, A, lda, B, ldb);
        orc_dtrsm_left(uplo, ORC_TRANS, ORC_NONUNIT, 1.0, N, NRHS, NB, A, lda, B, ldb);
    }
    return 0;
}

/* dplasma_dposv: src/zposv_wrapper.c:63-113 (non-composed branch :100-111):
 * factor, and solve only when info == 0. */
int orc_dposv(int uplo, int N, int NRHS, int NB, double *A, int lda, double *B, int ldb)
{
    if (uplo != ORC_UPPER && uplo != ORC_LOWER) return -1;
    int info = orc_dpotrf(uplo, N, NB, A, lda);
    if (info == 0) orc_dpotrs(uplo, N, NRHS, NB, A, lda, B, ldb);
    return info;
}

/* ------------------------------------------------------------------------ */
/* Residual checks: src/dplasma_zcheck.c.                                    */
/* ------------------------------------------------------------------------ */

/* LAPACK dlamch('e'): relative machine epsilon for rounding arithmetic,
 * the value src/dplasma_zcheck.c:75 obtains via LAPACKE_dlamch_work('e'). */
double orc_eps(void) { return DBL_EPSILON * 0.5; }

/* Infinity norm of a symmetric matrix given by its `uplo` triangle
 * (dplasma_dlansy with dplasmaInfNorm). */
double orc_dlansy_inf(int uplo, int N, const double *A, int lda)
{
    double *rs = (double *)calloc((size_t)N, sizeof(double));
    double nrm = 0.0;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            int in_tri = (uplo == ORC_LOWER) ? (i >= j) : (i <= j);
            if (!in_tri) continue;
            double v = fabs(A[i + (size_t)j * lda]);
            rs[i] += v;
            if (i != j) rs[j] += v;
        }
    for (int i = 0; i < N; i++) {
        if (isnan(rs[i])) { nrm = rs[i]; break; }
        if (rs[i] > nrm) nrm = rs[i];
    }
    free(rs);
    return nrm;
}

/* Infinity norm of a general M x N matrix (dplasma_dlange, dplasmaInfNorm). */
double orc_dlange_inf(int M, int N, const double *A, int lda)
{
    double *rs = (double *)calloc((size_t)M, sizeof(double));
    double nrm = 0.0;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < M; i++) rs[i] += fabs(A[i + (size_t)j * lda]);
    for (int i = 0; i < M; i++) {
        if (isnan(rs[i])) { nrm = rs[i]; break; }
        if (rs[i] > nrm) nrm = rs[i];
    }
    free(rs);
    return nrm;
}

/* check_dpotrf: src/dplasma_zcheck.c:63-133.
 * LLt = tri(A) ; LLt = LLt * tri(A)^T (Right/Lower) or tri(A)^T * LLt (Left/Upper);
 * R = LLt - A0 on the uplo triangle; ratio = ||R||_inf / (||A0||_inf N eps).
 * Returns the ratio; the reference flags a failure above 60 (:116-118). */
double orc_check_dpotrf(int uplo, int N, const double *A, int lda, const double *A0, int lda0,
                        double *Rnorm_out, double *Anorm_out)
{
    double *LLt = (double *)calloc((size_t)N * N, sizeof(double));
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            int in_tri = (uplo == ORC_LOWER) ? (i >= j) : (i <= j);
            if (in_tri) LLt[i + (size_t)j * N] = A[i + (size_t)j * lda];
        }
    if (uplo == ORC_LOWER)
        cblas_dtrmm(CblasColMajor, CblasRight, CblasLower, CblasTrans, CblasNonUnit, N, N, 1.0, A, lda, LLt, N);
    else
        cblas_dtrmm(CblasColMajor, CblasLeft, CblasUpper, CblasTrans, CblasNonUnit, N, N, 1.0, A, lda, LLt, N);
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            int in_tri = (uplo == ORC_LOWER) ? (i >= j) : (i <= j);
            if (in_tri) LLt[i + (size_t)j * N] -= A0[i + (size_t)j * lda0];
        }
    double Anorm = orc_dlansy_inf(uplo, N, A0, lda0);
    double Rnorm = orc_dlansy_inf(uplo, N, LLt, N);
    free(LLt);
    if (Rnorm_out) *Rnorm_out = Rnorm;
    if (Anorm_out) *Anorm_out = Anorm;
    return Rnorm / (Anorm * N * orc_eps());
}

/* check_daxmb: src/dplasma_zcheck.c:179-224.
 * ratio = ||B - A0 X||_inf / ((||A0||_inf ||X||_inf + ||B||_inf) N eps),
 * A0 symmetric given by its uplo triangle (dsymm). */
double orc_check_daxmb(int uplo, int N, int NRHS, const double *A0, int lda, const double *B, int ldb,
                       const double *X, int ldx)
{
    double Anorm = orc_dlansy_inf(uplo, N, A0, lda);
    double Bnorm = orc_dlange_inf(N, NRHS, B, ldb);
    double Xnorm = orc_dlange_inf(N, NRHS, X, ldx);
    double *R = (double *)malloc((size_t)N * NRHS * sizeof(double));
    for (int j = 0; j < NRHS; j++) memcpy(R + (size_t)j * N, B + (size_t)j * ldb, sizeof(double) * N);
    cblas_dsymm(CblasColMajor, CblasLeft, (CBLAS_UPLO)uplo, N, NRHS, -1.0, A0, lda, X, ldx, 1.0, R, N);
    double Rnorm = orc_dlange_inf(N, NRHS, R, N);
    free(R);
    return Rnorm / ((Anorm * Xnorm + Bnorm) * N * orc_eps());
}

void orc_set_blas_threads(int n) { scipy_openblas_set_num_threads(n); }

/* ------------------------------------------------------------------------ */
/* Parallel tile DAG on the host cores (CPU baseline timing).                */
/* ------------------------------------------------------------------------ */
#define TD_NAME orc_dag_dpotrf
#define TD_POTRF(uplo, n, T, ld, iinfo) \
    (*(iinfo) = LAPACKE_dpotrf_work(LAPACK_COL_MAJOR, (uplo) == ORC_LOWER ? 'L' : 'U', (n), (T), (ld)))
#define TD_TRSM(side, uplo, trans, m, n, T, ldt, C, ldc) \
    cblas_dtrsm(CblasColMajor, (CBLAS_SIDE)(side), (CBLAS_UPLO)(uplo), (CBLAS_TRANSPOSE)(trans), CblasNonUnit, \
                (m), (n), 1.0, (T), (ldt), (C), (ldc))
#define TD_SYRK(uplo, trans, n, k, A, lda, C, ldc) \
    cblas_dsyrk(CblasColMajor, (CBLAS_UPLO)(uplo), (CBLAS_TRANSPOSE)(trans), (n), (k), -1.0, (A), (lda), 1.0, (C), (ldc))
#define TD_GEMM(ta, tb, m, n, k, A, lda, B, ldb, C, ldc) \
    cblas_dgemm(CblasColMajor, (CBLAS_TRANSPOSE)(ta), (CBLAS_TRANSPOSE)(tb), (m), (n), (k), -1.0, (A), (lda), \
                (B), (ldb), 1.0, (C), (ldc))
#include "tile_dag.h"

/* Tile Cholesky as a parallel DAG with `nthreads` host threads, one BLAS
 * thread per task.  Same kernels and per-tile update order as orc_dpotrf. */
int orc_dpotrf_parallel(int uplo, int N, int NB, double *A, int lda, int nthreads)
{
    if (uplo != ORC_LOWER && uplo != ORC_UPPER) return -1;
    int saved = scipy_openblas_get_num_threads();
    scipy_openblas_set_num_threads(1);
    int info = orc_dag_dpotrf(uplo, N, NB, A, lda, nthreads);
    scipy_openblas_set_num_threads(saved);
    return info;
}
