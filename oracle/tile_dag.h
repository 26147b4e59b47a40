/*
 * tile_dag.h -- the tile Cholesky DAG of src/zpotrf_L.jdf / src/zpotrf_U.jdf
 * run as OpenMP dependent tasks over tiles, the way PaRSEC runs it on CPU
 * cores: one task per POTRF(k), TRSM(m,k), SYRK(k,m), GEMM(m,n,k), data
 * dependences on tiles (dataflow edges src/zpotrf_L.jdf:107-112,229-237,
 * 364-368,486-491) and the JDF priorities (src/zpotrf_L.jdf:53-64) as task
 * priority hints.  Each task calls a single-threaded tile kernel.
 *
 * TEST INFRASTRUCTURE ONLY (CPU baseline timing).  Included by oracle.c
 * (kernels = direct BLAS calls) and by ref_driver.c (kernels = the
 * reference's own CORE_d* routines built from its sources).
 *
 * Before including, define:
 *   TD_NAME                      name of the generated function
 *   TD_POTRF(uplo, n, T, ld, iinfo_ptr)
 *   TD_TRSM(side, uplo, trans, m, n, T, ldt, C, ldc)   (alpha = 1, NonUnit)
 *   TD_SYRK(uplo, trans, n, k, A, lda, C, ldc)          (alpha = -1, beta = 1)
 *   TD_GEMM(transA, transB, m, n, k, A, lda, B, ldb, C, ldc) (alpha=-1, beta=1)
 */
#include <omp.h>

static int TD_NAME(int uplo, int N, int NB, double *A, int lda, int nthreads)
{
    int MT = (N + NB - 1) / NB;
    int info = 0;
#define TD_T(m, n) (A + (size_t)(m) * NB + (size_t)(n) * NB * (size_t)lda)
#define TD_CLEAN(k) (((k) == MT - 1) ? N - (k) * NB : NB)
#define TD_PRI(x) ((x) > 2000000 ? 2000000 : (x))
#pragma omp parallel num_threads(nthreads) shared(info)
#pragma omp single
    {
        for (int k = 0; k < MT; k++) {
            double *Tkk = TD_T(k, k);
            int pk = TD_PRI((MT - k) * (MT - k) * (MT - k));
#pragma omp task depend(inout : Tkk[0]) firstprivate(k, Tkk) shared(info) priority(pk)
            {
                int iinfo = 0;
                TD_POTRF(uplo, TD_CLEAN(k), Tkk, lda, &iinfo);
                if (iinfo != 0) {
#pragma omp critical
                    if (info == 0) info = k * NB + iinfo;
                }
            }
            for (int m = k + 1; m < MT; m++) {
                double *C = (uplo == 122) ? TD_T(m, k) : TD_T(k, m);
                int pm = TD_PRI((MT - m) * (MT - m) * (MT - m) + 3 * (2 * MT - k - m - 1) * (m - k));
#pragma omp task depend(in : Tkk[0]) depend(inout : C[0]) firstprivate(m, k, C, Tkk) priority(pm)
                {
                    if (uplo == 122) TD_TRSM(142, 122, 112, TD_CLEAN(m), NB, Tkk, lda, C, lda);
                    else             TD_TRSM(141, 121, 112, NB, TD_CLEAN(m), Tkk, lda, C, lda);
                }
            }
            for (int m = k + 1; m < MT; m++) {
                double *Amk = (uplo == 122) ? TD_T(m, k) : TD_T(k, m);
                double *Tmm = TD_T(m, m);
                int ps = TD_PRI((MT - m) * (MT - m) * (MT - m) + 3 * (m - k));
#pragma omp task depend(in : Amk[0]) depend(inout : Tmm[0]) firstprivate(m, Amk, Tmm) priority(ps)
                {
                    if (uplo == 122) TD_SYRK(122, 111, TD_CLEAN(m), NB, Amk, lda, Tmm, lda);
                    else             TD_SYRK(121, 112, TD_CLEAN(m), NB, Amk, lda, Tmm, lda);
                }
                for (int n = k + 1; n < m; n++) {
                    int pg = TD_PRI((MT - m) * (MT - m) * (MT - m) + 3 * (m - n) * (2 * MT - m - n - 3) + 6 * (m - k));
                    if (uplo == 122) {
                        double *Ank = TD_T(n, k), *Cmn = TD_T(m, n);
#pragma omp task depend(in : Amk[0], Ank[0]) depend(inout : Cmn[0]) firstprivate(m, Amk, Ank, Cmn) priority(pg)
                        TD_GEMM(111, 112, TD_CLEAN(m), NB, NB, Amk, lda, Ank, lda, Cmn, lda);
                    } else {
                        double *Akn = TD_T(k, n), *Cnm = TD_T(n, m);
#pragma omp task depend(in : Amk[0], Akn[0]) depend(inout : Cnm[0]) firstprivate(m, Amk, Akn, Cnm) priority(pg)
                        TD_GEMM(112, 111, NB, TD_CLEAN(m), NB, Akn, lda, Amk, lda, Cnm, lda);
                    }
                }
            }
        }
#pragma omp taskwait
    }
#undef TD_T
#undef TD_CLEAN
#undef TD_PRI
    return info;
}
