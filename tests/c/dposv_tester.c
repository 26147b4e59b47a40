/* A plain C caller of the library, in the shape of the reference's
 * tests/testing_zposv.c: dplasma_dplgsy / dplasma_dplrnt, dplasma_dposv on
 * host TILE descriptors, the check_daxmb ratio (src/dplasma_zcheck.c:179-224)
 * restated with loops; then ScaLAPACK's PDPOTRF (pdpotrf_) on a column-major
 * copy of the same matrix, checked with the check_dpotrf ratio
 * (src/dplasma_zcheck.c:63-133).  Prints "ok" and returns 0 when both ratios
 * are below 10.  Usage: dposv_tester [N] [NB] [NRHS]. */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dplasma_b200.h"

static double get_sym(const parsec_tiled_matrix_t *A, int i, int j)
{
    if (i < j) {
        int t = i;
        i = j;
        j = t;
    }
    const double *T = (const double *)A->mat + dplasma_b200_tile_offset(A, i / A->mb, j / A->nb);
    return T[(j % A->nb) * A->mb + (i % A->mb)];
}

static double get_gen(const parsec_tiled_matrix_t *B, int i, int j)
{
    const double *T = (const double *)B->mat + dplasma_b200_tile_offset(B, i / B->mb, j / B->nb);
    return T[(j % B->nb) * B->mb + (i % B->mb)];
}

int main(int argc, char **argv)
{
    const int N = argc > 1 ? atoi(argv[1]) : 1000;
    const int NB = argc > 2 ? atoi(argv[2]) : 256;
    const int NRHS = argc > 3 ? atoi(argv[3]) : 8;
    const double eps = DBL_EPSILON / 2.0;   /* dlamch('e') */
    parsec_context_t *parsec = dplasma_b200_init(0);
    if (!parsec) return 2;

    parsec_tiled_matrix_t A, A0, B, X;
    dplasma_b200_sym_desc_init(&A, PARSEC_MATRIX_DOUBLE, NB, NB, N, N, 0, 0, N, N, dplasmaLower);
    dplasma_b200_sym_desc_init(&A0, PARSEC_MATRIX_DOUBLE, NB, NB, N, N, 0, 0, N, N, dplasmaLower);
    dplasma_b200_desc_init(&B, PARSEC_MATRIX_DOUBLE, PARSEC_MATRIX_TILE, NB, NB, N, NRHS, 0, 0, N, NRHS);
    dplasma_b200_desc_init(&X, PARSEC_MATRIX_DOUBLE, PARSEC_MATRIX_TILE, NB, NB, N, NRHS, 0, 0, N, NRHS);
    const size_t na = A.bsiz * A.nb_local_tiles, nbb = B.bsiz * B.nb_local_tiles;
    A.mat = calloc(na, sizeof(double));
    A0.mat = calloc(na, sizeof(double));
    B.mat = calloc(nbb, sizeof(double));
    X.mat = calloc(nbb, sizeof(double));
    if (!A.mat || !A0.mat || !B.mat || !X.mat) return 3;

    if (dplasma_dplgsy(parsec, (double)N, dplasmaLower, &A0, 3872) != 0) return 4;
    if (dplasma_dplrnt(parsec, 0, &B, 2354) != 0) return 4;
    memcpy(A.mat, A0.mat, na * sizeof(double));
    memcpy(X.mat, B.mat, nbb * sizeof(double));
    int info = dplasma_dposv(parsec, dplasmaLower, &A, &X);
    if (info != 0) {
        fprintf(stderr, "dplasma_dposv: info %d (%s)\n", info, dplasma_b200_last_error(parsec));
        return 5;
    }

    /* check_daxmb: ||B - A X||_inf / ((||A||_inf ||X||_inf + ||B||_inf) N eps) */
    double anorm = 0.0, bnorm = 0.0, xnorm = 0.0, rnorm = 0.0;
    for (int i = 0; i < N; ++i) {
        double s = 0.0;
        for (int j = 0; j < N; ++j) s += fabs(get_sym(&A0, i, j));
        if (s > anorm) anorm = s;
    }
    for (int i = 0; i < N; ++i) {
        double sb = 0.0, sx = 0.0;
        for (int c = 0; c < NRHS; ++c) {
            sb += fabs(get_gen(&B, i, c));
            sx += fabs(get_gen(&X, i, c));
        }
        if (sb > bnorm) bnorm = sb;
        if (sx > xnorm) xnorm = sx;
    }
    double *ax = calloc((size_t)N * NRHS, sizeof(double));
    for (int j = 0; j < N; ++j)
        for (int c = 0; c < NRHS; ++c) {
            const double xj = get_gen(&X, j, c);
            for (int i = 0; i < N; ++i) ax[(size_t)c * N + i] += get_sym(&A0, i, j) * xj;
        }
    for (int i = 0; i < N; ++i) {
        double s = 0.0;
        for (int c = 0; c < NRHS; ++c) s += fabs(get_gen(&B, i, c) - ax[(size_t)c * N + i]);
        if (s > rnorm) rnorm = s;
    }
    const double r1 = rnorm / ((anorm * xnorm + bnorm) * N * eps);

    /* PDPOTRF on a column-major copy, submatrix at (1, 1), LLD = N + 3 */
    const int lld = N + 3;
    double *F = calloc((size_t)lld * N, sizeof(double));
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) F[(size_t)j * lld + i] = get_sym(&A0, i, j);
    int desca[9] = {1, 0, N, N, NB, NB, 0, 0, lld}, one = 1, n = N;
    pdpotrf_("L", &n, F, &one, &one, desca, &info);
    if (info != 0) {
        fprintf(stderr, "pdpotrf_: info %d\n", info);
        return 6;
    }
    /* check_dpotrf: ||L L^T - A||_inf / (||A||_inf N eps) */
    double dnorm = 0.0;
    for (int i = 0; i < N; ++i) {
        double s = 0.0;
        for (int j = 0; j < N; ++j) {
            const int kmax = i < j ? i : j;
            double v = 0.0;
            for (int k = 0; k <= kmax; ++k) v += F[(size_t)k * lld + i] * F[(size_t)k * lld + j];
            s += fabs(v - get_sym(&A0, i, j));
        }
        if (s > dnorm) dnorm = s;
    }
    const double r2 = dnorm / (anorm * N * eps);

    printf("dposv N=%d NB=%d NRHS=%d: check_daxmb ratio %.3f; pdpotrf_: check_dpotrf ratio %.3f\n", N, NB, NRHS,
           r1, r2);
    free(ax);
    free(F);
    free(A.mat);
    free(A0.mat);
    free(B.mat);
    free(X.mat);
    dplasma_b200_fini(&parsec);
    if (!(r1 < 10.0) || !(r2 < 10.0)) return 1;
    printf("ok\n");
    return 0;
}
