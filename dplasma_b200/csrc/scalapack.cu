// scalapack.cu -- ScaLAPACK-compatible PDPOTRF, the entry point of the
// reference's src/scalapack_wrappers/dplasma_wrapper_pdpotrf.c:139-305
// (bound as pdpotrf_ by GENERATE_F77_BINDINGS, :297-303): an unmodified
// column-major application that links this library ahead of ScaLAPACK gets
// the GPU factorization.
//
// Here one process owns the whole matrix, i.e. a 1 x 1 process grid whose
// local array is the global one: the descriptor's source row and column must
// be 0 and its local leading dimension must cover the global rows.  The
// reference requires the submatrix to start on a block boundary (its
// assert at :217); PDPOTRF's argument checks report that as INFO = -4 / -5,
// which is what this entry returns.  The submatrix A(IA:IA+N-1, JA:JA+N-1)
// is factored through dplasma_dpotrf on a LAPACK-storage host descriptor
// (staged to the device tiles, factored, written back into the uplo
// triangle; the other triangle is not referenced).  INFO follows PDPOTRF:
// -(100*i + j) for entry j of array argument i, -i for scalar argument i,
// k > 0 when the leading minor of order k is not positive definite.
//
// The device is DPLASMA_B200_DEVICE (default 0); the context is created on
// the first call and released at process exit.  One host thread at a time.
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>

#include "dplasma_b200.h"

namespace {

// ScaLAPACK descriptor entries (0-based positions of DTYPE_ .. LLD_)
enum { D_DTYPE = 0, D_CTXT, D_M, D_N, D_MB, D_NB, D_RSRC, D_CSRC, D_LLD };

parsec_context_t *g_ctx = nullptr;

void release_context() { dplasma_b200_fini(&g_ctx); }

// argument checks of PDPOTRF (its CHK1MAT checks plus the block-alignment
// and square-block conditions), in the order ScaLAPACK reports them
int check_args(char u, int n, int ia, int ja, const int *desca)
{
    if (desca[D_DTYPE] != 1) return -(600 + D_DTYPE + 1);
    if (u != 'L' && u != 'U') return -1;
    if (n < 0) return -2;
    if (ia < 1) return -4;
    if (ja < 1) return -5;
    if (desca[D_M] < 0) return -(600 + D_M + 1);
    if (desca[D_N] < 0) return -(600 + D_N + 1);
    if (desca[D_MB] < 1) return -(600 + D_MB + 1);
    if (desca[D_NB] < 1) return -(600 + D_NB + 1);
    if (desca[D_RSRC] != 0) return -(600 + D_RSRC + 1);
    if (desca[D_CSRC] != 0) return -(600 + D_CSRC + 1);
    if (desca[D_LLD] < (desca[D_M] > 1 ? desca[D_M] : 1)) return -(600 + D_LLD + 1);
    if (ia + n - 1 > desca[D_M]) return -(600 + D_M + 1);
    if (ja + n - 1 > desca[D_N]) return -(600 + D_N + 1);
    if ((ia - 1) % desca[D_MB] != 0) return -4;
    if ((ja - 1) % desca[D_NB] != 0) return -5;
    if (desca[D_MB] != desca[D_NB]) return -(600 + D_NB + 1);
    return 0;
}

}  // namespace

extern "C" void pdpotrf_(const char *uplo, const int *n, double *a, const int *ia, const int *ja, const int *desca,
                         int *info)
{
    const char u = uplo ? (char)toupper((unsigned char)*uplo) : 0;
    *info = check_args(u, *n, *ia, *ja, desca);
    if (*info) {
        const int pos = *info < -99 ? (-*info) / 100 : -*info;
        fprintf(stderr, "{    0,    0}:  On entry to PDPOTRF parameter number %d had an illegal value\n", pos);
        return;
    }
    if (*n == 0) return;
    if (!g_ctx) {
        const char *dv = getenv("DPLASMA_B200_DEVICE");
        g_ctx = dplasma_b200_init(dv ? atoi(dv) : 0);
        if (!g_ctx) {
            *info = DPLASMA_ERR_NOT_INITIALIZED;
            return;
        }
        atexit(release_context);
    }
    const int lld = desca[D_LLD], nb = desca[D_NB];
    parsec_tiled_matrix_t d;
    dplasma_b200_desc_init(&d, PARSEC_MATRIX_DOUBLE, PARSEC_MATRIX_LAPACK, nb, nb, *n, *n, 0, 0, *n, *n);
    d.lda = lld;
    d.mat = a + (int64_t)(*ia - 1) + (int64_t)(*ja - 1) * lld;
    d.location = DPLASMA_B200_HOST;
    *info = dplasma_dpotrf(g_ctx, u == 'L' ? dplasmaLower : dplasmaUpper, &d);
}
