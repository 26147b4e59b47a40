/*
 * dplasma_b200.h -- C ABI of the B200-native tile Cholesky library.
 *
 * A drop-in for DPLASMA's Cholesky factor-and-solve path on a 1x1 process
 * grid: the entry points below keep the names, argument meaning, enum values
 * and return conventions of the dplasma C API they replace (each is cited
 * with the reference file:line it mirrors; paths are relative to the dplasma
 * source tree).  Signatures use only plain C types and pointers.
 *
 * Matrices are described by a parsec_tiled_matrix_t-shaped descriptor (the
 * reference type lives in PaRSEC; its field names and the meaning of each are
 * kept, the struct layout is this library's own).  `mat` points either to
 * host memory (the default, as in the reference, where the caller allocates
 * and owns it) or, when `location == DPLASMA_B200_DEVICE`, to device memory
 * on the context's GPU.  Calls are blocking and in place: results are in
 * `mat` when they return.
 */
#ifndef DPLASMA_B200_H
#define DPLASMA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- constants: src/include/dplasma/constants.h:32-42, 47, 78-99 -------- */
#define DPLASMA_SUCCESS                 0
#define DPLASMA_ERR_NOT_INITIALIZED  -101
#define DPLASMA_ERR_REINITIALIZED    -102
#define DPLASMA_ERR_NOT_SUPPORTED    -103
#define DPLASMA_ERR_ILLEGAL_VALUE    -104
#define DPLASMA_ERR_NOT_FOUND        -105
#define DPLASMA_ERR_OUT_OF_RESOURCES -106
#define DPLASMA_ERR_INTERNAL_LIMIT   -107
#define DPLASMA_ERR_UNALLOCATED      -108
#define DPLASMA_ERR_FILESYSTEM       -109
#define DPLASMA_ERR_UNEXPECTED       -110
#define DPLASMA_ERR_SEQUENCE_FLUSHED -111

typedef int dplasma_enum_t;

#define dplasmaNoTrans       111
#define dplasmaTrans         112
#define dplasmaConjTrans     113
#define dplasmaUpper         121
#define dplasmaLower         122
#define dplasmaUpperLower    123
#define dplasmaNonUnit       131
#define dplasmaUnit          132
#define dplasmaLeft          141
#define dplasmaRight         142
#define dplasmaOneNorm       171
#define dplasmaFrobeniusNorm 174
#define dplasmaInfNorm       175
#define dplasmaMaxNorm       177

/* ---- matrix descriptor -------------------------------------------------- */
/* Element types (the PaRSEC matrix-type enumeration: byte, int, float,
 * double, complex float, complex double).  Only DOUBLE is on this path. */
#define PARSEC_MATRIX_BYTE           0
#define PARSEC_MATRIX_INTEGER        1
#define PARSEC_MATRIX_FLOAT          2
#define PARSEC_MATRIX_DOUBLE         3
#define PARSEC_MATRIX_COMPLEX_FLOAT  4
#define PARSEC_MATRIX_COMPLEX_DOUBLE 5

/* Storage kinds (src/utils/dplasma_lapack_adtt.h:29-31 names them TILED and
 * LAPACK).  TILE: every tile is a contiguous mb*nb column-major block with
 * leading dimension mb, the last tile row/column padded to full size.
 * LAPACK: one column-major array with leading dimension `lda`. */
#define PARSEC_MATRIX_LAPACK 0
#define PARSEC_MATRIX_TILE   1

/* Where `mat` lives. */
#define DPLASMA_B200_HOST   0
#define DPLASMA_B200_DEVICE 1

typedef struct parsec_tiled_matrix_s {
    int mtype;            /* PARSEC_MATRIX_DOUBLE                                    */
    int storage;          /* PARSEC_MATRIX_TILE or PARSEC_MATRIX_LAPACK              */
    int uplo;             /* tiles held in TILE storage: dplasmaUpperLower (whole
                             grid), dplasmaLower / dplasmaUpper (symmetric storage,
                             only that triangle of tiles)                            */
    int mb, nb;           /* tile size                                               */
    int lm, ln;           /* size of the allocated matrix                            */
    int i, j;             /* first row/column of this (sub)matrix: 0 only            */
    int m, n;             /* size of the matrix                                      */
    int mt, nt;           /* tile rows / columns of the matrix                       */
    int lmt, lnt;         /* tile rows / columns of the allocation                   */
    int lda;              /* leading dimension (LAPACK storage)                      */
    int location;         /* DPLASMA_B200_HOST or DPLASMA_B200_DEVICE                */
    size_t bsiz;          /* elements per tile (mb*nb)                               */
    size_t nb_local_tiles;/* tiles in the allocation                                 */
    void *mat;            /* caller-owned data                                       */
} parsec_tiled_matrix_t;

/* Tile (m,n) of a TILE-storage descriptor starts at element
 * dplasma_b200_tile_offset(A, m, n) of `mat`:
 *   uplo == dplasmaUpperLower: tiles column-major over the lmt x lnt grid,
 *                              offset = (m + n*lmt) * bsiz;
 *   uplo == dplasmaLower:      only m >= n tiles, packed column by column,
 *                              offset = (n*lmt - n*(n-1)/2 + (m-n)) * bsiz;
 *   uplo == dplasmaUpper:      only m <= n tiles, packed column by column,
 *                              offset = (n*(n+1)/2 + m) * bsiz.
 * For LAPACK storage it is m*mb + n*nb*lda.  Returns -1 for a tile outside
 * the stored triangle. */
int64_t dplasma_b200_tile_offset(const parsec_tiled_matrix_t *A, int m, int n);

/* Fill a descriptor for a general (two-dimensional block-cyclic, 1x1 grid)
 * matrix; mirrors parsec_matrix_block_cyclic_init's size arguments
 * (as called in tests/testing_zposv.c:40-51).  `mat` is left NULL; the
 * number of elements to allocate is bsiz * nb_local_tiles (TILE) or
 * lda * n (LAPACK). */
void dplasma_b200_desc_init(parsec_tiled_matrix_t *A, int mtype, int storage,
                            int mb, int nb, int lm, int ln, int i, int j, int m, int n);
/* Same for symmetric TILE storage of one triangle of tiles; mirrors
 * parsec_matrix_sym_block_cyclic_init (tests/testing_zpotrf.c:42-45). */
void dplasma_b200_sym_desc_init(parsec_tiled_matrix_t *A, int mtype, int mb, int nb,
                                int lm, int ln, int i, int j, int m, int n, dplasma_enum_t uplo);

/* ---- context ------------------------------------------------------------ */
/* Replaces the parsec_context_t the dplasma calls take (created by
 * parsec_init, tests/common.c:684).  One context owns one GPU, a CUDA stream
 * and the device workspace; it is used from one host thread at a time. */
typedef struct parsec_context_s parsec_context_t;
typedef struct parsec_taskpool_s parsec_taskpool_t;

parsec_context_t *dplasma_b200_init(int device);
void dplasma_b200_fini(parsec_context_t **ctx);
/* Last error message of this context (empty when none). */
const char *dplasma_b200_last_error(const parsec_context_t *ctx);

/* ---- the Cholesky path -------------------------------------------------- */
/* dplasma_dpotrf: src/zpotrf_wrapper.c:345-371 (declared at
 * src/include/dplasma/dplasma_z.h:82).  Returns 0, -1 for a bad uplo, or
 * i > 0 when the leading minor of order i is not positive definite
 * (k*NB + iinfo, src/zpotrf_L.jdf:200-202). */
int dplasma_dpotrf(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A);

/* dplasma_dpotrf_New / _Destruct: src/zpotrf_wrapper.c:193-258, 280-297
 * (dplasma_z.h:172, 239).  New returns NULL on a bad uplo; the factorization
 * runs when the taskpool is executed by dplasma_b200_taskpool_run (the
 * analogue of parsec_context_add_taskpool + dplasma_wait_until_completion),
 * and *info receives the INFO value. */
parsec_taskpool_t *dplasma_dpotrf_New(dplasma_enum_t uplo, parsec_tiled_matrix_t *A, int *info);
void dplasma_dpotrf_Destruct(parsec_taskpool_t *tp);
int dplasma_b200_taskpool_run(parsec_context_t *parsec, parsec_taskpool_t *tp);

/* dplasma_dpotrf_rec / _setrecursive: src/zpotrf_wrapper.c:425-451
 * (dplasma_z.h:83, 273).  With 0 < hmb < NB the tasks of the factorization
 * run on hmb x hmb sub-tiles (the reference's recursive bodies split each NB
 * tile task into a sub-DAG on hmb tiles, src/zpotrf_L.jdf:168-192; together
 * they are the tile algorithm with tile edge hmb); the caller's NB tiles are
 * copied to and from that layout.  Otherwise the same as dplasma_dpotrf.
 * _setrecursive sets hmb for a taskpool made by dplasma_dpotrf_New. */
int dplasma_dpotrf_rec(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A, int hmb);
void dplasma_dpotrf_setrecursive(parsec_taskpool_t *tp, int hmb);

/* dplasma_dpotrs: src/zpotrs_wrapper.c:56-97 (dplasma_z.h:84).  A holds the
 * factor from dplasma_dpotrf, B (N x NRHS) is overwritten by the solution.
 * Returns 0 or -1 for a bad uplo. */
int dplasma_dpotrs(parsec_context_t *parsec, dplasma_enum_t uplo, const parsec_tiled_matrix_t *A,
                   parsec_tiled_matrix_t *B);

/* dplasma_dposv: src/zposv_wrapper.c:63-113 (dplasma_z.h:81).  Factor, then
 * solve when INFO == 0; returns INFO. */
int dplasma_dposv(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A,
                  parsec_tiled_matrix_t *B);

/* dplasma_dtrsm: src/ztrsm_wrapper.c:263-309 (dplasma_z.h:51).  Left side
 * only (the four sweeps src/ztrsm_L{LN,LT,UN,UT}.jdf); side == dplasmaRight
 * returns DPLASMA_ERR_NOT_SUPPORTED.  -1..-4 bad enums, -6 bad shapes. */
int dplasma_dtrsm(parsec_context_t *parsec, dplasma_enum_t side, dplasma_enum_t uplo,
                  dplasma_enum_t trans, dplasma_enum_t diag, double alpha,
                  const parsec_tiled_matrix_t *A, parsec_tiled_matrix_t *B);

/* Generators.  dplasma_dplgsy: src/zplgsy_wrapper.c:185-215 with
 * CORE_dplgsy (src/cores/core_zplgsy.c:72-150); dplasma_dplrnt:
 * src/zplrnt_wrapper.c (CORE_dplrnt, src/cores/core_zplrnt.c:68-91)
 * (dplasma_z.h:108-109).  Bit-identical values.  Return 0 or -i for a bad
 * argument i. */
int dplasma_dplgsy(parsec_context_t *parsec, double bump, dplasma_enum_t uplo,
                   parsec_tiled_matrix_t *A, unsigned long long int seed);
int dplasma_dplrnt(parsec_context_t *parsec, int diagdom, parsec_tiled_matrix_t *A,
                   unsigned long long int seed);

/* Infinity norm of a symmetric matrix stored by its `uplo` triangle
 * (dplasma_dlansy with dplasmaInfNorm, dplasma_z.h:101), computed on the GPU;
 * returns a negative value for an unsupported norm or descriptor. */
double dplasma_dlansy(parsec_context_t *parsec, dplasma_enum_t ntype, dplasma_enum_t uplo,
                      const parsec_tiled_matrix_t *A);

/* ---- task insertion (the DTD front-end) ---------------------------------- */
/* The counterpart of dplasma's DTD Cholesky (src/dtd_wrappers/zpotrf.c and
 * the insertion loop of tests/testing_zpotrf_dtd.c:125-200): the caller
 * inserts the tile tasks of a lower Cholesky in a sequential program order and
 * flushes; each flush runs the tasks inserted since the last one as one
 * launch of the device scheduler, in insertion order, with dependency
 * counters that persist across flushes.  An insertion whose dependencies have
 * not all been inserted before it is refused (DPLASMA_ERR_ILLEGAL_VALUE), so
 * every flush completes.  A: lower descriptor (device-resident lower TILE
 * storage with nb a multiple of 128 dividing n is used in place; any other
 * layout is copied to the device by _new and written back by
 * _data_flush_all).  Tasks (indices of tiles):
 *   POTRF k       A(k,k) = chol(A(k,k))
 *   TRSM  k, m    A(m,k) = A(m,k) A(k,k)^-T            m > k
 *   SYRK  k, m    A(m,m) -= A(m,k) A(m,k)^T             m > k
 *   GEMM  k, m, n A(m,n) -= A(m,k) A(n,k)^T             m > n > k */
#define DPLASMA_B200_TASK_POTRF 1
#define DPLASMA_B200_TASK_TRSM  2
#define DPLASMA_B200_TASK_SYRK  3
#define DPLASMA_B200_TASK_GEMM  4
typedef struct dplasma_b200_dtd_s dplasma_b200_dtd_t;
dplasma_b200_dtd_t *dplasma_b200_dtd_new(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A);
/* Insert one task (m, n ignored where the task has no such index). */
int dplasma_b200_dtd_insert(dplasma_b200_dtd_t *tp, int op, int k, int m, int n);
/* Tile column k was factored elsewhere (POTRF(k) and TRSM(:,k) by another
 * process) and its tiles copied into this matrix: later tasks may use it. */
int dplasma_b200_dtd_panel_received(dplasma_b200_dtd_t *tp, int k);
/* Run the pending tasks and wait: 0, INFO > 0, or a negative code. */
int dplasma_b200_dtd_flush(dplasma_b200_dtd_t *tp);
/* Flush, then write the tiles back to A when the pool works on a copy
 * (parsec_dtd_data_flush_all). */
int dplasma_b200_dtd_data_flush_all(dplasma_b200_dtd_t *tp);
/* Device address of the tile storage the pool works on (lower tiles packed
 * by columns, tile edge nb rounded up to a multiple of 128). */
void *dplasma_b200_dtd_tiles(dplasma_b200_dtd_t *tp);
/* Tickets (scheduler tasks) launched so far. */
long long dplasma_b200_dtd_tickets(const dplasma_b200_dtd_t *tp);
/* Free the pool; returns its INFO (or its first error). */
int dplasma_b200_dtd_destruct(dplasma_b200_dtd_t *tp);
/* dplasma_dpotrf through the task-insertion front-end (the reference's
 * testing_zpotrf_dtd flow): inserts POTRF, TRSM, SYRK, GEMM of every step in
 * the reference's order and flushes once.  Lower only (dplasmaUpper:
 * DPLASMA_ERR_NOT_SUPPORTED).  Returns INFO as dplasma_dpotrf. */
int dplasma_dpotrf_dtd(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A);

/* dplasma_dlange: src/zlange_wrapper.c (dplasma_z.h:98).  dplasmaInfNorm,
 * OneNorm, MaxNorm or FrobeniusNorm of a general matrix, computed on the GPU;
 * returns a negative value for an unsupported norm or descriptor. */
double dplasma_dlange(parsec_context_t *parsec, dplasma_enum_t ntype, const parsec_tiled_matrix_t *A);

/* dplasma_dsymm: src/zsymm_wrapper.c (dplasma_z.h:40), the product of the
 * reference's residual check (src/dplasma_zcheck.c:196-197).  C = alpha A B +
 * beta C, A symmetric given by its uplo triangle.  Left side only
 * (dplasmaRight: DPLASMA_ERR_NOT_SUPPORTED); A's tile size in 129..256, B
 * and C of any tiling.  Returns 0, -1 / -2 for a bad side / uplo,
 * -4 / -5 / -6 for bad shapes, or a negative code. */
int dplasma_dsymm(parsec_context_t *parsec, dplasma_enum_t side, dplasma_enum_t uplo, double alpha,
                  const parsec_tiled_matrix_t *A, const parsec_tiled_matrix_t *B, double beta,
                  parsec_tiled_matrix_t *C);

/* dplasma_b200_dpotrf_noalloc: no counterpart in the reference.  The lower
 * tile Cholesky of a device-resident matrix (TILE storage of the lower
 * triangle of tiles, nb a multiple of 128 and at most 512, n a multiple of nb,
 * n <= 8192) for callers that cannot allocate device memory, e.g. code that
 * hands the library memory from its own pool and may not let the device heap
 * grow.  It allocates nothing: its scratch is one fixed array of about
 * 8.4 MiB in the library's device image, held on every GPU that loads the
 * library until exit; larger n is rejected with DPLASMA_ERR_INTERNAL_LIMIT.
 * Runs on `stream` (a cudaStream_t, or NULL for the default stream); the
 * current device must hold A->mat and own the stream (else
 * DPLASMA_ERR_ILLEGAL_VALUE).  Returns INFO as dplasma_dpotrf does.  Calls in
 * one process are serialized: a host mutex is held and the call returns once
 * its stream has finished, so they never overlap on the shared scratch.  The
 * call waits for its stream and copies from host memory, so it cannot run
 * under stream capture (DPLASMA_ERR_NOT_SUPPORTED).  The first call on a
 * device looks up the scratch's device address.  Waits are bounded by
 * DPLASMA_B200_WAIT_LIMIT_MS as in the other entry points. */
int dplasma_b200_dpotrf_noalloc(void *stream, dplasma_enum_t uplo, parsec_tiled_matrix_t *A);

/* ---- mixed precision ---------------------------------------------------- */
/* Type of the tensor-core operands of the trailing updates. */
#define DPLASMA_B200_FP16 0
#define DPLASMA_B200_BF16 1
/* Each panel value as the sum of two FP16 numbers (hi + lo); three products
 * per update (hi*hi + hi*lo + lo*hi, the split-FP16 method of Ootomo and
 * Yokota, 2022) give about 22 bits: for condition numbers near 1e6, where a
 * single 16-bit factorization can lose positive definiteness. */
#define DPLASMA_B200_FP16_SPLIT 2
/* Correction solver of the refinement. */
#define DPLASMA_B200_IR_AUTO  0   /* plain refinement, GMRES-IR once it stops contracting */
#define DPLASMA_B200_IR_PLAIN 1   /* x += L^-T L^-1 r */
#define DPLASMA_B200_IR_GMRES 2   /* GMRES on L^-T L^-1 A d = L^-T L^-1 r */

typedef struct dplasma_b200_refine_opts_s {
    int    fmt;        /* DPLASMA_B200_FP16, DPLASMA_B200_BF16 or DPLASMA_B200_FP16_SPLIT */
    int    solver;     /* DPLASMA_B200_IR_* */
    int    itermax;    /* refinement iterations before the FP64 fallback (LAPACK dsposv ITERMAX = 30) */
    int    gmres_m;    /* largest Krylov dimension of one GMRES-IR correction */
    double gmres_tol;  /* residual reduction asked of one GMRES-IR correction */
    double bwdmax;     /* LAPACK dsposv BWDMAX: stop when ||r_j|| < ||x_j|| ||A|| eps sqrt(n) bwdmax */
    int    escalate;   /* 1: when an FP16/BF16 factorization loses positive definiteness, retry in
                          the split-FP16 form before the FP64 fallback */
    double shift;      /* s >= 0: the 16-bit factorization is of A + s diag(A) (the shifted, diagonally
                          scaled factor of Higham and Pranesh, SISC 2021), kept positive definite at
                          large condition numbers; the refinement solves A.  0: no shift */
} dplasma_b200_refine_opts_t;

typedef struct dplasma_b200_refine_stats_s {
    int    iter;           /* LAPACK dsposv ITER: refinement steps, or -3 (low-precision factorization
                              failed) / -(itermax+1) (no convergence): FP64 factorization used */
    int    inner_iters;    /* GMRES iterations over all corrections */
    int    fallback;       /* 1 when the FP64 factorization produced the solution */
    int    solver_used;    /* highest DPLASMA_B200_IR_* used (1 plain, 2 GMRES) */
    int    fmt_used;       /* operand form of the factor that was refined (-1: FP64 fallback) */
    double backward_error; /* max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf) */
    double factor_ms;      /* device time of the mixed factorization (with its working copy) */
    double refine_ms;      /* device time of the solves and refinement (and of a fallback) */
    double anorm;          /* ||A||_inf of the FP64 matrix, the scale of the stopping test */
} dplasma_b200_refine_stats_t;

/* Defaults: FP16, IR_AUTO, itermax 30, gmres_m 30, gmres_tol 1e-4, bwdmax 1, escalate 1, shift 0. */
void dplasma_b200_refine_opts_default(dplasma_b200_refine_opts_t *opts);

/* dplasma_b200_dplgsy_cond: no dplasma counterpart; a test-matrix generator
 * beside dplasma_dplgsy for the mixed-precision solve.  Fills the symmetric
 * matrix A = Q diag(sigma) Q^T, Q the product of `nrefl` Householder
 * reflectors of random unit vectors drawn from `seed`, sigma geometric from
 * 1 (first row) to kappa (last row), so that cond_2(A) = kappa.  Built on the
 * GPU in FP64 by nrefl two-sided rank-2 updates.  A: N x N, tile nb with
 * 128 < nb <= 256, `uplo` triangle written.  Returns 0 or a negative code. */
int dplasma_b200_dplgsy_cond(parsec_context_t *parsec, double kappa, int nrefl, dplasma_enum_t uplo,
                             parsec_tiled_matrix_t *A, unsigned long long int seed);

/* dplasma_dsposv: no dplasma counterpart; the argument meaning of LAPACK
 * dsposv (LAPACKE_dsposv, src/include/lapacke.h:2987 of the reference).
 * Solves A X = B for symmetric positive definite A with a factorization whose
 * trailing updates run on the FP16 tensor cores, refined in FP64 to the
 * dsposv accuracy, falling back to the FP64 factorization after 30
 * non-converging steps.  A (N x N, tile nb with 128 < nb <= 256) is unchanged
 * unless the fallback ran, in which case it holds the FP64 factor, as in
 * dsposv; B is unchanged; X (N x NRHS, same tiling as B) receives the
 * solution.  *iter as dsposv ITER.  Returns 0, INFO > 0 when A is not
 * positive definite, or a negative code. */
int dplasma_dsposv(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A,
                   const parsec_tiled_matrix_t *B, parsec_tiled_matrix_t *X, int *iter);

/* dplasma_dsposv with explicit options (NULL: defaults) and statistics
 * (may be NULL). */
int dplasma_b200_dsposv_ex(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A,
                           const parsec_tiled_matrix_t *B, parsec_tiled_matrix_t *X,
                           const dplasma_b200_refine_opts_t *opts, dplasma_b200_refine_stats_t *stats);

/* ---- inverses (the next path after potrf/potrs) --------------------------- */
/* dplasma_dtrtri: src/ztrtri_wrapper.c (dplasma_z.h:86).  In place inverse of
 * the uplo triangle; diag dplasmaUnit takes the diagonal as 1.  Returns 0,
 * -1 / -2 for a bad uplo / diag, or INFO = i when A(i,i) is exactly zero
 * (A untouched then). */
int dplasma_dtrtri(parsec_context_t *parsec, dplasma_enum_t uplo, dplasma_enum_t diag, parsec_tiled_matrix_t *A);
/* dplasma_dlauum: src/zlauum_wrapper.c (dplasma_z.h:78).  L^T L (uplo Lower)
 * or U U^T (Upper) of the triangle, in place. */
int dplasma_dlauum(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A);
/* dplasma_dpotri: src/zpotri_wrapper.c (dplasma_z.h:85).  A holds the factor
 * from dplasma_dpotrf; on return its uplo triangle holds A^-1 (trtri then
 * lauum).  Returns trtri's INFO. */
int dplasma_dpotri(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A);
/* dplasma_dpoinv / _sync: src/zpoinv_wrapper.c (dplasma_z.h:79-80).  potrf then
 * potri: the uplo triangle of SPD A is replaced by that of A^-1; returns INFO. */
int dplasma_dpoinv(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A);
int dplasma_dpoinv_sync(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A);

/* ---- adjoint ------------------------------------------------------------ */
/* dplasma_dpotrf_adjoint: no dplasma counterpart; the reverse-mode derivative
 * of dplasma_dpotrf.  L holds the factor of A = L L^T (uplo Lower) or
 * A = U^T U (uplo Upper: the Upper triangle holds U = L^T), as dplasma_dpotrf
 * leaves it; Lbar holds dF/dL (resp. dF/dU) of a scalar F in the same
 * triangle and is overwritten there by the symmetric dF/dA,
 *     Abar = sym( L^-T Phi(L^T Lbar) L^-1 ),  Phi = lower triangle, diagonal halved.
 * The log-determinant adjoint is the case Lbar = diag(2 dF/dlogdet / L(i,i))
 * (Abar = dF/dlogdet * A^-1); the adjoint of x = A^-1 b is
 * Abar = -sym(bbar x^T) with bbar = A^-1 xbar, a dplasma_dpotrs.  Same tile
 * sizes and storages as dplasma_dpotrf.  Returns 0 or a negative code. */
int dplasma_dpotrf_adjoint(parsec_context_t *parsec, dplasma_enum_t uplo, const parsec_tiled_matrix_t *L,
                           parsec_tiled_matrix_t *Lbar);

/* ---- batched ------------------------------------------------------------ */
/* dplasma_b200_dposv_batched / _sposv_batched: no dplasma counterpart.  Factor
 * (Cholesky, lower), solve and log-determinant of `batch` independent SPD
 * systems A_i X_i = B_i of orders n[i] (0 <= n[i] <= 512 in FP64, 1024 in
 * FP32), in one persistent launch replayed from a CUDA graph.  Every array
 * argument is DEVICE memory: n, lda (int[batch]); A (pointers to the
 * column-major n[i] x n[i] matrices, lower triangle read, overwritten by
 * L_i); B (pointers to the n[i] x nrhs right-hand sides, leading dimension
 * n[i], overwritten by X_i; B itself or B[i] may be NULL to factor only);
 * logdet (double[batch], 2 sum log L_i(j,j); NaN when INFO > 0; may be
 * NULL); info (int[batch], LAPACK INFO of each problem).  The first call for
 * a size class (largest n up to the next power of two) times the kernel
 * variants on the caller's batch and keeps the fastest.  Returns 0 or a
 * negative code. */
int dplasma_b200_dposv_batched(parsec_context_t *parsec, int batch, const int *n, const int *lda,
                               double *const *A, double *const *B, int nrhs, double *logdet, int *info);
int dplasma_b200_sposv_batched(parsec_context_t *parsec, int batch, const int *n, const int *lda,
                               float *const *A, float *const *B, int nrhs, double *logdet, int *info);
/* dplasma_b200_dpotri_batched: no dplasma counterpart; dplasma_dpotri for a
 * batch.  A[i] holds the lower factor L_i (as dplasma_b200_dposv_batched
 * leaves it); on return its lower triangle holds A_i^-1.  info[i] as
 * dplasma_dpotri.  All arrays in device memory; one persistent launch. */
int dplasma_b200_dpotri_batched(parsec_context_t *parsec, int batch, const int *n, const int *lda,
                                double *const *A, int *info);
/* Name of the kernel variant the last batched call used (autotuner choice). */
const char *dplasma_b200_batched_variant(const parsec_context_t *parsec);

/* ---- ScaLAPACK-compatible entry ------------------------------------------ */
/* pdpotrf_: src/scalapack_wrappers/dplasma_wrapper_pdpotrf.c:139-305 (the
 * Fortran binding pdpotrf_ of GENERATE_F77_BINDINGS, :297-303); ScaLAPACK's
 * PDPOTRF(UPLO, N, A, IA, JA, DESCA, INFO).  DESCA is the 9-integer
 * ScaLAPACK descriptor {DTYPE=1, CTXT, M, N, MB, NB, RSRC, CSRC, LLD}; one
 * process owns the whole matrix (a 1 x 1 grid: RSRC = CSRC = 0, LLD >= M).
 * The column-major submatrix A(IA:IA+N-1, JA:JA+N-1) (1-based, starting on
 * a block boundary, MB = NB) is factored in place on the GPU.  INFO = 0,
 * -(100*i+j) / -i for an illegal entry j of array argument i / scalar
 * argument i, k > 0 when the leading minor of order k is not positive
 * definite, DPLASMA_ERR_NOT_INITIALIZED without a usable GPU.  Device:
 * DPLASMA_B200_DEVICE (default 0), context kept until process exit. */
void pdpotrf_(const char *uplo, const int *n, double *a, const int *ia, const int *ja, const int *desca,
              int *info);

/* ---- instrumentation ---------------------------------------------------- */
/* Device time in milliseconds of the last factorization (CUDA events around
 * the scheduler launch only) and of the last triangular-solve pair. */
double dplasma_b200_last_factor_ms(const parsec_context_t *ctx);
double dplasma_b200_last_solve_ms(const parsec_context_t *ctx);
/* Number of kernel launches issued by the last public call. */
int dplasma_b200_last_launches(const parsec_context_t *ctx);

/* ---- failure detection --------------------------------------------------- */
/* Every wait inside the device scheduler is bounded: a dependency wait gives
 * up after `dep_ms`, a pipeline wait after `pipe_ms` milliseconds (default
 * DPLASMA_B200_WAIT_LIMIT_MS, 4000); the kernel then stops every CTA and the
 * call returns DPLASMA_ERR_UNEXPECTED with the site, CTA and ticket in
 * dplasma_b200_last_error.  The context stays usable. */
int dplasma_b200_set_wait_limits(parsec_context_t *ctx, int dep_ms, int pipe_ms);
/* Host-side fault injection for the next factorization of this context (the
 * reference's failure paths -- PARSEC_HOOK_RETURN_ERROR from a task body,
 * src/zpotrf_L.jdf:136,261,390,530 -- made testable without faulting a GPU):
 *   DPLASMA_B200_INJECT_TASK_FAILED, arg k: POTRF(k) reports failure when it
 *     is fetched; the scheduler stops and the call returns
 *     DPLASMA_ERR_UNEXPECTED ("task reported failed");
 *   DPLASMA_B200_INJECT_WITHHOLD, arg i: ticket i of the ticket order is taken
 *     but neither run nor released, so the tasks that depend on it wait until
 *     the dependency-wait limit and the call returns DPLASMA_ERR_UNEXPECTED
 *     ("dependency wait timed out", site recorded).
 * The injection is consumed by that one call.  Returns 0 or
 * DPLASMA_ERR_ILLEGAL_VALUE. */
#define DPLASMA_B200_INJECT_NONE        0
#define DPLASMA_B200_INJECT_TASK_FAILED 1
#define DPLASMA_B200_INJECT_WITHHOLD    2
int dplasma_b200_inject_fault(parsec_context_t *ctx, int kind, int arg);
/* Scheduler self check (also DPLASMA_B200_SELFCHECK=1 at dplasma_b200_init):
 * every factorization counts the runs of each ticket on the device and the
 * call fails with DPLASMA_ERR_UNEXPECTED unless each ran exactly once.
 * dplasma_b200_selfcheck reports the last factorization's tickets, task runs
 * and tickets that did not run exactly once; it returns
 * DPLASMA_ERR_NOT_INITIALIZED when the check is off. */
int dplasma_b200_set_selfcheck(parsec_context_t *ctx, int on);
int dplasma_b200_selfcheck(const parsec_context_t *ctx, long long *tickets, long long *runs, long long *bad);

/* Measured FP64 tensor-core (DMMA) throughput of this GPU in TFLOP/s: a
 * register-only mma.sync.m16n8k4.f64 loop on every SM, timed with CUDA
 * events.  The roofline denominator for the FP64 kernels. */
double dplasma_b200_fp64_peak_tflops(parsec_context_t *ctx);

#ifdef __cplusplus
}
#endif

#endif /* DPLASMA_B200_H */
