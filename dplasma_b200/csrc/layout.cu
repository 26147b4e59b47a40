// layout.cu -- moves matrices between the caller's descriptor layout (TILE
// or LAPACK storage, host or device) and the device tile layout the kernels
// use, and the seeded generators dplasma_dplgsy / dplasma_dplrnt.
#include <cuda_runtime.h>
#include <string.h>

#include "dev_common.cuh"
#include "internal.h"

namespace db2 {

Geom make_geom(int n, int nb)
{
    Geom g;
    g.n = n;
    g.nb = nb;
    g.nbi = ((nb + 127) / 128) * 128;
    g.mt = (n + nb - 1) / nb;
    return g;
}

// ---------------------------------------------------------------------------
// caller layout description, usable on the device
// ---------------------------------------------------------------------------
struct DescView {
    double *mat;
    int storage;   // PARSEC_MATRIX_TILE / PARSEC_MATRIX_LAPACK
    int sym;       // 0 whole grid, 1 lower tiles packed, 2 upper tiles packed
    int mb, nb, lmt, lda;
    int m, n, mt, nt;
    int64_t bsiz;
};

static DescView view_of(const parsec_tiled_matrix_t *A, double *mat)
{
    DescView v;
    v.mat = mat;
    v.storage = A->storage;
    v.sym = (A->storage == PARSEC_MATRIX_TILE) ? (A->uplo == dplasmaLower ? 1 : (A->uplo == dplasmaUpper ? 2 : 0)) : 0;
    v.mb = A->mb;
    v.nb = A->nb;
    v.lmt = A->lmt;
    v.lda = A->lda;
    v.m = A->m;
    v.n = A->n;
    v.mt = A->mt;
    v.nt = A->nt;
    v.bsiz = (int64_t)A->bsiz;
    return v;
}

__host__ __device__ __forceinline__ int64_t view_tile_offset(const DescView &v, int m, int n)
{
    if (v.storage == PARSEC_MATRIX_LAPACK) return (int64_t)m * v.mb + (int64_t)n * v.nb * v.lda;
    if (v.sym == 1) return (m < n) ? -1 : ((int64_t)n * v.lmt - ((int64_t)n * (n - 1)) / 2 + (m - n)) * v.bsiz;
    if (v.sym == 2) return (m > n) ? -1 : (((int64_t)n * (n + 1)) / 2 + m) * v.bsiz;
    return ((int64_t)m + (int64_t)n * v.lmt) * v.bsiz;
}
__host__ __device__ __forceinline__ int view_ld(const DescView &v) { return v.storage == PARSEC_MATRIX_LAPACK ? v.lda : v.mb; }

int64_t tile_offset(const parsec_tiled_matrix_t *A, int m, int n)
{
    DescView v = view_of(A, nullptr);
    return view_tile_offset(v, m, n);
}

size_t desc_elems(const parsec_tiled_matrix_t *A)
{
    if (A->storage == PARSEC_MATRIX_LAPACK) return (size_t)A->lda * (size_t)A->ln;
    return A->bsiz * A->nb_local_tiles;
}

// Element (r,c) of internal tile `idx` = (m,n), m >= n.  Thread block per tile.
__device__ __forceinline__ void tile_of_index(int64_t idx, int mt, int &m, int &n)
{
    // column n holds mt - n tiles
    int nn = 0;
    int64_t rem = idx;
    // binary search on the column start offset
    int lo = 0, hi = mt - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        int64_t start = (int64_t)mid * mt - ((int64_t)mid * (mid - 1)) / 2;
        if (start <= idx) lo = mid; else hi = mid - 1;
    }
    nn = lo;
    rem = idx - ((int64_t)nn * mt - ((int64_t)nn * (nn - 1)) / 2);
    n = nn;
    m = nn + (int)rem;
}

__global__ void to_internal_kernel(DescView src, int uplo_upper, int n_user, int nb, int nbi, int mt, double *dA)
{
    int m, n;
    tile_of_index(blockIdx.x, mt, m, n);
    double *T = dA + (int64_t)blockIdx.x * nbi * nbi;
    const int tm = (m == mt - 1) ? n_user - m * nb : nb;
    const int tn = (n == mt - 1) ? n_user - n * nb : nb;
    const int ld = view_ld(src);
    const int64_t off = uplo_upper ? view_tile_offset(src, n, m) : view_tile_offset(src, m, n);
    const double *S = src.mat + off;
    for (int e = threadIdx.x; e < nbi * nbi; e += blockDim.x) {
        const int r = e % nbi, c = e / nbi;
        double v;
        if (r < tm && c < tn)
            v = uplo_upper ? S[(int64_t)r * ld + c] : S[(int64_t)c * ld + r];
        else
            v = (m == n && r == c) ? 1.0 : 0.0;
        T[e] = v;
    }
}

__global__ void from_internal_kernel(DescView dst, int uplo_upper, int n_user, int nb, int nbi, int mt, const double *dA)
{
    int m, n;
    tile_of_index(blockIdx.x, mt, m, n);
    const double *T = dA + (int64_t)blockIdx.x * nbi * nbi;
    const int tm = (m == mt - 1) ? n_user - m * nb : nb;
    const int tn = (n == mt - 1) ? n_user - n * nb : nb;
    const int ld = view_ld(dst);
    const int64_t off = uplo_upper ? view_tile_offset(dst, n, m) : view_tile_offset(dst, m, n);
    double *D = dst.mat + off;
    for (int e = threadIdx.x; e < nbi * nbi; e += blockDim.x) {
        const int r = e % nbi, c = e / nbi;
        if (r < tm && c < tn) {
            if (uplo_upper)
                D[(int64_t)r * ld + c] = T[e];
            else
                D[(int64_t)c * ld + r] = T[e];
        }
    }
}

// Internal tiles of a different edge than the caller's (the recursive
// variant's sub-tiles): element by element.  Internal tile (m,n) element
// (r,c) is matrix element (i,j) = (m nb + r, n nb + c); only i >= j is moved
// (the stored triangle), the rest of a diagonal tile is zero and the padding
// the identity.
__global__ void to_internal_retile_kernel(DescView src, int uplo_upper, int n_user, int nb, int nbi, int mt,
                                          double *dA)
{
    int m, n;
    tile_of_index(blockIdx.x, mt, m, n);
    double *T = dA + (int64_t)blockIdx.x * nbi * nbi;
    const int tm = (m == mt - 1) ? n_user - m * nb : nb;
    const int tn = (n == mt - 1) ? n_user - n * nb : nb;
    const int ld = view_ld(src);
    for (int e = threadIdx.x; e < nbi * nbi; e += blockDim.x) {
        const int r = e % nbi, c = e / nbi;
        const int64_t i = (int64_t)m * nb + r, j = (int64_t)n * nb + c;
        double v;
        if (r < tm && c < tn) {
            if (i < j) {
                v = 0.0;
            } else {
                // lower storage holds (i, j); upper storage its mirror (j, i)
                const int64_t a = uplo_upper ? j : i, b = uplo_upper ? i : j;
                v = src.mat[view_tile_offset(src, (int)(a / src.mb), (int)(b / src.nb)) + (a % src.mb) +
                            (b % src.nb) * ld];
            }
        } else {
            v = (m == n && r == c) ? 1.0 : 0.0;
        }
        T[e] = v;
    }
}

__global__ void from_internal_retile_kernel(DescView dst, int uplo_upper, int n_user, int nb, int nbi, int mt,
                                            const double *dA)
{
    int m, n;
    tile_of_index(blockIdx.x, mt, m, n);
    const double *T = dA + (int64_t)blockIdx.x * nbi * nbi;
    const int tm = (m == mt - 1) ? n_user - m * nb : nb;
    const int tn = (n == mt - 1) ? n_user - n * nb : nb;
    const int ld = view_ld(dst);
    for (int e = threadIdx.x; e < nbi * nbi; e += blockDim.x) {
        const int r = e % nbi, c = e / nbi;
        const int64_t i = (int64_t)m * nb + r, j = (int64_t)n * nb + c;
        if (r < tm && c < tn && i >= j) {
            const int64_t a = uplo_upper ? j : i, b = uplo_upper ? i : j;
            dst.mat[view_tile_offset(dst, (int)(a / dst.mb), (int)(b / dst.nb)) + (a % dst.mb) + (b % dst.nb) * ld] =
                T[e];
        }
    }
}

static bool fast_path(const parsec_tiled_matrix_t *A, dplasma_enum_t uplo, const Geom &g)
{
    return A->storage == PARSEC_MATRIX_TILE && A->uplo == dplasmaLower && uplo == dplasmaLower &&
           g.nbi == g.nb && (g.n % g.nb) == 0 && A->lmt == g.mt && A->mb == A->nb;
}

int upload_sym(Context *ctx, const parsec_tiled_matrix_t *A, dplasma_enum_t uplo, const Geom &g, double *dA)
{
    cudaStream_t st = ctx->stream;
    const size_t bytes = desc_elems(A) * sizeof(double);
    if (fast_path(A, uplo, g)) {
        CK(cudaMemcpyAsync(dA, A->mat, g.elems() * sizeof(double),
                           A->location == DPLASMA_B200_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
        return 0;
    }
    double *src = (double *)A->mat;
    if (A->location != DPLASMA_B200_DEVICE) {
        src = (double *)ctx->buffer(BUF_STAGE, bytes);
        if (!src) return DPLASMA_ERR_OUT_OF_RESOURCES;
        CK(cudaMemcpyAsync(src, A->mat, bytes, cudaMemcpyHostToDevice, st));
    }
    DescView v = view_of(A, src);
    if (g.nb != A->mb)
        to_internal_retile_kernel<<<(unsigned)g.ntiles(), 256, 0, st>>>(v, uplo == dplasmaUpper, g.n, g.nb, g.nbi,
                                                                        g.mt, dA);
    else
        to_internal_kernel<<<(unsigned)g.ntiles(), 256, 0, st>>>(v, uplo == dplasmaUpper, g.n, g.nb, g.nbi, g.mt, dA);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

int download_sym(Context *ctx, parsec_tiled_matrix_t *A, dplasma_enum_t uplo, const Geom &g, const double *dA)
{
    cudaStream_t st = ctx->stream;
    const size_t bytes = desc_elems(A) * sizeof(double);
    if (fast_path(A, uplo, g)) {
        CK(cudaMemcpyAsync(A->mat, dA, g.elems() * sizeof(double),
                           A->location == DPLASMA_B200_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return 0;
    }
    double *dst = (double *)A->mat;
    if (A->location != DPLASMA_B200_DEVICE) dst = (double *)ctx->buffer(BUF_STAGE, 0);   // filled by upload_sym
    DescView v = view_of(A, dst);
    if (g.nb != A->mb)
        from_internal_retile_kernel<<<(unsigned)g.ntiles(), 256, 0, st>>>(v, uplo == dplasmaUpper, g.n, g.nb, g.nbi,
                                                                          g.mt, dA);
    else
        from_internal_kernel<<<(unsigned)g.ntiles(), 256, 0, st>>>(v, uplo == dplasmaUpper, g.n, g.nb, g.nbi, g.mt,
                                                                   dA);
    CK(cudaGetLastError());
    ctx->launches++;
    if (A->location != DPLASMA_B200_DEVICE) CK(cudaMemcpyAsync(A->mat, dst, bytes, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

// ---------------------------------------------------------------------------
// right-hand sides: caller N x NRHS matrix <-> padded column-major npad x nrhs
// ---------------------------------------------------------------------------
// Device right-hand sides live in the padded row space of the tiles: row
// m*nbi + r holds global row m*nb + r for r < (rows of tile m), zero otherwise.
__global__ void rhs_in_kernel(DescView src, int nb, int nbi, int npad, int nrhs, double *dB)
{
    const int64_t total = (int64_t)npad * nrhs;
    const int ld = view_ld(src);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int ip = (int)(e % npad), j = (int)(e / npad);
        const int t = ip / nbi, r = ip % nbi;
        const int64_t i = (int64_t)t * nb + r;
        double v = 0.0;
        if (r < nb && i < src.m && j < src.n) {
            const int64_t off = view_tile_offset(src, (int)(i / src.mb), j / src.nb);
            v = src.mat[off + (i % src.mb) + (int64_t)(j % src.nb) * ld];
        }
        dB[e] = v;
    }
}
__global__ void rhs_out_kernel(DescView dst, int nb, int nbi, int npad, int nrhs, const double *dB)
{
    const int64_t total = (int64_t)npad * nrhs;
    const int ld = view_ld(dst);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int ip = (int)(e % npad), j = (int)(e / npad);
        const int t = ip / nbi, r = ip % nbi;
        const int64_t i = (int64_t)t * nb + r;
        if (r < nb && i < dst.m && j < dst.n) {
            const int64_t off = view_tile_offset(dst, (int)(i / dst.mb), j / dst.nb);
            dst.mat[off + (i % dst.mb) + (int64_t)(j % dst.nb) * ld] = dB[e];
        }
    }
}

int upload_rhs(Context *ctx, const parsec_tiled_matrix_t *B, int nb, int nbi, int npad, int nrhs, double *dB)
{
    cudaStream_t st = ctx->stream;
    double *src = (double *)B->mat;
    if (B->location != DPLASMA_B200_DEVICE) {
        const size_t bytes = desc_elems(B) * sizeof(double);
        src = (double *)ctx->buffer(BUF_BSTAGE, bytes);
        if (!src) return DPLASMA_ERR_OUT_OF_RESOURCES;
        CK(cudaMemcpyAsync(src, B->mat, bytes, cudaMemcpyHostToDevice, st));
    }
    DescView v = view_of(B, src);
    rhs_in_kernel<<<ctx->sms * 4, 256, 0, st>>>(v, nb, nbi, npad, nrhs, dB);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

int download_rhs(Context *ctx, parsec_tiled_matrix_t *B, int nb, int nbi, int npad, int nrhs, const double *dB)
{
    cudaStream_t st = ctx->stream;
    double *dst = (B->location != DPLASMA_B200_DEVICE) ? (double *)ctx->buffer(BUF_BSTAGE, desc_elems(B) * sizeof(double))
                                                       : (double *)B->mat;
    if (!dst) return DPLASMA_ERR_OUT_OF_RESOURCES;
    DescView v = view_of(B, dst);
    rhs_out_kernel<<<ctx->sms * 4, 256, 0, st>>>(v, nb, nbi, npad, nrhs, dB);
    CK(cudaGetLastError());
    ctx->launches++;
    if (B->location != DPLASMA_B200_DEVICE)
        CK(cudaMemcpyAsync(B->mat, dst, desc_elems(B) * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

// ---------------------------------------------------------------------------
// Generators.  64-bit LCG with jump-ahead (src/cores/random.h:19-41); each
// value is formed in single precision, `0.5f - ran * RndF_Mul`
// (src/cores/core_zplgsy.c:89), with the conversion, multiply and subtract
// each rounded to nearest (no contraction), then stored as double.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t rnd64_jump(uint64_t n, uint64_t seed)
{
    uint64_t a_k = 6364136223846793005ULL, c_k = 1ULL, ran = seed;
    while (n) {
        if (n & 1ULL) ran = a_k * ran + c_k;
        c_k *= (a_k + 1ULL);
        a_k *= a_k;
        n >>= 1;
    }
    return ran;
}
__device__ __forceinline__ uint64_t rnd64_next(uint64_t ran) { return 6364136223846793005ULL * ran + 1ULL; }
__device__ __forceinline__ double rnd_value(uint64_t ran)
{
    const float r = __ull2float_rn(ran);
    const float p = __fmul_rn(r, 5.4210108624275222e-20f);
    return (double)__fsub_rn(0.5f, p);
}

constexpr int GEN_CHUNK = 32;

// One thread per (tile column, chunk of GEN_CHUNK rows) of every generated
// tile.  sym != 0: symmetric (dplgsy), value(i,j) from jump max(i,j) +
// min(i,j)*gM, bump on the diagonal.  sym == 0: general (dplrnt), value(i,j)
// from jump i + j*gM, `bump` added on the local diagonal of tiles (m,m).
__global__ void gen_kernel(DescView d, int sym, int region, double bump, uint64_t seed, int gM)
{
    const int ext = max(d.mb, d.nb);
    const int chunks = (ext + GEN_CHUNK - 1) / GEN_CHUNK;
    const int64_t per_tile = (int64_t)chunks * ext;
    const int64_t total = per_tile * d.mt * d.nt;
    const int ld = view_ld(d);
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total; w += (int64_t)gridDim.x * blockDim.x) {
        const int64_t tile = w / per_tile;
        const int rem = (int)(w % per_tile);
        const int a = rem / chunks, ch = rem % chunks;
        const int m = (int)(tile % d.mt), n = (int)(tile / d.mt);
        if (region == dplasmaLower && m < n) continue;
        if (region == dplasmaUpper && m > n) continue;
        const int tm = (m == d.mt - 1) ? d.m - m * d.mb : d.mb;
        const int tn = (n == d.nt - 1) ? d.n - n * d.nb : d.nb;
        const int64_t off = view_tile_offset(d, m, n);
        if (off < 0) continue;
        double *T = d.mat + off;
        const int64_t i0 = (int64_t)m * d.mb, j0 = (int64_t)n * d.nb;
        if (sym && i0 + tm <= j0) {
            // tile strictly above the diagonal: value(i,j) = LCG at j + i*gM,
            // consecutive along a row -> walk row `a`, columns of chunk ch
            const int r = a, c0 = ch * GEN_CHUNK;
            if (r >= tm || c0 >= tn) continue;
            const int c1 = min(tn, c0 + GEN_CHUNK);
            uint64_t ran = rnd64_jump((uint64_t)(j0 + c0) + (uint64_t)(i0 + r) * (uint64_t)gM, seed);
            for (int c = c0; c < c1; ++c) {
                T[r + (int64_t)c * ld] = rnd_value(ran);
                ran = rnd64_next(ran);
            }
            continue;
        }
        const int c = a, r0 = ch * GEN_CHUNK;
        if (c >= tn || r0 >= tm) continue;
        const int r1 = min(tm, r0 + GEN_CHUNK);
        double *col = T + (int64_t)c * ld;
        const int64_t j = j0 + c;
        if (!sym) {
            uint64_t ran = rnd64_jump((uint64_t)(i0 + r0) + (uint64_t)j * (uint64_t)gM, seed);
            for (int r = r0; r < r1; ++r) {
                double v = rnd_value(ran);
                if (m == n && r == c) v += bump;
                col[r] = v;
                ran = rnd64_next(ran);
            }
        } else {
            // rows above the diagonal: mirrored values, one jump each
            int r = r0;
            for (; r < r1 && i0 + r < j; ++r)
                col[r] = rnd_value(rnd64_jump((uint64_t)j + (uint64_t)(i0 + r) * (uint64_t)gM, seed));
            if (r < r1) {
                uint64_t ran = rnd64_jump((uint64_t)(i0 + r) + (uint64_t)j * (uint64_t)gM, seed);
                for (; r < r1; ++r) {
                    double v = rnd_value(ran);
                    if (i0 + r == j) v += bump;
                    col[r] = v;
                    ran = rnd64_next(ran);
                }
            }
        }
    }
}

static bool generates_everything(const parsec_tiled_matrix_t *A, int region)
{
    if (A->storage != PARSEC_MATRIX_TILE) return false;
    if (region == dplasmaUpperLower) return A->uplo == dplasmaUpperLower || A->uplo == dplasmaLower || A->uplo == dplasmaUpper;
    return A->uplo == region;
}

static int run_generator(Context *ctx, parsec_tiled_matrix_t *A, int sym, int region, double bump, unsigned long long seed)
{
    cudaStream_t st = ctx->stream;
    const size_t bytes = desc_elems(A) * sizeof(double);
    double *dst = (double *)A->mat;
    if (A->location != DPLASMA_B200_DEVICE) {
        dst = (double *)ctx->buffer(BUF_STAGE, bytes);
        if (!dst) return DPLASMA_ERR_OUT_OF_RESOURCES;
        if (!generates_everything(A, region)) CK(cudaMemcpyAsync(dst, A->mat, bytes, cudaMemcpyHostToDevice, st));
    }
    DescView v = view_of(A, dst);
    gen_kernel<<<ctx->sms * 8, 256, 0, st>>>(v, sym, region, bump, seed, A->m);
    CK(cudaGetLastError());
    ctx->launches++;
    if (A->location != DPLASMA_B200_DEVICE) CK(cudaMemcpyAsync(A->mat, dst, bytes, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

int generate_plgsy(Context *ctx, double bump, dplasma_enum_t uplo, parsec_tiled_matrix_t *A, unsigned long long seed)
{
    return run_generator(ctx, A, 1, uplo, bump, seed);
}

int generate_plrnt(Context *ctx, int diagdom, parsec_tiled_matrix_t *A, unsigned long long seed)
{
    const double alpha = diagdom ? (double)(A->m > A->n ? A->m : A->n) : 0.0;
    return run_generator(ctx, A, 0, dplasmaUpperLower, alpha, seed);
}

}  // namespace db2
