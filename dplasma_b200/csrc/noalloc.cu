// noalloc.cu -- dplasma_b200_dpotrf_noalloc: the tile Cholesky factorization
// of a matrix that already lives in device memory, for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is off limits -- a host
// process that hands the library memory from its own pool and must not let
// anything else grow the device heap (an allocator-controlled framework or a
// memory-capped service), or a caller holding a fixed device budget that
// cannot absorb the library's grow-on-demand workspace.  The regular entry
// points keep a per-context workspace that grows with cudaMalloc; this one
// takes its scratch (inverses of the diagonal blocks, scheduler counters,
// ticket order) from one file-scope device array instead.
//
// Limits and sharing:
//   * the matrix: device-resident, TILE storage of the lower triangle of
//     tiles (dplasma_b200_sym_desc_init with dplasmaLower), nb a multiple of
//     128 and at most 512, n a multiple of nb, and at most
//     NOALLOC_MAX_BLOCK_ROWS row blocks of 128 (n <= 8192);
//   * the array is sized for that maximum (about 8.4 MiB) and stays allocated
//     on every GPU that loads the library until the process exits;
//   * every call uses the same array and finds the previous call's contents:
//     the counters that must start at zero are cleared on the caller's stream
//     at the start of each call;
//   * calls are serialized inside the process: a host mutex is held for the
//     whole call, and the call returns only after its stream has finished the
//     factorization, so a second caller (another thread, another stream)
//     blocks until the first one's factorization is complete.  (Each process
//     has its own copy of the array, so processes sharing a GPU do not share
//     it.)  Nothing that goes through this entry point can race on it;
//   * the current device must be the device that holds A->mat and owns
//     `stream`; a mismatch is rejected before anything is launched;
//   * the call cannot be recorded into a CUDA graph: it copies the ticket
//     order from host memory and waits for its stream, which a stream
//     capture forbids, so it returns DPLASMA_ERR_NOT_SUPPORTED when `stream`
//     is capturing;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it;
//   * dependency and pipeline waits are bounded by DPLASMA_B200_WAIT_LIMIT_MS
//     (milliseconds, default 4000), the setting of the regular entry points.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#include <mutex>

#include "internal.h"
#include "potrf_kernel.cuh"

namespace db2 {
size_t potrf_smem_bytes();
int potrf_max_blocks_per_sm();
size_t build_potrf_tasks_into(uint64_t *out, size_t cap, int mt, int nbs, int delay);
int potrf_launch_prealloc(cudaStream_t st, double *dA, int mt, int nbi, int nb_user, int n_user, double *W,
                          const uint64_t *tasks, int ntasks, int *ctr, int grid, uint64_t limit_ns, int *info,
                          int *status, int diag[4]);
}  // namespace db2

using namespace db2;

namespace {

constexpr int NOALLOC_MAX_BLOCK_ROWS = 64;    // mt * nb/128 <= 64: n <= 8192
constexpr int NOALLOC_MAX_MT = 64;
constexpr int NOALLOC_MAX_TASKS = 49152;      // >= tickets of every allowed shape
constexpr size_t W_BYTES = (size_t)NOALLOC_MAX_BLOCK_ROWS * 128 * 128 * sizeof(double);   // 8 MiB
constexpr size_t TASK_BYTES = (size_t)NOALLOC_MAX_TASKS * sizeof(uint64_t);               // 384 KiB
constexpr size_t CTR_INTS = 8 + NOALLOC_MAX_MT + 2 * (size_t)NOALLOC_MAX_MT * NOALLOC_MAX_MT;
constexpr size_t CTR_BYTES = ((CTR_INTS * sizeof(int) + 255) / 256) * 256;
constexpr size_t SCRATCH_BYTES = W_BYTES + TASK_BYTES + CTR_BYTES;
constexpr int MAX_DEVICES = 64;

// Host order of the ticket list is built here before the copy (no heap use).
uint64_t g_host_tasks[NOALLOC_MAX_TASKS];
std::mutex g_lock;
void *g_scratch_addr[MAX_DEVICES] = {};

}  // namespace

// The scratch itself.  In host code this name is only a handle for
// cudaGetSymbolAddress; its device address is what the kernel receives.
static __device__ __align__(256) unsigned char g_potrf_scratch[SCRATCH_BYTES];

extern "C" int dplasma_b200_dpotrf_noalloc(void *stream, dplasma_enum_t uplo, parsec_tiled_matrix_t *A)
{
    if (uplo != dplasmaLower) {
        fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] uplo must be dplasmaLower\n");
        return uplo == dplasmaUpper ? DPLASMA_ERR_NOT_SUPPORTED : -1;
    }
    if (!A || A->mtype != PARSEC_MATRIX_DOUBLE || A->location != DPLASMA_B200_DEVICE ||
        A->storage != PARSEC_MATRIX_TILE || A->uplo != dplasmaLower || A->m != A->n || A->mb != A->nb ||
        A->i != 0 || A->j != 0 || (A->m > 0 && !A->mat)) {
        fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] needs a device-resident lower symmetric TILE descriptor\n");
        return DPLASMA_ERR_ILLEGAL_VALUE;
    }
    const int n = A->m, nb = A->mb;
    if (n == 0) return 0;
    if (nb % 128 != 0 || nb > 512 || n % nb != 0 || A->lmt != n / nb) {
        fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] nb must be a multiple of 128 (<= 512) dividing n\n");
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    const int mt = n / nb, nbs = nb / 128;
    if ((size_t)mt * nbs > (size_t)NOALLOC_MAX_BLOCK_ROWS) {
        fprintf(stderr,
                "[dplasma_b200_dpotrf_noalloc] n=%d exceeds the fixed scratch (at most %d rows, %zu bytes); "
                "use dplasma_dpotrf\n",
                n, NOALLOC_MAX_BLOCK_ROWS * 128, SCRATCH_BYTES);
        return DPLASMA_ERR_INTERNAL_LIMIT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return DPLASMA_ERR_UNEXPECTED;
    // the matrix and the stream must belong to the current device
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, A->mat) != cudaSuccess || pa.type != cudaMemoryTypeDevice || pa.device != dev) {
        cudaGetLastError();
        fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] A->mat is not device memory of the current device %d\n", dev);
        return DPLASMA_ERR_ILLEGAL_VALUE;
    }
    if (st) {
        int sdev = -1;
        if (cudaStreamGetDevice(st, &sdev) != cudaSuccess || sdev != dev) {
            cudaGetLastError();
            fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] the stream does not belong to the current device %d\n", dev);
            return DPLASMA_ERR_ILLEGAL_VALUE;
        }
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] cannot run under stream capture\n");
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    const char *lim = getenv("DPLASMA_B200_WAIT_LIMIT_MS");
    const long lim_ms = lim ? atol(lim) : 4000;
    const uint64_t limit_ns = (uint64_t)(lim_ms > 0 ? lim_ms : 4000) * 1000000ull;

    std::lock_guard<std::mutex> guard(g_lock);
    // one-time set-up on this device: the device address of the scratch array
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_potrf_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            cudaGetLastError();
            return DPLASMA_ERR_UNEXPECTED;
        }
        g_scratch_addr[dev] = p;
    }
    unsigned char *base = (unsigned char *)g_scratch_addr[dev];
    double *W = (double *)base;
    uint64_t *tasks = (uint64_t *)(base + W_BYTES);
    int *ctr = (int *)(base + W_BYTES + TASK_BYTES);

    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int occ = potrf_max_blocks_per_sm();
    if (occ < 1 || sms < 1) return DPLASMA_ERR_UNEXPECTED;
    const int grid = sms * occ;
    const size_t ntasks = build_potrf_tasks_into(g_host_tasks, NOALLOC_MAX_TASKS, mt, nbs, 3 * grid);
    if (ntasks == 0) {
        fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] ticket list exceeds the fixed scratch\n");
        return DPLASMA_ERR_INTERNAL_LIMIT;
    }
    // counters start at zero; the ticket order is rewritten every call
    const size_t nctr = 8 + (size_t)mt + 2 * (size_t)mt * mt;
    if (cudaMemsetAsync(ctr, 0, nctr * sizeof(int), st) != cudaSuccess ||
        cudaMemcpyAsync(tasks, g_host_tasks, ntasks * sizeof(uint64_t), cudaMemcpyHostToDevice, st) != cudaSuccess) {
        cudaGetLastError();
        return DPLASMA_ERR_UNEXPECTED;
    }
    int info = 0, status = 0, diag[4] = {0, 0, 0, 0};
    const int rc = potrf_launch_prealloc(st, (double *)A->mat, mt, nb, nb, n, W, tasks, (int)ntasks, ctr, grid,
                                         limit_ns, &info, &status, diag);
    if (rc) return rc;
    if (status != 0) {
        fprintf(stderr, "[dplasma_b200_dpotrf_noalloc] scheduler status %d (site %d)\n", status, diag[0]);
        return DPLASMA_ERR_UNEXPECTED;
    }
    return info;
}
