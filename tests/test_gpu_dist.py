"""GPU tests of the task-insertion front-end (dplasma_b200_dtd_*,
dplasma_dpotrf_dtd: the counterpart of src/dtd_wrappers/zpotrf.c and
tests/testing_zpotrf_dtd.c) and of the column-cyclic multi-GPU factorization's
device path: P ranks' engines driven in lockstep from one process on one GPU
(each launch completes before the panel copy, so no kernel waits on another
rank), against the oracle."""
import numpy as np
import pytest
import torch

import oracle
import dplasma_b200 as db
from dplasma_b200 import dist as ddist

pytestmark = pytest.mark.gpu
FACTOR_TOL = 1e-12


def oracle_factor(A0, NB):
    L = A0.copy(order="F")
    info = oracle.dpotrf(oracle.LOWER, L, NB)
    return info, np.tril(L)


def rel(L, R):
    return np.linalg.norm(L - R) / np.linalg.norm(R)


@pytest.mark.parametrize("N,NB,device", [(2048, 256, True), (1536, 128, True), (1000, 200, False)])
def test_dpotrf_dtd_matches_oracle(gpu_ctx, N, NB, device):
    A0 = oracle.dplgsy(N, NB, 3872)
    d = db.desc_sym(N, NB, db.Lower)
    host = db.pack(A0, d)
    buf = torch.from_numpy(host.copy()).cuda() if device else host
    db.attach(d, buf)
    assert gpu_ctx.dpotrf_dtd(db.Lower, d) == 0, gpu_ctx.last_error()
    out = buf.cpu().numpy() if device else buf
    L = np.tril(db.unpack(out, d))
    _, Lo = oracle_factor(A0, NB)
    assert rel(L, Lo) <= FACTOR_TOL
    assert gpu_ctx.dpotrf_dtd(db.Upper, d) == db.ERR_NOT_SUPPORTED


def test_dtd_insertion_order_is_checked(gpu_ctx):
    N, NB = 1024, 256
    A0 = oracle.dplgsy(N, NB, 3872)
    d = db.desc_sym(N, NB, db.Lower)
    buf = torch.from_numpy(db.pack(A0, d)).cuda()
    db.attach(d, buf)
    tp = gpu_ctx.dtd(db.Lower, d)
    E = db.ERR_ILLEGAL_VALUE
    assert tp.insert(db.TASK_TRSM, 0, 1) == E             # before POTRF(0)
    assert tp.insert(db.TASK_POTRF, 1) == E               # tile (1,1) not updated by step 0
    assert tp.insert(db.TASK_POTRF, 0) == 0
    assert tp.insert(db.TASK_POTRF, 0) == E               # twice
    assert tp.insert(db.TASK_GEMM, 0, 2, 1) == E          # TRSM(1,0), TRSM(2,0) missing
    assert tp.insert(db.TASK_TRSM, 0, 1) == 0
    assert tp.insert(db.TASK_TRSM, 0, 2) == 0
    assert tp.insert(db.TASK_GEMM, 0, 1, 2) == E          # m > n required
    assert tp.insert(db.TASK_GEMM, 0, 2, 1) == 0
    assert tp.insert(db.TASK_GEMM, 0, 9, 1) == E          # out of range
    # a flush in the middle of the program: later tasks depend on earlier flushes
    assert tp.flush() == 0
    assert tp.insert(db.TASK_TRSM, 0, 3) == 0
    assert tp.insert(db.TASK_SYRK, 0, 1) == 0
    assert tp.insert(db.TASK_POTRF, 1) == 0
    assert tp.flush() == 0
    assert tp.tickets() > 0
    assert tp.destruct() == 0


def test_dtd_not_positive_definite(gpu_ctx):
    N, NB = 1024, 256
    A0 = oracle.dplgsy(N, NB, 3872)
    A0[600, 600] = -1.0
    info_o, _ = oracle_factor(A0, NB)
    d = db.desc_sym(N, NB, db.Lower)
    buf = torch.from_numpy(db.pack(A0, d)).cuda()
    db.attach(d, buf)
    assert gpu_ctx.dpotrf_dtd(db.Lower, d) == info_o == 601


def _lockstep(N, NB, P, A0):
    mt = N // NB
    ctxs, engines = [], []
    d = db.desc_sym(N, NB, db.Lower)
    full = db.pack(A0, d)
    t = NB * NB
    for r in range(P):
        ctx = db.Context(0)
        tiles = torch.zeros(db.desc_elems(d), dtype=torch.float64, device="cuda")
        for c in ddist.local_columns(mt, P, r):
            first, count = ddist.panel_tiles(mt, c)
            tiles[first * t:(first + count) * t] = torch.from_numpy(full[first * t:(first + count) * t])
        ctxs.append(ctx)
        engines.append(ddist.DeviceEngine(ctx, N, NB, tiles))
    info = ddist.run_lockstep(engines)
    # assemble the owned columns
    out = np.zeros_like(full)
    for r, e in enumerate(engines):
        h = e.tiles.cpu().numpy()
        for c in ddist.local_columns(mt, P, r):
            first, count = ddist.panel_tiles(mt, c)
            out[first * t:(first + count) * t] = h[first * t:(first + count) * t]
    for e in engines:
        e.close()
    for c in ctxs:
        c.close()
    return info, np.tril(db.unpack(out, d))


@pytest.mark.parametrize("N,NB,P", [(2048, 256, 2), (3072, 256, 3), (2048, 128, 4)])
def test_column_cyclic_lockstep_matches_oracle(N, NB, P):
    A0 = oracle.dplgsy(N, NB, 3872)
    info, L = _lockstep(N, NB, P, A0)
    assert info == 0
    _, Lo = oracle_factor(A0, NB)
    assert rel(L, Lo) <= FACTOR_TOL


def test_column_cyclic_lockstep_info():
    N, NB, P = 2048, 256, 2
    A0 = oracle.dplgsy(N, NB, 3872)
    A0[1300, 1300] = -1.0
    info_o, _ = oracle_factor(A0, NB)
    info, _ = _lockstep(N, NB, P, A0)
    assert info == info_o == 1301


@pytest.mark.parametrize("N,NB,hmb,uplo", [(2048, 512, 256, db.Lower), (1700, 400, 200, db.Lower),
                                            (1536, 512, 128, db.Upper)])
def test_dpotrf_rec_subtiles(gpu_ctx, N, NB, hmb, uplo):
    # the recursive variant runs the tasks on hmb sub-tiles: the tile
    # algorithm with tile edge hmb, checked against the oracle's with that edge
    A0 = oracle.dplgsy(N, NB, 3872)
    d = db.desc_sym(N, NB, uplo)
    buf = db.pack(A0, d)
    db.attach(d, buf)
    assert db.lib().dplasma_dpotrf_rec(gpu_ctx.h, uplo, d, hmb) == 0, gpu_ctx.last_error()
    out = db.unpack(buf, d)
    ouplo = oracle.LOWER if uplo == db.Lower else oracle.UPPER
    R = A0.copy(order="F")
    assert oracle.dpotrf(ouplo, R, hmb) == 0
    tri = np.tril if uplo == db.Lower else np.triu
    assert rel(tri(out), tri(R)) <= FACTOR_TOL
    # the other triangle of the diagonal tiles is left untouched
    mask = np.zeros((N, N), bool)
    for t in range(0, N, NB):
        e = min(N, t + NB)
        mask[t:e, t:e] = True
    other = np.triu(np.ones((N, N), bool), 1) if uplo == db.Lower else np.tril(np.ones((N, N), bool), -1)
    assert np.array_equal(out[mask & other], A0[mask & other])


def test_taskpool_setrecursive(gpu_ctx):
    import ctypes
    N, NB, hmb = 1024, 512, 256
    A0 = oracle.dplgsy(N, NB, 3872)
    A0[700, 700] = -1.0
    d = db.desc_sym(N, NB, db.Lower)
    buf = db.pack(A0, d)
    db.attach(d, buf)
    L = db.lib()
    info = ctypes.c_int(-1)
    tp = L.dplasma_dpotrf_New(db.Lower, ctypes.byref(d), ctypes.byref(info))
    L.dplasma_dpotrf_setrecursive(tp, hmb)
    assert L.dplasma_b200_taskpool_run(gpu_ctx.h, tp) == 0
    L.dplasma_dpotrf_Destruct(tp)
    R = A0.copy(order="F")
    assert info.value == oracle.dpotrf(oracle.LOWER, R, hmb) == 701
