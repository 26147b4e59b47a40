"""GPU tests of the streamed mixed-precision solve: a host matrix in pinned
memory is copied in phases of tile columns while the factorization runs
(potrf_run_streamed: one launch over the phases' ticket orders; the first
task touching a tile column waits for that phase's arrival flag and reads the
untouched copy).  Every tile receives the same chunk updates in the same
order as in the factorization of an uploaded matrix, so the refinement takes
the same steps and the solution agrees with that of the same call on pageable
host memory (which uploads first) to the rounding of the residual products
(whose reductions across CTAs are unordered); both meet the check_zaxmb bar of
src/dplasma_zcheck.c."""
import os

import numpy as np
import pytest
import torch

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu


def _solve(ctx, A0, B0, NB, fmt, pinned):
    N, NRHS = B0.shape
    dA, dB, dX = db.desc_sym(N, NB, db.Lower), db.desc_general(N, NRHS, NB, NB), db.desc_general(N, NRHS, NB, NB)
    bufs = []
    for d, M in ((dA, A0), (dB, B0), (dX, np.zeros_like(B0))):
        host = db.pack(M, d)
        if pinned:
            t = torch.empty(host.size, dtype=torch.float64, pin_memory=True)
            t.copy_(torch.from_numpy(host))
            host = t.numpy()
            bufs.append(t)
        db.attach(d, host)
        bufs.append(host)
    rc, st = ctx.dsposv(db.Lower, dA, dB, dX, fmt=fmt)
    assert rc == 0, ctx.last_error()
    X = db.unpack(bufs[-1], dX)
    Aafter = db.unpack(bufs[-5] if pinned else bufs[0], dA)
    return X, st, Aafter


@pytest.mark.parametrize("N,fmt,cb", [(2048, db.FP16_SPLIT, 16), (8192, db.FP16_SPLIT, 16), (12288, db.FP16, 16),
                                      (6144, db.FP16_SPLIT, 8), (6144, db.BF16, 32)])
def test_streamed_solve_matches_uploaded(N, fmt, cb):
    NB, NRHS = 256, 8
    A0 = oracle.dplgsy(N, NB, 3872)
    B0 = oracle.dplrnt(N, NRHS, NB, NB, 3873)
    old = os.environ.get("DPLASMA_B200_STREAM_CB")
    os.environ["DPLASMA_B200_STREAM_CB"] = str(cb)
    try:
        with db.Context(0) as ctx:
            Xs, sts, As = _solve(ctx, A0, B0, NB, fmt, pinned=True)
            launches = ctx.last_launches()
            Xu, stu, _ = _solve(ctx, A0, B0, NB, fmt, pinned=False)
    finally:
        if old is None:
            del os.environ["DPLASMA_B200_STREAM_CB"]
        else:
            os.environ["DPLASMA_B200_STREAM_CB"] = old
    assert launches >= 2                           # the factorization and the refinement's kernels
    assert sts["iter"] == stu["iter"] and sts["fallback"] == stu["fallback"] == 0, (sts, stu)
    assert np.abs(Xs - Xu).max() <= 1e-13 * np.abs(Xu).max()
    keep = np.tril(np.ones((N, N), bool))
    assert np.array_equal(As[keep], A0[keep])          # A unchanged
    assert abs(sts["anorm"] - stu["anorm"]) <= 1e-13 * stu["anorm"]
    assert oracle.check_daxmb(oracle.LOWER, A0, B0, np.asfortranarray(Xs)) < 10.0


def test_streamed_not_positive_definite():
    N, NB = 4096, 256
    A0 = oracle.dplgsy(N, NB, 3872)
    A0[3000, 3000] = -1.0
    B0 = np.ones((N, 2))
    with db.Context(0) as ctx:
        dA, dB, dX = db.desc_sym(N, NB, db.Lower), db.desc_general(N, 2, NB, NB), db.desc_general(N, 2, NB, NB)
        ts = []
        for d, M in ((dA, A0), (dB, B0), (dX, np.zeros_like(B0))):
            t = torch.empty(db.desc_elems(d), dtype=torch.float64, pin_memory=True)
            t.copy_(torch.from_numpy(db.pack(M, d)))
            db.attach(d, t.numpy())
            ts.append(t)
        rc, st = ctx.dsposv(db.Lower, dA, dB, dX, fmt=db.FP16_SPLIT)
    Lo = A0.copy(order="F")
    info = oracle.dpotrf(oracle.LOWER, Lo, NB)
    assert info > 0 and rc == info
