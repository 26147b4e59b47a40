"""GPU tests of dplasma_dlange and dplasma_dsymm, the calls the reference's
residual check check_zaxmb makes (src/dplasma_zcheck.c:179-224), against numpy
and the oracle's check_daxmb."""
import numpy as np
import pytest

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,MB,NB,storage", [(1000, 37, 256, 256, db.STORAGE_TILE),
                                               (300, 300, 128, 64, db.STORAGE_TILE),
                                               (777, 5, 100, 100, db.STORAGE_LAPACK)])
def test_dlange_norms(gpu_ctx, M, N, MB, NB, storage):
    X = np.random.default_rng(M).standard_normal((M, N))
    d = db.desc_general(M, N, MB, NB, storage=storage, lda=M + 3 if storage == db.STORAGE_LAPACK else None)
    buf = db.pack(X, d)
    db.attach(d, buf)
    assert abs(gpu_ctx.dlange(db.InfNorm, d) - np.abs(X).sum(1).max()) <= 1e-13 * np.abs(X).sum(1).max()
    assert abs(gpu_ctx.dlange(db.OneNorm, d) - np.abs(X).sum(0).max()) <= 1e-13 * np.abs(X).sum(0).max()
    assert gpu_ctx.dlange(db.MaxNorm, d) == np.abs(X).max()
    assert abs(gpu_ctx.dlange(db.FrobeniusNorm, d) - np.linalg.norm(X)) <= 1e-13 * np.linalg.norm(X)
    assert gpu_ctx.dlange(db.UpperLower, d) < 0          # not a norm type


@pytest.mark.parametrize("N,NB,NRHS,uplo,alpha,beta", [(1000, 256, 16, db.Lower, -1.0, 1.0),
                                                       (700, 200, 3, db.Upper, 0.5, -2.0),
                                                       (513, 256, 1, db.Lower, 1.0, 0.0)])
def test_dsymm_left(gpu_ctx, N, NB, NRHS, uplo, alpha, beta):
    rng = np.random.default_rng(N)
    A = oracle.dplgsy(N, NB, 3872)
    B = rng.standard_normal((N, NRHS))
    C = rng.standard_normal((N, NRHS))
    dA = db.desc_sym(N, NB, uplo)
    bA = db.pack(A, dA)
    db.attach(dA, bA)
    dB = db.desc_general(N, NRHS, NB, NB)
    bB = db.pack(B, dB)
    db.attach(dB, bB)
    dC = db.desc_general(N, NRHS, 128, 128)       # C tiled differently from A
    bC = db.pack(C, dC)
    db.attach(dC, bC)
    assert gpu_ctx.dsymm(db.Left, uplo, alpha, dA, dB, beta, dC) == 0, gpu_ctx.last_error()
    ref = alpha * A @ B + beta * C
    got = db.unpack(bC, dC)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_dsymm_argument_checks(gpu_ctx):
    N = 300
    dA = db.desc_sym(N, 256, db.Lower)
    bA = np.zeros(db.desc_elems(dA))
    db.attach(dA, bA)
    dB = db.desc_general(N, 2, 256, 256)
    bB = np.zeros(db.desc_elems(dB))
    db.attach(dB, bB)
    dC = db.desc_general(N + 1, 2, 256, 256)
    bC = np.zeros(db.desc_elems(dC))
    db.attach(dC, bC)
    assert gpu_ctx.dsymm(0, db.Lower, 1.0, dA, dB, 0.0, dB) == -1
    assert gpu_ctx.dsymm(db.Left, 0, 1.0, dA, dB, 0.0, dB) == -2
    assert gpu_ctx.dsymm(db.Left, db.Lower, 1.0, dA, dB, 0.0, dC) == -5
    # right side: A's order must match C's columns (-6, src/zsymm_wrapper.c), then not provided
    assert gpu_ctx.dsymm(db.Right, db.Lower, 1.0, dA, dB, 0.0, dB) == -6
    dR = db.desc_general(2, N, 256, 256)
    bR = np.zeros(db.desc_elems(dR))
    db.attach(dR, bR)
    assert gpu_ctx.dsymm(db.Right, db.Lower, 1.0, dA, dR, 0.0, dR) == db.ERR_NOT_SUPPORTED


@pytest.mark.parametrize("noise,tol", [(1e-10, 1e-4), (1e-14, 0.5)])
def test_gpu_check_daxmb_matches_oracle(gpu_ctx, noise, tol):
    # noise 1e-10: a residual far above the rounding of the product, so both
    # checks must agree closely; 1e-14: a residual at the rounding level, where
    # the two summation orders may differ by a fair fraction of it
    N, NB, NRHS = 1500, 256, 16
    A = oracle.dplgsy(N, NB, 3872)
    B = oracle.dplrnt(N, NRHS, NB, NB, 3873)
    X = np.linalg.solve(A, B)
    X = X * (1.0 + noise * np.random.default_rng(1).standard_normal(X.shape))
    dA = db.desc_sym(N, NB, db.Lower)
    bA = db.pack(A, dA)
    db.attach(dA, bA)
    descs = []
    for M in (B, X, B):
        d = db.desc_general(N, NRHS, NB, NB)
        b = db.pack(M, d)
        db.attach(d, b)
        descs.append((d, b))
    ratio = gpu_ctx.check_daxmb(db.Lower, dA, descs[0][0], descs[1][0], descs[2][0])
    ref = oracle.check_daxmb(oracle.LOWER, A, B, np.asfortranarray(X))
    assert abs(ratio - ref) <= tol * ref, (ratio, ref)
