"""GPU tests of the inverse routines next to the Cholesky path:
dplasma_dtrtri, dplasma_dlauum, dplasma_dpotri, dplasma_dpoinv (the
reference's src/ztrtri_wrapper.c, src/zlauum_wrapper.c, src/zpotri_wrapper.c,
src/zpoinv_wrapper.c), checked by the reference's own check_zpoinv ratio
||I - A^-1 A||_1 / (||A||_1 ||A^-1||_1 N eps) < 10 (src/dplasma_zcheck.c:264-314)
and against numpy on the triangular pieces."""
import numpy as np
import pytest

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu
EPS = 2.0 ** -53


def sym_full(T, uplo):
    tri = np.tril(T) if uplo == db.Lower else np.triu(T)
    return tri + tri.T - np.diag(np.diag(tri))


def packed(A0, NB, uplo):
    d = db.desc_sym(A0.shape[0], NB, uplo)
    buf = db.pack(A0, d)
    db.attach(d, buf)
    return d, buf


@pytest.mark.parametrize("N,NB,uplo", [(378, 93, db.Lower), (1000, 256, db.Lower), (700, 128, db.Upper),
                                       (1, 1, db.Lower), (513, 256, db.Upper)])
def test_dpoinv_check_zpoinv(gpu_ctx, N, NB, uplo):
    A = oracle.dplgsy(N, NB, 3872, bump=float(N))
    d, buf = packed(A, NB, uplo)
    assert gpu_ctx.dpoinv(uplo, d) == 0, gpu_ctx.last_error()
    Ainv = sym_full(db.unpack(buf, d), uplo)
    R = np.eye(N) - Ainv @ A
    n1 = lambda X: np.abs(X).sum(0).max()
    ratio = n1(R) / (n1(A) * n1(Ainv) * N * EPS)
    assert ratio < 10, ratio


def test_dpotri_after_dpotrf(gpu_ctx):
    N, NB = 600, 128
    A = oracle.dplgsy(N, NB, 3872, bump=float(N))
    d, buf = packed(A, NB, db.Lower)
    assert gpu_ctx.dpotrf(db.Lower, d) == 0
    assert gpu_ctx.dpotri(db.Lower, d) == 0
    Ainv = sym_full(db.unpack(buf, d), db.Lower)
    assert np.linalg.norm(Ainv - np.linalg.inv(A)) / np.linalg.norm(np.linalg.inv(A)) < 1e-12


@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
@pytest.mark.parametrize("diag", [db.NonUnit, db.Unit])
def test_dtrtri_and_dlauum(gpu_ctx, uplo, diag):
    N, NB = 300, 128
    rng = np.random.default_rng(4)
    L = np.tril(rng.uniform(-0.5, 0.5, (N, N))) + 4.0 * np.eye(N)
    T = L if uplo == db.Lower else L.T
    d, buf = packed(T, NB, uplo)
    assert gpu_ctx.dtrtri(uplo, diag, d) == 0, gpu_ctx.last_error()
    got = db.unpack(buf, d)
    got = np.tril(got) if uplo == db.Lower else np.triu(got)
    Tu = T.copy()
    if diag == db.Unit:
        np.fill_diagonal(Tu, 1.0)
    ref = np.linalg.inv(Tu)
    if diag == db.Unit:
        np.fill_diagonal(ref, np.diag(T))      # the diagonal is not referenced nor written
        np.fill_diagonal(got, np.diag(T))
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-13
    d2, buf2 = packed(T, NB, uplo)
    assert gpu_ctx.dlauum(uplo, d2) == 0
    got2 = db.unpack(buf2, d2)
    ref2 = T.T @ T if uplo == db.Lower else T @ T.T
    tri = np.tril if uplo == db.Lower else np.triu
    assert np.linalg.norm(tri(got2) - tri(ref2)) / np.linalg.norm(ref2) < 1e-14


def test_dtrtri_singular_info(gpu_ctx):
    N, NB = 200, 64
    L = np.tril(np.ones((N, N))) + np.eye(N)
    L[150, 150] = 0.0
    d, buf = packed(L, NB, db.Lower)
    before = buf.copy()
    assert gpu_ctx.dtrtri(db.Lower, db.NonUnit, d) == 151
    assert np.array_equal(buf, before)
