"""GPU tests of the ScaLAPACK-compatible entry pdpotrf_ (the reference's
src/scalapack_wrappers/dplasma_wrapper_pdpotrf.c): a column-major global
array with a leading dimension larger than the matrix, a submatrix that
starts on a block boundary (IA, JA > 1), both uplo.

Bars: the factor of the submatrix within 1e-12 relative Frobenius norm of
the oracle's; everything outside the submatrix's uplo triangle untouched;
INFO identical to the oracle's for a matrix that is not positive definite.
"""
import numpy as np
import pytest

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu

SEED_A = 3872


def tri(A, uplo):
    return np.tril(A) if uplo == "L" else np.triu(A)


@pytest.mark.parametrize("uplo", ["L", "U", "l"])
def test_pdpotrf_submatrix(gpu_ctx, uplo):
    N, NB = 700, 100
    IA, JA = 201, 101                     # 1-based, on block boundaries
    M, NG, LLD = IA - 1 + N + 50, JA - 1 + N + 30, IA - 1 + N + 77
    rng = np.random.default_rng(5)
    G = np.asfortranarray(rng.standard_normal((LLD, NG)))
    A0 = oracle.dplgsy(N, NB, SEED_A)
    G[IA - 1:IA - 1 + N, JA - 1:JA - 1 + N] = A0
    before = G.copy(order="F")
    info = db.pdpotrf(uplo, N, G, IA, JA, [1, 0, M, NG, NB, NB, 0, 0, LLD])
    assert info == 0, gpu_ctx.last_error()
    ref = A0.copy(order="F")
    u = db.Lower if uplo.upper() == "L" else db.Upper
    oracle.dpotrf(u, ref, NB)
    sub = G[IA - 1:IA - 1 + N, JA - 1:JA - 1 + N]
    U = uplo.upper()
    err = np.linalg.norm(tri(sub, U) - tri(ref, U)) / np.linalg.norm(tri(ref, U))
    assert err <= 1e-12
    # the other triangle and everything outside the submatrix are untouched
    mask = np.ones_like(G, bool)
    inside = np.tril(np.ones((N, N), bool)) if U == "L" else np.triu(np.ones((N, N), bool))
    mask[IA - 1:IA - 1 + N, JA - 1:JA - 1 + N] = ~inside
    assert np.array_equal(G[mask], before[mask])


def test_pdpotrf_info(gpu_ctx):
    N, NB = 500, 100
    A0 = oracle.dplgsy(N, NB, SEED_A)
    A0[357, 357] = -1.0e6
    ref = A0.copy(order="F")
    want = oracle.dpotrf(db.Lower, ref, NB)
    assert want == 358
    G = np.asfortranarray(A0.copy())
    assert db.pdpotrf("L", N, G, 1, 1, [1, 0, N, N, NB, NB, 0, 0, N]) == want
