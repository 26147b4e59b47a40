"""GPU tests of the mixed-precision solve (dplasma_dsposv / dplasma_b200_dsposv_ex):
a Cholesky factorization whose trailing updates run on the FP16/BF16 tensor
cores, refined in FP64 (plain refinement, GMRES-IR) to the accuracy of LAPACK
dsposv, with the FP64 fallback.

Bars:
  * the converged solution meets dsposv's stopping test, hence the dplasma
    check_daxmb ratio ||Ax-b||_inf / ((||A|| ||x|| + ||b||) N eps) < 10
    (src/dplasma_zcheck.c), and agrees with the FP64 dposv solution to the
    accuracy the conditioning allows;
  * matrices A = Q diag(sigma) Q^T (Q a product of 64 Householder
    reflectors of random unit vectors, seed 7; sigma geometric from 1 to
    kappa) reach backward error < 10 N eps for kappa up to 1e6, and a
    forward error within the kappa N eps bound that FP64 obeys;
  * the FP64 fallback leaves the FP64 factor in A (dsposv semantics) and a
    non positive definite A returns dplasma's INFO.
"""
import numpy as np
import pytest

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu

EPS = 2.0 ** -53


def householder_spd(N, kappa, seed=7, nrefl=64):
    """A = Q diag(sigma) Q^T with Q = H_1 ... H_nrefl, H_i = I - 2 v v^T."""
    rng = np.random.default_rng(seed)
    sigma = np.geomspace(1.0, kappa, N)
    A = np.diag(sigma)
    for _ in range(nrefl):
        v = rng.standard_normal(N)
        v /= np.linalg.norm(v)
        Av = A @ v
        vAv = v @ Av
        A = A - 2.0 * np.outer(v, Av) - 2.0 * np.outer(Av, v) + 4.0 * vAv * np.outer(v, v)
    return 0.5 * (A + A.T)


def sym_desc_with(A0, NB, uplo):
    d = db.desc_sym(A0.shape[0], NB, uplo)
    buf = db.pack(A0, d)
    db.attach(d, buf)
    return d, buf


def gen_desc(B0, NB):
    d = db.desc_general(B0.shape[0], B0.shape[1], NB, NB)
    buf = db.pack(B0, d)
    db.attach(d, buf)
    return d, buf


def daxmb_ratio(A, X, B):
    N = A.shape[0]
    an = np.abs(A).sum(axis=1).max()
    R = B - A @ X
    return np.abs(R).max() / ((an * np.abs(X).max() + np.abs(B).max()) * N * EPS)


def run_dsposv(ctx, A0, B0, NB, uplo, **kw):
    dA, bufA = sym_desc_with(A0, NB, uplo)
    dB, bufB = gen_desc(B0, NB)
    dX, bufX = gen_desc(np.zeros_like(B0), NB)
    rc, st = ctx.dsposv(uplo, dA, dB, dX, **kw)
    return rc, st, db.unpack(bufX, dX), (dA, bufA), db.unpack(bufB, dB)


def run_dposv(ctx, A0, B0, NB, uplo):
    dA, bufA = sym_desc_with(A0, NB, uplo)
    dB, bufB = gen_desc(B0, NB)
    assert ctx.dposv(uplo, dA, dB) == 0, ctx.last_error()
    return db.unpack(bufB, dB)


@pytest.mark.parametrize("N,NB,NRHS,uplo,fmt", [
    (2048, 256, 16, db.Lower, db.FP16),
    (2048, 256, 16, db.Lower, db.BF16),
    (2048, 256, 16, db.Upper, db.FP16),
    (1000, 256, 5, db.Lower, db.FP16),      # ragged: identity-padded last tile
    (1300, 200, 3, db.Lower, db.BF16),      # nb 200 -> 256-wide internal tiles
    (256, 256, 1, db.Lower, db.FP16),       # one tile: no tensor-core update at all
    (2048, 256, 16, db.Lower, db.FP16_SPLIT),
    (1300, 200, 3, db.Upper, db.FP16_SPLIT),
])
def test_dsposv_dplgsy(gpu_ctx, N, NB, NRHS, uplo, fmt):
    A = oracle.dplgsy(N, NB, 3872, bump=float(N))
    B = oracle.dplrnt(N, NRHS, NB, NB, 3873)
    rc, st, X, (dA, bufA), Bafter = run_dsposv(gpu_ctx, A, B, NB, uplo, fmt=fmt)
    assert rc == 0, gpu_ctx.last_error()
    assert st["fallback"] == 0 and st["iter"] >= 0, st
    assert np.array_equal(Bafter, B)                       # B is input only
    Aafter = db.unpack(bufA, dA)
    keep = np.tril(np.ones((N, N), bool)) if uplo == db.Lower else np.triu(np.ones((N, N), bool))
    assert np.array_equal(Aafter[keep], A[keep])           # A unchanged when refinement succeeded
    assert daxmb_ratio(A, X, B) < 10.0
    X64 = run_dposv(gpu_ctx, A, B, NB, uplo)
    assert np.abs(X - X64).max() / np.abs(X64).max() < 1e-12
    assert st["backward_error"] < 10 * N * EPS
    # the infinity norm formed on the way through the working copy (padding excluded)
    anorm = np.abs(A).sum(axis=1).max()
    assert abs(st["anorm"] - anorm) <= 1e-13 * anorm, (st["anorm"], anorm)


@pytest.mark.parametrize("kappa", [1e2, 1e4, 1e6])
@pytest.mark.parametrize("fmt", [db.FP16, db.BF16, db.FP16_SPLIT])
def test_dsposv_conditioned(gpu_ctx, kappa, fmt):
    N, NB, NRHS = 2048, 256, 16
    A = householder_spd(N, kappa)
    rng = np.random.default_rng(8)
    Xt = rng.standard_normal((N, NRHS))
    B = A @ Xt
    rc, st, X, _, _ = run_dsposv(gpu_ctx, A, B, NB, db.Lower, fmt=fmt)
    assert rc == 0, gpu_ctx.last_error()
    # no FP64 fallback: a 16-bit breakdown escalates to the split form, which
    # keeps kappa = 1e6 positive definite
    assert st["fallback"] == 0 and st["fmt_used"] in (fmt, db.FP16_SPLIT), st
    assert st["backward_error"] < 10 * N * EPS, st
    assert daxmb_ratio(A, X, B) < 10.0
    X64 = run_dposv(gpu_ctx, A, B, NB, db.Lower)
    fwd = np.abs(X - Xt).max() / np.abs(Xt).max()
    fwd64 = np.abs(X64 - Xt).max() / np.abs(Xt).max()
    # a backward error below N eps bounds the forward error by kappa N eps,
    # the bound the FP64 solve obeys as well
    assert fwd <= kappa * N * EPS and fwd64 <= kappa * N * EPS, (fwd, fwd64, st)


@pytest.mark.parametrize("solver", [db.IR_PLAIN, db.IR_GMRES])
def test_dsposv_solvers(gpu_ctx, solver):
    N, NB, NRHS = 1536, 256, 8
    A = householder_spd(N, 1e3, seed=7)
    B = np.random.default_rng(9).standard_normal((N, NRHS))
    rc, st, X, _, _ = run_dsposv(gpu_ctx, A, B, NB, db.Lower, fmt=db.BF16, solver=solver)
    assert rc == 0, gpu_ctx.last_error()
    # a second call on the same context (cached task list, grown buffers) agrees
    rc2, st2, X2, _, _ = run_dsposv(gpu_ctx, A, B, NB, db.Lower, fmt=db.BF16, solver=solver)
    assert rc2 == 0 and (st2["iter"], st2["fallback"]) == (st["iter"], st["fallback"])
    assert np.abs(X2 - X).max() <= 1e-12 * np.abs(X).max()
    assert st["fallback"] == 0 and st["solver_used"] == solver, st
    if solver == db.IR_GMRES:
        assert st["inner_iters"] >= 1
    assert daxmb_ratio(A, X, B) < 10.0


def test_dsposv_fallback_leaves_fp64_factor(gpu_ctx):
    # no refinement step allowed and a matrix the first solve cannot finish:
    # the FP64 factorization produces the solution and stays in A
    N, NB, NRHS = 1024, 256, 4
    A = householder_spd(N, 1e6)
    B = np.random.default_rng(10).standard_normal((N, NRHS))
    rc, st, X, (dA, bufA), _ = run_dsposv(gpu_ctx, A, B, NB, db.Lower, fmt=db.BF16, itermax=0, escalate=False)
    assert rc == 0, gpu_ctx.last_error()
    # -1: the refinement may not iterate; -3: the 16-bit factorization broke down
    assert st["fallback"] == 1 and st["iter"] in (-1, -3), st
    L = np.tril(db.unpack(bufA, dA))
    dR, bufR = sym_desc_with(A, NB, db.Lower)
    assert gpu_ctx.dpotrf(db.Lower, dR) == 0
    Lref = np.tril(db.unpack(bufR, dR))
    assert np.array_equal(L, Lref)
    assert daxmb_ratio(A, X, B) < 10.0


def test_dsposv_not_spd_returns_info(gpu_ctx):
    N, NB = 1024, 256
    A = oracle.dplgsy(N, NB, 3872, bump=float(N))
    A[700, 700] = -1.0
    B = np.ones((N, 2))
    rc, st, _, _, _ = run_dsposv(gpu_ctx, A, B, NB, db.Lower)
    dR, _ = sym_desc_with(A, NB, db.Lower)
    info = gpu_ctx.dpotrf(db.Lower, dR)
    assert info > 0 and rc == info
    assert st["fallback"] == 1 and st["iter"] == -3 and st["fmt_used"] == -1


def test_dsposv_rejects_tile_size(gpu_ctx):
    N, NB = 640, 320           # 384-wide internal tiles: not supported by the tensor-core update
    A = oracle.dplgsy(N, NB, 3872, bump=float(N))
    rc, _, _, _, _ = run_dsposv(gpu_ctx, A, np.ones((N, 1)), NB, db.Lower)
    assert rc == db.ERR_NOT_SUPPORTED


@pytest.mark.parametrize("N,NB,uplo", [(768, 256, db.Lower), (700, 200, db.Upper)])
def test_dplgsy_cond_spectrum(gpu_ctx, N, NB, uplo):
    # the generated matrix is symmetric with eigenvalues geomspace(1, kappa, N)
    kappa = 1e4
    d = db.desc_sym(N, NB, uplo)
    buf = np.zeros(db.desc_elems(d))
    db.attach(d, buf)
    assert gpu_ctx.dplgsy_cond(kappa, 64, uplo, d, 7) == 0, gpu_ctx.last_error()
    T = db.unpack(buf, d)
    A = np.tril(T) + np.tril(T, -1).T if uplo == db.Lower else np.triu(T) + np.triu(T, 1).T
    ev = np.linalg.eigvalsh(A)
    assert np.allclose(ev, np.geomspace(1.0, kappa, N), rtol=1e-9, atol=1e-9 * kappa)
    # not diagonal: the reflectors mixed the coordinates
    assert np.abs(A - np.diag(np.diag(A))).max() > 1e-3


@pytest.mark.parametrize("kappa,shift", [(1e6, 2.0 ** -8), (1e4, 2.0 ** -10)])
def test_dsposv_shifted_fp16_gmres(gpu_ctx, kappa, shift):
    # the shifted FP16 factor of A + s diag(A) (positive definite where A's own
    # FP16 factor breaks down at kappa 1e6) refined by GMRES-IR to the dsposv accuracy
    N, NB, NRHS = 2048, 256, 4
    A = householder_spd(N, kappa)
    B = np.random.default_rng(12).standard_normal((N, NRHS))
    rc, st, X, _, _ = run_dsposv(gpu_ctx, A, B, NB, db.Lower, fmt=db.FP16, solver=db.IR_GMRES, shift=shift,
                                 escalate=False, gmres_m=60)
    assert rc == 0, gpu_ctx.last_error()
    assert st["fallback"] == 0 and st["fmt_used"] == db.FP16 and st["solver_used"] == db.IR_GMRES, st
    assert st["inner_iters"] > 0
    assert st["backward_error"] < 10 * N * EPS, st
    assert daxmb_ratio(A, X, B) < 10.0


def test_dsposv_rejects_bad_shift(gpu_ctx):
    N, NB = 512, 256
    A = oracle.dplgsy(N, NB, 3872, bump=float(N))
    rc, _, _, _, _ = run_dsposv(gpu_ctx, A, np.ones((N, 1)), NB, db.Lower, shift=-1.0)
    assert rc == db.ERR_ILLEGAL_VALUE


def _ctx_with_trsm_tc(value):
    import os
    old = os.environ.get("DPLASMA_B200_TRSM_TC")
    os.environ["DPLASMA_B200_TRSM_TC"] = value
    try:
        return db.Context(0)
    finally:
        if old is None:
            del os.environ["DPLASMA_B200_TRSM_TC"]
        else:
            os.environ["DPLASMA_B200_TRSM_TC"] = old


@pytest.fixture
def tc_ctx():
    """A context with the tensor-core TRSM strips (DPLASMA_B200_TRSM_TC=1, the
    default): the mixed split-FP16 factorization solves its panels as
    X = A Linv^T on the 16-bit tensor cores instead of FP64 DMMA."""
    ctx = _ctx_with_trsm_tc("1")
    yield ctx
    ctx.close()


@pytest.fixture
def fp64_strip_ctx():
    """A context whose split-FP16 factorization keeps its TRSM strips in FP64
    (DPLASMA_B200_TRSM_TC=0)."""
    ctx = _ctx_with_trsm_tc("0")
    yield ctx
    ctx.close()


@pytest.mark.parametrize("N,kappa", [(2048, 1e2), (2048, 1e6), (4096, 1e6), (1536, 1e4)])
def test_dsposv_tensor_core_trsm(fp64_strip_ctx, tc_ctx, N, kappa):
    # the panels in split FP16 products (about 2^-22 relative) keep the factor
    # as good a preconditioner as the FP64 panels: at most one more refinement
    # step, and the same dsposv accuracy
    NB, NRHS = 256, 8
    A = householder_spd(N, kappa)
    Xt = np.random.default_rng(8).standard_normal((N, NRHS))
    B = A @ Xt
    rc0, st0, X0, _, _ = run_dsposv(fp64_strip_ctx, A, B, NB, db.Lower, fmt=db.FP16_SPLIT)
    rc, st, X, _, _ = run_dsposv(tc_ctx, A, B, NB, db.Lower, fmt=db.FP16_SPLIT)
    assert rc0 == 0 and rc == 0, tc_ctx.last_error()
    assert st["fallback"] == 0 and st["fmt_used"] == db.FP16_SPLIT, st
    assert st["iter"] <= st0["iter"] + 1, (st, st0)
    assert st["backward_error"] < 10 * N * EPS, st
    assert daxmb_ratio(A, X, B) < 10.0
    X64 = run_dposv(tc_ctx, A, B, NB, db.Lower)
    assert np.abs(X - X64).max() / np.abs(X64).max() <= max(kappa * N * EPS, 1e-12)
    print(f"N={N} kappa={kappa:.0e}: iterations {st['iter']} (FP64 panels {st0['iter']})")


def test_dsposv_tensor_core_trsm_dplgsy_ragged(tc_ctx):
    # nb 200 -> 256-wide internal tiles with an identity-padded last tile
    N, NB, NRHS = 1300, 200, 3
    A = oracle.dplgsy(N, NB, 3872, bump=float(N))
    B = oracle.dplrnt(N, NRHS, NB, NB, 3873)
    rc, st, X, _, _ = run_dsposv(tc_ctx, A, B, NB, db.Lower, fmt=db.FP16_SPLIT)
    assert rc == 0, tc_ctx.last_error()
    assert st["fallback"] == 0 and st["fmt_used"] == db.FP16_SPLIT, st
    assert st["backward_error"] < 10 * N * EPS
    assert daxmb_ratio(A, X, B) < 10.0
