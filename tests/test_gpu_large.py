"""GPU parity at the sizes of the FP64 and mixed-precision workloads, where the
device scheduler runs 64-256 steps: N = 16384 for NB in {256, 384, 512} and
uplo in {L, U}, one N = 32768 case, a mixed-precision solve at N = 16384 and
kappa = 1e6, and the GP log-marginal-likelihood gradient at N = 16384.

Bars (src/dplasma_zcheck.c:63-133 check_zpotrf and :179-224 check_zaxmb,
tightened from the reference's 60 to 10; shapes from the FP64 sweep
N x NB x uplo):
  * the factor within 1e-12 relative Frobenius norm of the oracle's (the
    tile algorithm of src/zpotrf_L.jdf / zpotrf_U.jdf restated over
    OpenBLAS, run as the tile DAG on all host cores);
  * ||LL^T - A||_inf / (||A||_inf N eps) < 10 and the dpotrs residual
    ||Ax - b||_inf / ((||A|| ||x|| + ||b||) N eps) < 10 (NRHS = 16);
  * mixed: backward error < 10 N eps without fallback, and the solution
    within the kappa N eps bound of the FP64 solve;
  * gradient: against torch float64 autograd through its own Cholesky and
    against central differences in the lengthscale to their own accuracy.
"""
import os

import numpy as np
import pytest

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu

SEED_A, SEED_B = 3872, 3873
FACTOR_TOL = 1e-12
RATIO_TOL = 10.0
EPS = 2.0 ** -53
THREADS = os.cpu_count() or 1


def tri_rel_err(X, Y, uplo, step=2048):
    """||tri(X) - tri(Y)||_F / ||tri(Y)||_F by column blocks (no N x N temporaries)."""
    N = X.shape[0]
    num = den = 0.0
    for j0 in range(0, N, step):
        j1 = min(N, j0 + step)
        if uplo == db.Lower:
            xs, ys = X[j0:, j0:j1], Y[j0:, j0:j1]
            d = np.tril(xs - ys)
            y = np.tril(ys)
        else:
            xs, ys = X[:j1, j0:j1], Y[:j1, j0:j1]
            d = np.triu(xs - ys, j0)
            y = np.triu(ys, j0)
        num += float((d * d).sum())
        den += float((y * y).sum())
    return np.sqrt(num / den)


def gpu_factor_and_solve(ctx, A0, B0, NB, uplo):
    N = A0.shape[0]
    dA = db.desc_sym(N, NB, uplo)
    bufA = db.pack(A0, dA)
    db.attach(dA, bufA)
    info = ctx.dpotrf(uplo, dA)
    assert info == 0, (info, ctx.last_error())
    factor_ms = ctx.last_factor_ms()
    dB = db.desc_general(N, B0.shape[1], NB, NB)
    bufB = db.pack(B0, dB)
    db.attach(dB, bufB)
    assert ctx.dpotrs(uplo, dA, dB) == 0, ctx.last_error()
    L = db.unpack(bufA, dA)
    del bufA
    return L, db.unpack(bufB, dB), factor_ms


def check_case(ctx, N, NB, uplo):
    ouplo = oracle.LOWER if uplo == db.Lower else oracle.UPPER
    A0 = oracle.dplgsy(N, NB, SEED_A)
    B0 = oracle.dplrnt(N, 16, NB, NB, SEED_B)
    L, X, factor_ms = gpu_factor_and_solve(ctx, A0, B0, NB, uplo)
    Lo = A0.copy(order="F")
    assert oracle.dpotrf_parallel(ouplo, Lo, NB, THREADS) == 0
    err = tri_rel_err(L, Lo, uplo)
    del Lo
    assert err <= FACTOR_TOL, (N, NB, uplo, err)
    r_fac = oracle.check_dpotrf(ouplo, L, A0)
    assert r_fac < RATIO_TOL, (N, NB, uplo, r_fac)
    del L
    r_sol = oracle.check_daxmb(ouplo, A0, B0, np.asfortranarray(X))
    assert r_sol < RATIO_TOL, (N, NB, uplo, r_sol)
    print(f"N={N} NB={NB} uplo={'L' if uplo == db.Lower else 'U'}: factor {factor_ms:.1f} ms, "
          f"rel err {err:.2e}, check_dpotrf {r_fac:.3f}, check_daxmb {r_sol:.3f}")


@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
@pytest.mark.parametrize("NB", [256, 384, 512])
def test_factor_and_solve_n16384(gpu_ctx, NB, uplo):
    check_case(gpu_ctx, 16384, NB, uplo)


def test_factor_and_solve_n32768(gpu_ctx):
    check_case(gpu_ctx, 32768, 256, db.Lower)


def test_mixed_solve_n16384_kappa1e6():
    torch = pytest.importorskip("torch")
    N, NB, NRHS, kappa = 16384, 256, 16, 1e6
    with db.Context(0) as ctx:
        dA = db.desc_sym(N, NB, db.Lower)
        A = torch.empty(db.desc_elems(dA), dtype=torch.float64, device="cuda")
        db.attach(dA, A)
        assert ctx.dplgsy_cond(kappa, 64, db.Lower, dA, 7) == 0, ctx.last_error()
        dB = db.desc_general(N, NRHS, NB, NB)
        B = torch.empty(db.desc_elems(dB), dtype=torch.float64, device="cuda")
        db.attach(dB, B)
        assert ctx.dplrnt(0, dB, SEED_B) == 0
        A_keep, B_keep = A.clone(), B.clone()
        # FP64 reference solve on copies
        dA64, dB64 = db.desc_sym(N, NB, db.Lower), db.desc_general(N, NRHS, NB, NB)
        A64, B64 = A.clone(), B.clone()
        db.attach(dA64, A64)
        db.attach(dB64, B64)
        assert ctx.dposv(db.Lower, dA64, dB64) == 0, ctx.last_error()
        del A64
        X64 = db.unpack(B64.cpu().numpy(), dB64)
        Bh = db.unpack(B_keep.cpu().numpy(), dB)
        for fmt in (db.FP16_SPLIT, db.FP16):
            dX = db.desc_general(N, NRHS, NB, NB)
            X = torch.zeros(db.desc_elems(dX), dtype=torch.float64, device="cuda")
            db.attach(dX, X)
            rc, st = ctx.dsposv(db.Lower, dA, dB, dX, fmt=fmt)
            assert rc == 0, ctx.last_error()
            assert st["fallback"] == 0, st
            assert st["backward_error"] < 10 * N * EPS, st
            assert torch.equal(A, A_keep) and torch.equal(B, B_keep)       # inputs untouched
            Xh = db.unpack(X.cpu().numpy(), dX)
            fwd = np.abs(Xh - X64).max() / np.abs(X64).max()
            assert fwd <= kappa * N * EPS, (fmt, fwd, st)
            print(f"mixed fmt={fmt}: iter {st['iter']} gmres {st['inner_iters']} fmt_used {st['fmt_used']} "
                  f"bwd {st['backward_error']:.2e} fwd vs fp64 {fwd:.2e}")
        del Bh


def test_gp_gradient_n16384():
    torch = pytest.importorskip("torch")
    from dplasma_b200 import autograd as dag
    n = 16384
    g = torch.Generator(device="cuda").manual_seed(13)
    x = torch.rand(n, 3, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)

    def f(l):
        with torch.no_grad():
            return dag.gp_log_marginal_likelihood(dag.se_kernel(x, torch.tensor(l, dtype=torch.float64,
                                                                                  device="cuda")), y).item()

    ls = torch.tensor(0.2, dtype=torch.float64, device="cuda", requires_grad=True)
    val = dag.gp_log_marginal_likelihood(dag.se_kernel(x, ls), y)
    val.backward()
    grad = ls.grad.item()
    # FP64 reference gradient: torch autograd through its own Cholesky
    lr = torch.tensor(0.2, dtype=torch.float64, device="cuda", requires_grad=True)
    K = dag.se_kernel(x, lr)
    L = torch.linalg.cholesky(K)
    a = torch.cholesky_solve(y[:, None], L)[:, 0]
    ref = -0.5 * y @ a - torch.log(torch.diagonal(L)).sum() - 0.5 * n * np.log(2 * np.pi)
    ref.backward()
    assert abs(val.item() - ref.item()) <= 1e-8 * abs(ref.item()), (val.item(), ref.item())
    assert abs(grad - lr.grad.item()) <= 1e-6 * abs(lr.grad.item()), (grad, lr.grad.item())
    del K, L, a
    # central differences (h = 1e-6), checked to their own accuracy: the
    # difference between steps h and 2h measures the rounding noise of the
    # differences of this ill-conditioned kernel matrix
    h = 1e-6
    fd1 = (f(0.2 + h) - f(0.2 - h)) / (2 * h)
    fd2 = (f(0.2 + 2 * h) - f(0.2 - 2 * h)) / (4 * h)
    tol = min(1e-2 * abs(grad), max(1e-5 * abs(grad), 3.0 * abs(fd1 - fd2)))
    assert abs(fd1 - grad) <= tol, (fd1, fd2, grad)
    print(f"GP N={n}: dlengthscale {grad:.6e}, torch {lr.grad.item():.6e}, FD {fd1:.6e} / {fd2:.6e}")
