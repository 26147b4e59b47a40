"""GPU tests of the Cholesky adjoint (dplasma_dpotrf_adjoint) and the
torch.autograd wrappers over it (dplasma_b200.autograd).

References: torch float64 autograd through torch.linalg.cholesky on the CPU
(the symmetric part of its gradient), and central finite differences with
h = 1e-6 along random symmetric directions.  The GP log-marginal-likelihood
gradient is checked with respect to K and to the kernel lengthscale."""
import ctypes

import numpy as np
import pytest
import torch

import dplasma_b200 as db
from dplasma_b200 import autograd as dag

pytestmark = pytest.mark.gpu


def spd(n, seed):
    g = torch.Generator().manual_seed(seed)
    x = torch.rand(n, 3, generator=g, dtype=torch.float64)
    return dag.se_kernel(x, torch.tensor(0.3, dtype=torch.float64), nugget=1e-2)


def sym(X):
    return 0.5 * (X + X.T)


def torch_ref_grad(A, G):
    A = A.clone().requires_grad_(True)
    L = torch.linalg.cholesky(A)
    (L * G).sum().backward()
    return sym(A.grad)


@pytest.mark.parametrize("n", [1, 5, 100, 300, 512, 700])
def test_cholesky_adjoint_vs_torch_cpu(gpu_ctx, n):
    A = spd(n, n)
    G = torch.tril(torch.randn(n, n, dtype=torch.float64, generator=torch.Generator().manual_seed(7)))
    ref = torch_ref_grad(A, G)
    Ad = A.cuda().requires_grad_(True)
    L = dag.cholesky(Ad)
    assert torch.allclose(L.cpu(), torch.linalg.cholesky(A), rtol=0, atol=1e-12 * A.abs().max().item())
    (L * G.cuda()).sum().backward()
    got = Ad.grad.cpu()
    assert torch.allclose(got, got.T)
    err = (got - ref).norm() / ref.norm()
    assert err < 1e-10, err


def test_cholesky_adjoint_finite_differences(gpu_ctx):
    n, h = 200, 1e-6
    A = spd(n, 3)
    G = torch.tril(torch.randn(n, n, dtype=torch.float64, generator=torch.Generator().manual_seed(11)))
    ref = torch_ref_grad(A, G)                      # exact gradient, CPU autograd
    A, G = A.cuda(), G.cuda()
    Ad = A.clone().requires_grad_(True)
    (dag.cholesky(Ad) * G).sum().backward()
    for s in range(3):
        E = sym(torch.randn(n, n, dtype=torch.float64, generator=torch.Generator().manual_seed(s))).cuda()
        fp = (torch.linalg.cholesky(A + h * E) * G).sum()
        fm = (torch.linalg.cholesky(A - h * E) * G).sum()
        fd = ((fp - fm) / (2 * h)).item()
        an = (Ad.grad * E).sum().item()
        an_ref = (ref.cuda() * E).sum().item()
        # the directional derivative agrees with the exact one ...
        assert abs(an - an_ref) <= 1e-9 * abs(an_ref), (an, an_ref)
        # ... and with central differences to their own accuracy (O(h^2)
        # truncation grows with the conditioning of this SE-kernel matrix)
        assert abs(fd - an) <= max(2e-5 * max(1.0, abs(an)), 2.0 * abs(fd - an_ref) + 1e-9), (fd, an, an_ref)


@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
def test_adjoint_c_abi_tile_storage(gpu_ctx, uplo):
    # TILE storage, ragged N (NB does not divide N), through the C ABI
    N, NB = 333, 128
    A = spd(N, 5).numpy()
    L = np.linalg.cholesky(A)
    G = np.tril(np.random.default_rng(1).standard_normal((N, N)))
    ref = torch_ref_grad(torch.tensor(A), torch.tensor(G)).numpy()
    dL = db.desc_sym(N, NB, uplo)
    dG = db.desc_sym(N, NB, uplo)
    bL = db.pack(L if uplo == db.Lower else L.T, dL)
    bG = db.pack(G if uplo == db.Lower else G.T, dG)
    db.attach(dL, bL)
    db.attach(dG, bG)
    assert gpu_ctx.dpotrf_adjoint(uplo, dL, dG) == 0, gpu_ctx.last_error()
    out = db.unpack(bG, dG)
    tri = np.tril(out) if uplo == db.Lower else np.triu(out)
    full = tri + tri.T - np.diag(np.diag(tri))
    assert np.linalg.norm(full - ref) / np.linalg.norm(ref) < 1e-10


def test_gp_log_marginal_likelihood_gradients(gpu_ctx):
    n = 400
    gen = torch.Generator().manual_seed(13)
    x = torch.rand(n, 3, generator=gen, dtype=torch.float64)
    y = torch.randn(n, generator=gen, dtype=torch.float64)
    # reference: torch float64 autograd on the CPU
    ls = torch.tensor(0.2, dtype=torch.float64, requires_grad=True)
    K = dag.se_kernel(x, ls)
    Kr = K.detach().clone().requires_grad_(True)
    L = torch.linalg.cholesky(Kr)
    a = torch.cholesky_solve(y[:, None], L)[:, 0]
    ref = -0.5 * y @ a - torch.log(torch.diagonal(L)).sum() - 0.5 * n * np.log(2 * np.pi)
    ref.backward()
    (dls_ref,) = torch.autograd.grad(
        -0.5 * y @ torch.cholesky_solve(y[:, None], torch.linalg.cholesky(dag.se_kernel(x, ls)))[:, 0]
        - torch.log(torch.diagonal(torch.linalg.cholesky(dag.se_kernel(x, ls)))).sum(), ls)
    # ours
    xc, yc = x.cuda(), y.cuda()
    lsc = torch.tensor(0.2, dtype=torch.float64, device="cuda", requires_grad=True)
    Kc = dag.se_kernel(xc, lsc)
    Kc.retain_grad()
    val = dag.gp_log_marginal_likelihood(Kc, yc)
    assert abs(val.item() - ref.item()) <= 1e-9 * abs(ref.item())
    val.backward()
    gK = Kc.grad.cpu()
    assert (gK - sym(Kr.grad)).norm() / sym(Kr.grad).norm() < 1e-9
    assert abs(lsc.grad.item() - dls_ref.item()) <= 1e-8 * abs(dls_ref.item())
    # central differences in the lengthscale
    h = 1e-6
    f = lambda l: dag.gp_log_marginal_likelihood(dag.se_kernel(xc, torch.tensor(l, dtype=torch.float64, device="cuda")), yc).item()
    fd = (f(0.2 + h) - f(0.2 - h)) / (2 * h)
    assert abs(fd - lsc.grad.item()) <= 1e-5 * abs(lsc.grad.item())


def test_batched_potri_and_gp_gradients(gpu_ctx):
    # the batch part of the GP configuration: n in [64, 256]
    rng = np.random.default_rng(13)
    sizes = [int(v) for v in rng.integers(64, 257, 12)] + [1, 31, 33]
    gen = torch.Generator().manual_seed(13)
    xs = [torch.rand(n, 3, generator=gen, dtype=torch.float64) for n in sizes]
    ys = [torch.randn(n, generator=gen, dtype=torch.float64) for n in sizes]
    # batched inverse against numpy
    Ks = [dag.se_kernel(x, torch.tensor(0.2, dtype=torch.float64), nugget=1e-2) for x in xs]
    mats = [K.cuda().contiguous() for K in Ks]
    info, _ = gpu_ctx.posv_batched(mats, None)
    assert (info.numpy() == 0).all()
    info = gpu_ctx.potri_batched(mats)
    assert (info.numpy() == 0).all()
    for K, M in zip(Ks, mats):
        Mh = M.cpu()
        Kinv = torch.triu(Mh) + torch.triu(Mh, 1).T
        ref = torch.linalg.inv(K)
        assert (Kinv - ref).norm() / ref.norm() < 1e-11
    # gradients of the summed likelihoods in K and a shared lengthscale
    ls_ref = torch.tensor(0.2, dtype=torch.float64, requires_grad=True)
    tot = 0
    for x, y in zip(xs, ys):
        K = dag.se_kernel(x, ls_ref)
        L = torch.linalg.cholesky(K)
        a = torch.cholesky_solve(y[:, None], L)[:, 0]
        tot = tot + (-0.5 * y @ a - torch.log(torch.diagonal(L)).sum() - 0.5 * x.shape[0] * np.log(2 * np.pi))
    tot.backward()
    ls = torch.tensor(0.2, dtype=torch.float64, device="cuda", requires_grad=True)
    vals = dag.gp_log_marginal_likelihood_batched([dag.se_kernel(x.cuda(), ls) for x in xs], [y.cuda() for y in ys])
    assert abs(vals.sum().item() - tot.item()) <= 1e-9 * abs(tot.item())
    vals.sum().backward()
    assert abs(ls.grad.item() - ls_ref.grad.item()) <= 1e-8 * abs(ls_ref.grad.item())
    # the same through the whole-batch kernel construction
    ls2 = torch.tensor(0.2, dtype=torch.float64, device="cuda", requires_grad=True)
    Kb = dag.se_kernel_batched([x.cuda() for x in xs], ls2)
    for Kbi, x in zip(Kb, xs):
        assert Kbi.shape == (x.shape[0], x.shape[0])
        assert (Kbi.detach() - dag.se_kernel(x.cuda(), ls2.detach())).abs().max().item() <= 1e-15
    vals2 = dag.gp_log_marginal_likelihood_batched(Kb, [y.cuda() for y in ys])
    assert (vals2.detach() - vals.detach()).abs().max().item() <= 1e-9 * vals.detach().abs().max().item()
    vals2.sum().backward()
    assert abs(ls2.grad.item() - ls.grad.item()) <= 1e-9 * abs(ls.grad.item())
    # and in the flat form (one autograd node)
    ls3 = torch.tensor(0.2, dtype=torch.float64, device="cuda", requires_grad=True)
    Kf = dag.se_kernel_batched([x.cuda() for x in xs], ls3, flat=True)
    vals3 = dag.gp_log_marginal_likelihood_flat(Kf, torch.cat([y.cuda() for y in ys]), sizes)
    assert (vals3.detach() - vals.detach()).abs().max().item() <= 1e-9 * vals.detach().abs().max().item()
    vals3.sum().backward()
    assert abs(ls3.grad.item() - ls.grad.item()) <= 1e-9 * abs(ls.grad.item())
