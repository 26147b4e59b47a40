"""torch.autograd functions over the library's C ABI.

* ``cholesky(A)``: lower Cholesky factor of a symmetric positive definite
  float64 CUDA matrix; forward is ``dplasma_dpotrf``, backward
  ``dplasma_dpotrf_adjoint`` (the reverse Cholesky sweep; the gradient returned
  for A is symmetric).
* ``gp_log_marginal_likelihood_batched(Ks, ys)``: the same for a list of
  independent problems; forward is one batched launch
  (``dplasma_b200_dposv_batched``: factor, solve, log-det), backward one
  batched inverse (``dplasma_b200_dpotri_batched``) for the K_i^-1.
* ``gp_log_marginal_likelihood(K, y)``: ``-1/2 y^T K^-1 y - 1/2 log det K
  - n/2 log 2 pi`` for a Gaussian-process kernel matrix K and targets y
  (vector or n x m); forward is one factorization and one solve
  (``dplasma_dpotrf`` + ``dplasma_dpotrs``), backward
  ``dK = 1/2 alpha alpha^T - 1/2 K^-1`` with ``K^-1`` -- the Cholesky adjoint
  of the log-determinant (``Lbar = diag(2 / L(i,i))``) -- formed from the
  factor by ``dplasma_dpotri``, and ``dy = -alpha``.  Gradients with respect to
  parameters of K (a lengthscale, ...) follow by torch's own chain rule.

Matrices cross the C ABI as LAPACK-storage device descriptors: a row-major
torch tensor is the column-major transpose, so a symmetric K reads the same,
and the column-major lower factor appears as the upper triangle of the
row-major buffer.
"""
from __future__ import annotations

import math

import torch

from . import Context, desc_general, attach, Lower, STORAGE_LAPACK, torch_ready

_ctx = {}


def context(device=None) -> Context:
    d = torch.device("cuda" if device is None else device)
    idx = d.index if d.index is not None else torch.cuda.current_device()
    if idx not in _ctx:
        _ctx[idx] = Context(idx)
    return _ctx[idx]


def _lapack_desc(buf: torch.Tensor, n: int, m: int | None = None, nb: int = 256):
    m = n if m is None else m
    d = desc_general(n, m, nb, nb, storage=STORAGE_LAPACK, lda=max(n, 1))
    attach(d, buf)
    return d


def _check_square(A: torch.Tensor):
    if not (A.is_cuda and A.dtype == torch.float64 and A.dim() == 2 and A.shape[0] == A.shape[1]):
        raise ValueError("expected a square float64 CUDA matrix")


def _factor(A: torch.Tensor):
    """column-major lower factor in a row-major buffer (its upper triangle)"""
    n = A.shape[0]
    buf = A.detach().contiguous().clone()
    torch_ready(buf)
    ctx = context(A.device)
    info = ctx.dpotrf(Lower, _lapack_desc(buf, n))
    if info != 0:
        raise RuntimeError(f"dplasma_dpotrf: INFO = {info} (matrix not positive definite)" if info > 0
                           else f"dplasma_dpotrf: {info} {ctx.last_error()}")
    return buf


def _adjoint(Lrow: torch.Tensor, Lbar: torch.Tensor) -> torch.Tensor:
    """Abar (symmetric) from L and Lbar given as ordinary (row-major, lower) tensors."""
    n = Lrow.shape[0]
    ctx = context(Lrow.device)
    Lc = Lrow.t().contiguous()              # column-major L
    Bc = torch.tril(Lbar).t().contiguous()  # column-major Lbar (lower)
    torch_ready(Lc, Bc)
    rc = ctx.dpotrf_adjoint(Lower, _lapack_desc(Lc, n), _lapack_desc(Bc, n))
    if rc != 0:
        raise RuntimeError(f"dplasma_dpotrf_adjoint: {rc} {ctx.last_error()}")
    up = torch.triu(Bc)                      # column-major lower part = row-major upper
    return up + torch.triu(Bc, 1).t()


def _inverse_from_factor(Lrow: torch.Tensor) -> torch.Tensor:
    """K^-1 (symmetric, row-major) from the lower factor L of K."""
    n = Lrow.shape[0]
    ctx = context(Lrow.device)
    buf = Lrow.t().contiguous()              # column-major L
    torch_ready(buf)
    rc = ctx.dpotri(Lower, _lapack_desc(buf, n))
    if rc != 0:
        raise RuntimeError(f"dplasma_dpotri: {rc} {ctx.last_error()}")
    up = torch.triu(buf)                     # column-major lower part = row-major upper
    return up + torch.triu(buf, 1).t()


class _Cholesky(torch.autograd.Function):
    @staticmethod
    def forward(ctx_, A):
        _check_square(A)
        buf = _factor(A)
        L = torch.tril(buf.t())
        ctx_.save_for_backward(L)
        return L

    @staticmethod
    def backward(ctx_, gL):
        (L,) = ctx_.saved_tensors
        return _adjoint(L, gL.contiguous())


def cholesky(A: torch.Tensor) -> torch.Tensor:
    return _Cholesky.apply(A)


class _GPLogML(torch.autograd.Function):
    @staticmethod
    def forward(ctx_, K, y):
        _check_square(K)
        n = K.shape[0]
        Y = y.reshape(n, -1) if y.dim() == 1 else y
        buf = _factor(K)
        L = torch.tril(buf.t())
        ctx = context(K.device)
        # alpha = K^-1 y by dplasma_dpotrs on the factor (column-major rhs)
        # m x n row-major = n x m column-major; a copy (for one column the
        # transpose is already contiguous and would alias y)
        rhs = Y.detach().t().contiguous().clone()
        torch_ready(rhs)
        rc = ctx.dpotrs(Lower, _lapack_desc(buf, n), _lapack_desc(rhs, n, Y.shape[1]))
        if rc != 0:
            raise RuntimeError(f"dplasma_dpotrs: {rc} {ctx.last_error()}")
        alpha = rhs.t()
        logdet = 2.0 * torch.log(torch.diagonal(L)).sum()
        m = Y.shape[1]
        val = -0.5 * (Y * alpha).sum() - 0.5 * m * logdet - 0.5 * m * n * math.log(2 * math.pi)
        ctx_.save_for_backward(L, alpha)
        ctx_.ydim = y.dim()
        return val

    @staticmethod
    def backward(ctx_, g):
        L, alpha = ctx_.saved_tensors
        m = alpha.shape[1]
        # K^-1, the adjoint of log det K through the factor, by dplasma_dpotri
        Kinv = _inverse_from_factor(L)
        dK = g * (0.5 * alpha @ alpha.t() - 0.5 * m * Kinv)
        dy = -g * alpha
        if ctx_.ydim == 1:
            dy = dy.reshape(-1)
        return dK, dy


def gp_log_marginal_likelihood(K: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    return _GPLogML.apply(K, y)


class _GPLogMLBatched(torch.autograd.Function):
    @staticmethod
    def forward(ctx_, nb, *args):
        Ks, ys = args[:nb], args[nb:]
        ctx = context(Ks[0].device)
        mats = [K.detach().contiguous().clone() for K in Ks]
        rhs = [y.detach().reshape(1, -1).contiguous().clone() for y in ys]
        info, logdet = ctx.posv_batched(mats, rhs)
        if (info != 0).any():
            raise RuntimeError(f"batched factorization: INFO {info[info != 0][:4].tolist()} (not positive definite)")
        vals = []
        for K, y, a, ld in zip(Ks, ys, rhs, logdet.tolist()):
            n = K.shape[0]
            vals.append(-0.5 * (y.reshape(-1) * a.reshape(-1)).sum() - 0.5 * ld - 0.5 * n * math.log(2 * math.pi))
        ctx_.nb = nb
        ctx_.save_for_backward(*mats, *rhs)
        ctx_.shapes = [y.shape for y in ys]
        return torch.stack(vals)

    @staticmethod
    def backward(ctx_, g):
        nb = ctx_.nb
        saved = ctx_.saved_tensors
        mats, rhs = list(saved[:nb]), saved[nb:]
        ctx = context(mats[0].device)
        inv = [m.clone() for m in mats]
        info = ctx.potri_batched(inv)            # K_i^-1, column-major lower = row-major upper
        if (info != 0).any():
            raise RuntimeError("batched inverse failed")
        dKs, dys = [], []
        for i, (M, a) in enumerate(zip(inv, rhs)):
            Kinv = torch.triu(M) + torch.triu(M, 1).t()
            al = a.reshape(-1, 1)
            dKs.append(g[i] * (0.5 * al @ al.t() - 0.5 * Kinv))
            dys.append((-g[i] * al).reshape(ctx_.shapes[i]))
        return (None, *dKs, *dys)


def gp_log_marginal_likelihood_batched(Ks, ys) -> torch.Tensor:
    """Values (batch,) of the GP log-marginal likelihoods of independent
    problems K_i (n_i x n_i, float64 CUDA) and y_i (n_i,)."""
    return _GPLogMLBatched.apply(len(Ks), *Ks, *ys)


def se_kernel(x: torch.Tensor, lengthscale: torch.Tensor, nugget: float = 1e-4) -> torch.Tensor:
    """Squared-exponential kernel exp(-|xi - xj|^2 / (2 l^2)) + nugget I (torch ops)."""
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    return torch.exp(-d2 / (2.0 * lengthscale ** 2)) + nugget * torch.eye(x.shape[0], dtype=x.dtype, device=x.device)
