"""torch.autograd functions over the library's C ABI.

* ``cholesky(A)``: lower Cholesky factor of a symmetric positive definite
  float64 CUDA matrix; forward is ``dplasma_dpotrf``, backward
  ``dplasma_dpotrf_adjoint`` (the reverse Cholesky sweep; the gradient returned
  for A is symmetric).
* ``gp_log_marginal_likelihood_batched(Ks, ys)``: the same for a list of
  independent problems; forward is one batched launch
  (``dplasma_b200_dposv_batched``: factor, solve, log-det), backward one
  batched inverse (``dplasma_b200_dpotri_batched``) for the K_i^-1, with all
  problems in one flat buffer so that the rest is a fixed number of
  whole-batch tensor operations; ``se_kernel_batched`` builds the K_i the
  same way, and ``gp_log_marginal_likelihood_flat`` takes the batch as one
  flat tensor (one autograd node).
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


_layouts = {}


def _batch_layout(sizes, device):
    """Flat and padded index maps of a batch of orders `sizes` (cached): every
    problem's matrix lives row-major at moff[b] in one flat buffer and at
    [b, :n, :n] of a (batch, nmax, nmax) padded array; mpad / vpad give the
    padded position of each flat matrix / vector entry."""
    key = (tuple(sizes), str(device))
    lay = _layouts.get(key)
    if lay is not None:
        return lay
    import numpy as np
    sz = np.asarray(sizes, dtype=np.int64)
    B, nmax = len(sz), int(sz.max())
    moff = np.concatenate([[0], np.cumsum(sz * sz)[:-1]]).astype(np.int64)
    voff = np.concatenate([[0], np.cumsum(sz)[:-1]]).astype(np.int64)
    mpad = np.empty(int((sz * sz).sum()), np.int64)
    vpad = np.empty(int(sz.sum()), np.int64)
    for b in range(B):
        n = int(sz[b])
        r = np.arange(n, dtype=np.int64)
        mpad[moff[b]:moff[b] + n * n] = b * nmax * nmax + (r[:, None] * nmax + r[None, :]).ravel()
        vpad[voff[b]:voff[b] + n] = b * nmax + r

    def dev(a):
        return torch.from_numpy(a).to(device)

    lay = {"B": B, "nmax": nmax, "sizes": list(int(v) for v in sz), "n32": dev(sz.astype(np.int32)),
           "moff": dev(moff), "voff": dev(voff), "mpad": dev(mpad), "vpad": dev(vpad),
           "pid": dev(np.repeat(np.arange(B, dtype=np.int64), sz)), "nf": dev(sz.astype(np.float64)),
           "moff_h": moff.tolist(), "voff_h": voff.tolist()}
    if len(_layouts) > 8:
        _layouts.clear()
    _layouts[key] = lay
    return lay


def _split(flat, offs, sizes, square):
    return [flat[o:o + n * n].view(n, n) if square else flat[o:o + n] for o, n in zip(offs, sizes)]


def _gp_flat_forward(Kflat, y0, lay):
    """values of the batch and (factors, alpha) for the backward; Kflat is
    consumed (overwritten by the factors)"""
    dev = Kflat.device
    ctx = context(dev)
    nb = lay["B"]
    alpha = y0.clone()
    ptrK = Kflat.data_ptr() + 8 * lay["moff"]
    ptrY = alpha.data_ptr() + 8 * lay["voff"]
    logdet = torch.empty(nb, dtype=torch.float64, device=dev)
    info = torch.empty(nb, dtype=torch.int32, device=dev)
    torch_ready(Kflat, alpha, ptrK, ptrY, lay["n32"])
    rc = ctx.posv_batched_arrays(torch.float64, nb, lay["n32"], lay["n32"], ptrK, ptrY, 1, logdet, info)
    if rc != 0:
        raise RuntimeError(f"dplasma_b200_dposv_batched: {rc} {ctx.last_error()}")
    bad = info != 0
    if bool(bad.any()):
        raise RuntimeError(f"batched factorization: INFO {info[bad][:4].tolist()} (not positive definite)")
    dots = torch.zeros(nb, dtype=torch.float64, device=dev).index_add_(0, lay["pid"], y0 * alpha)
    vals = -0.5 * dots - 0.5 * logdet - 0.5 * lay["nf"] * math.log(2 * math.pi)
    return vals, alpha


def _gp_flat_backward(Lflat, alpha, g, lay):
    """(dK flat, dy flat) of the batch from the factors and alpha"""
    dev = Lflat.device
    ctx = context(dev)
    B, nmax = lay["B"], lay["nmax"]
    inv = Lflat.clone()
    ptr = inv.data_ptr() + 8 * lay["moff"]
    info = torch.empty(B, dtype=torch.int32, device=dev)
    torch_ready(inv, ptr, lay["n32"])
    from . import lib
    rc = lib().dplasma_b200_dpotri_batched(ctx.h, B, lay["n32"].data_ptr(), lay["n32"].data_ptr(), ptr.data_ptr(),
                                           info.data_ptr())
    if rc != 0 or bool((info != 0).any()):
        raise RuntimeError(f"batched inverse failed: {rc} {ctx.last_error()}")
    # K_i^-1 is the column-major lower = row-major upper triangle of each block
    P = torch.zeros(B * nmax * nmax, dtype=torch.float64, device=dev).index_copy_(0, lay["mpad"], inv)
    P = P.view(B, nmax, nmax)
    Kinv = torch.triu(P) + torch.triu(P, 1).transpose(1, 2)
    al = torch.zeros(B * nmax, dtype=torch.float64, device=dev).index_copy_(0, lay["vpad"], alpha).view(B, nmax)
    dK = g.view(B, 1, 1) * (0.5 * al[:, :, None] * al[:, None, :] - 0.5 * Kinv)
    return dK.reshape(-1).index_select(0, lay["mpad"]), -g.index_select(0, lay["pid"]) * alpha


class _GPLogMLBatched(torch.autograd.Function):
    """List form: the problems are gathered into one flat buffer, then one
    batched factor + solve + log-det launch forward and one batched inverse
    launch backward, with a fixed number of whole-batch tensor operations
    around them."""

    @staticmethod
    def forward(ctx_, nb, *args):
        Ks, ys = args[:nb], args[nb:]
        lay = _batch_layout([K.shape[0] for K in Ks], Ks[0].device)
        Kflat = torch.cat([K.detach().reshape(-1) for K in Ks])
        y0 = torch.cat([y.detach().reshape(-1) for y in ys])
        vals, alpha = _gp_flat_forward(Kflat, y0, lay)
        ctx_.lay = lay
        ctx_.yshapes = [y.shape for y in ys]
        ctx_.save_for_backward(Kflat, alpha)
        return vals

    @staticmethod
    def backward(ctx_, g):
        Lflat, alpha = ctx_.saved_tensors
        lay = ctx_.lay
        dKflat, dyflat = _gp_flat_backward(Lflat, alpha, g, lay)
        dKs = _split(dKflat, lay["moff_h"], lay["sizes"], True)
        dys = [v.reshape(sh) for v, sh in zip(_split(dyflat, lay["voff_h"], lay["sizes"], False), ctx_.yshapes)]
        return (None, *dKs, *dys)


class _GPLogMLFlat(torch.autograd.Function):
    """Flat form: Kflat holds the row-major K_i one after the other, yflat
    the y_i; one autograd node for the whole batch."""

    @staticmethod
    def forward(ctx_, Kflat, yflat, sizes):
        lay = _batch_layout(list(sizes), Kflat.device)
        work = Kflat.detach().clone()
        vals, alpha = _gp_flat_forward(work, yflat.detach().contiguous(), lay)
        ctx_.lay = lay
        ctx_.save_for_backward(work, alpha)
        return vals

    @staticmethod
    def backward(ctx_, g):
        Lflat, alpha = ctx_.saved_tensors
        dKflat, dyflat = _gp_flat_backward(Lflat, alpha, g, ctx_.lay)
        return dKflat, dyflat, None


def gp_log_marginal_likelihood_batched(Ks, ys) -> torch.Tensor:
    """Values (batch,) of the GP log-marginal likelihoods of independent
    problems K_i (n_i x n_i, float64 CUDA) and y_i (n_i,)."""
    return _GPLogMLBatched.apply(len(Ks), *Ks, *ys)


def gp_log_marginal_likelihood_flat(Kflat: torch.Tensor, yflat: torch.Tensor, sizes) -> torch.Tensor:
    """The same with the problems concatenated: Kflat the row-major K_i one
    after the other (sum n_i^2 values), yflat the y_i (sum n_i values), sizes
    the n_i.  One autograd node for the batch (use with se_kernel_batched(...,
    flat=True))."""
    return _GPLogMLFlat.apply(Kflat, yflat, tuple(int(n) for n in sizes))


def se_kernel_batched(xs, lengthscale: torch.Tensor, nugget: float = 1e-4, flat: bool = False):
    """se_kernel for a list of point sets x_i (n_i x d) with one shared
    lengthscale, built in a fixed number of whole-batch operations on a
    padded array; returns the K_i as views into one flat tensor, or with
    flat=True that tensor itself (row-major K_i one after the other)."""
    dev = xs[0].device
    lay = _batch_layout([x.shape[0] for x in xs], dev)
    B, nmax, d = lay["B"], lay["nmax"], xs[0].shape[1]
    X = torch.zeros(B * nmax, d, dtype=xs[0].dtype, device=dev).index_copy(0, lay["vpad"], torch.cat(xs, 0))
    X = X.view(B, nmax, d)
    d2 = ((X[:, :, None, :] - X[:, None, :, :]) ** 2).sum(-1)
    Kp = torch.exp(-d2 / (2.0 * lengthscale ** 2)) + nugget * torch.eye(nmax, dtype=X.dtype, device=dev)
    Kflat = Kp.reshape(-1).index_select(0, lay["mpad"])
    return Kflat if flat else _split(Kflat, lay["moff_h"], lay["sizes"], True)


def se_kernel(x: torch.Tensor, lengthscale: torch.Tensor, nugget: float = 1e-4) -> torch.Tensor:
    """Squared-exponential kernel exp(-|xi - xj|^2 / (2 l^2)) + nugget I (torch ops)."""
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    return torch.exp(-d2 / (2.0 * lengthscale ** 2)) + nugget * torch.eye(x.shape[0], dtype=x.dtype, device=x.device)
