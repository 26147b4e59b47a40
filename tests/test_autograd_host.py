"""Host-side logic of the batched GP path (no GPU): the flat <-> padded index
maps of a batch of uneven orders and the whole-batch kernel construction,
against per-problem construction."""
import numpy as np
import torch

from dplasma_b200 import autograd as dag


def test_batch_layout_maps():
    sizes = [5, 1, 7, 3]
    lay = dag._batch_layout(sizes, "cpu")
    B, nmax = lay["B"], lay["nmax"]
    assert (B, nmax) == (4, 7)
    assert lay["moff_h"] == [0, 25, 26, 75] and lay["voff_h"] == [0, 5, 6, 13]
    mpad = lay["mpad"].numpy()
    vpad = lay["vpad"].numpy()
    assert len(mpad) == sum(n * n for n in sizes) and len(vpad) == sum(sizes)
    for b, n in enumerate(sizes):
        o, v = lay["moff_h"][b], lay["voff_h"][b]
        for r in range(n):
            assert vpad[v + r] == b * nmax + r
            for c in range(n):
                assert mpad[o + r * n + c] == b * nmax * nmax + r * nmax + c   # row-major in both
    assert lay["pid"].tolist() == [b for b, n in enumerate(sizes) for _ in range(n)]
    assert dag._batch_layout(sizes, "cpu") is lay                           # cached


def test_se_kernel_batched_matches_per_problem():
    gen = torch.Generator().manual_seed(3)
    sizes = [9, 2, 17, 1, 30]
    xs = [torch.rand(n, 3, generator=gen, dtype=torch.float64) for n in sizes]
    ls = torch.tensor(0.25, dtype=torch.float64, requires_grad=True)
    Kb = dag.se_kernel_batched(xs, ls, nugget=1e-3)
    Kf = dag.se_kernel_batched(xs, ls.detach(), nugget=1e-3, flat=True)
    off = 0
    for K, x, n in zip(Kb, xs, sizes):
        ref = dag.se_kernel(x, ls.detach(), nugget=1e-3)
        assert K.shape == (n, n)
        assert torch.equal(K.detach(), ref)                                   # the same arithmetic
        assert torch.equal(Kf[off:off + n * n].view(n, n), ref)
        off += n * n
    # gradient in the shared lengthscale through the views
    sum(K.sum() for K in Kb).backward()
    ls2 = ls.detach().clone().requires_grad_(True)
    sum(dag.se_kernel(x, ls2, nugget=1e-3).sum() for x in xs).backward()
    assert np.isclose(ls.grad.item(), ls2.grad.item(), rtol=1e-14)
