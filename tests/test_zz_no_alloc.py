"""GPU test of dplasma_b200_dpotrf_noalloc, the entry point for callers that
cannot allocate device memory (its scratch is a fixed array in the library's
device image).  It must give the factor that dplasma_dpotrf gives for the same
device-resident input, on two calls in a row (the second call finds the first
call's scratch contents and must not depend on them).

Collected last on purpose (file name) so that a failure here leaves every other
test already run; it also passes when run alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu
FACTOR_TOL = 1e-12


def _noalloc():
    f = db.lib().dplasma_b200_dpotrf_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(db.Desc)]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("N,NB", [(2048, 256), (1024, 128), (4096, 512)])
def test_noalloc_matches_dpotrf_twice(N, NB):
    torch = pytest.importorskip("torch")
    A0 = oracle.dplgsy(N, NB, 3872)
    d_ref = db.desc_sym(N, NB, db.Lower)
    host = db.pack(A0, d_ref)
    with db.Context(0) as ctx:
        ref_dev = torch.from_numpy(host.copy()).cuda()
        db.attach(d_ref, ref_dev)
        assert ctx.dpotrf(db.Lower, d_ref) == 0, ctx.last_error()
        L_ref = np.tril(db.unpack(ref_dev.cpu().numpy(), d_ref))
    f = _noalloc()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        d = db.desc_sym(N, NB, db.Lower)
        dev = torch.from_numpy(host.copy()).cuda()
        db.attach(d, dev)
        torch.cuda.current_stream().synchronize()
        assert f(ctypes.c_void_p(stream), db.Lower, ctypes.byref(d)) == 0
        L = np.tril(db.unpack(dev.cpu().numpy(), d))
        err = np.linalg.norm(L - L_ref) / np.linalg.norm(L_ref)
        assert err <= FACTOR_TOL, (call, err)


def test_noalloc_rejects_too_large():
    torch = pytest.importorskip("torch")
    N, NB = 8192 + 256, 256
    d = db.desc_sym(N, NB, db.Lower)
    dev = torch.zeros(db.desc_elems(d), dtype=torch.float64, device="cuda")
    db.attach(d, dev)
    assert _noalloc()(None, db.Lower, ctypes.byref(d)) == -107   # DPLASMA_ERR_INTERNAL_LIMIT
