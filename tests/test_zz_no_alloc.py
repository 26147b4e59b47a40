"""GPU test of dplasma_b200_dpotrf_noalloc, the entry point for callers that
cannot allocate device memory (its scratch is a fixed array in the library's
device image).  It must give the factor that dplasma_dpotrf gives for the same
device-resident input, and the oracle's factor, on two calls in a row (the
second call finds the first call's scratch contents and must not depend on
them); a call must not change the device's free memory; a non positive
definite input must return INFO and leave the next call correct.

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


def _factor_noalloc(torch, host, N, NB):
    d = db.desc_sym(N, NB, db.Lower)
    dev = torch.from_numpy(host.copy()).cuda()
    db.attach(d, dev)
    torch.cuda.current_stream().synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    info = _noalloc()(ctypes.c_void_p(stream), db.Lower, ctypes.byref(d))
    return info, np.tril(db.unpack(dev.cpu().numpy(), d))


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
    L_orc = A0.copy(order="F")
    assert oracle.dpotrf(oracle.LOWER, L_orc, NB) == 0
    L_orc = np.tril(L_orc)
    for call in range(2):
        info, L = _factor_noalloc(torch, host, N, NB)
        assert info == 0
        err = np.linalg.norm(L - L_ref) / np.linalg.norm(L_ref)
        assert err <= FACTOR_TOL, (call, err)
        err_orc = np.linalg.norm(L - L_orc) / np.linalg.norm(L_orc)
        assert err_orc <= FACTOR_TOL, (call, err_orc)


def test_noalloc_allocates_nothing():
    torch = pytest.importorskip("torch")
    N, NB = 2048, 256
    A0 = oracle.dplgsy(N, NB, 3872)
    d = db.desc_sym(N, NB, db.Lower)
    host = db.pack(A0, d)
    dev = torch.from_numpy(host.copy()).cuda()
    db.attach(d, dev)
    f = _noalloc()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert f(stream, db.Lower, ctypes.byref(d)) == 0      # first call: module and scratch look-up
    dev.copy_(torch.from_numpy(host))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert f(stream, db.Lower, ctypes.byref(d)) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_not_positive_definite_then_good_call():
    torch = pytest.importorskip("torch")
    N, NB = 2048, 256
    A0 = oracle.dplgsy(N, NB, 3872)
    d_ref = db.desc_sym(N, NB, db.Lower)
    host = db.pack(A0, d_ref)
    Abad = A0.copy(order="F")
    k = 700
    Abad[k, k] = -1.0
    Lbad = Abad.copy(order="F")
    info_orc = oracle.dpotrf(oracle.LOWER, Lbad, NB)
    assert info_orc == k + 1
    info, _ = _factor_noalloc(torch, db.pack(Abad, db.desc_sym(N, NB, db.Lower)), N, NB)
    assert info == info_orc
    # the aborted call left partial counters and inverses behind; the next one must not see them
    L_orc = A0.copy(order="F")
    assert oracle.dpotrf(oracle.LOWER, L_orc, NB) == 0
    L_orc = np.tril(L_orc)
    info, L = _factor_noalloc(torch, host, N, NB)
    assert info == 0
    assert np.linalg.norm(L - L_orc) / np.linalg.norm(L_orc) <= FACTOR_TOL


def test_noalloc_rejects_too_large():
    torch = pytest.importorskip("torch")
    N, NB = 8192 + 256, 256
    d = db.desc_sym(N, NB, db.Lower)
    dev = torch.zeros(db.desc_elems(d), dtype=torch.float64, device="cuda")
    db.attach(d, dev)
    assert _noalloc()(None, db.Lower, ctypes.byref(d)) == -107   # DPLASMA_ERR_INTERNAL_LIMIT


def test_noalloc_rejects_host_memory():
    N, NB = 1024, 256
    d = db.desc_sym(N, NB, db.Lower)
    buf = np.zeros(db.desc_elems(d))
    db.attach(d, buf)
    d.location = db.DEVICE          # claims device memory, points at host memory
    assert _noalloc()(None, db.Lower, ctypes.byref(d)) == db.ERR_ILLEGAL_VALUE
