"""GPU parity tests: the B200 library, called through its C ABI, against the
CPU oracle (a restatement of dplasma's tile algorithm over OpenBLAS, pinned to
the reference's own kernels in tests/test_oracle.py).

Bars (from the reference's checks, src/dplasma_zcheck.c, tightened):
  * generators bit-identical;
  * factor within 1e-12 relative Frobenius norm of the oracle factor;
  * ||LL^T - A||_inf / (||A||_inf N eps) < 10 and
    ||Ax - b||_inf / ((||A|| ||x|| + ||b||) N eps) < 10;
  * INFO identical for non positive definite input.
Shapes mirror the reference's ctest configurations (tests/Testings.cmake:
378/93, 874/76, 1700/320 ragged, 3200/320) and the workload configs, plus
edge cases N=1, N<NB, N=NB+-1, NRHS=1.
"""
import numpy as np
import pytest

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu

SEED_A, SEED_B = 3872, 3873
FACTOR_TOL = 1e-12
RATIO_TOL = 10.0


def tri(A, uplo):
    return np.tril(A) if uplo == db.Lower else np.triu(A)


def rel_fro(X, Y):
    ny = np.linalg.norm(Y)
    return np.linalg.norm(X - Y) / (ny if ny > 0 else 1.0)


def sym_desc_with(A0, NB, uplo):
    d = db.desc_sym(A0.shape[0], NB, uplo)
    buf = db.pack(A0, d)
    db.attach(d, buf)
    return d, buf


def gen_desc(B0, MB, NB):
    d = db.desc_general(B0.shape[0], B0.shape[1], MB, NB)
    buf = db.pack(B0, d)
    db.attach(d, buf)
    return d, buf


# ---------------------------------------------------------------------------
# generators
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("N,NB,region", [(378, 93, db.Lower), (378, 93, db.Upper), (378, 93, db.UpperLower),
                                         (1700, 320, db.Lower), (1, 1, db.Lower), (129, 128, db.UpperLower)])
def test_dplgsy_bitexact(gpu_ctx, N, NB, region):
    ref = oracle.dplgsy(N, NB, SEED_A)
    if region == db.UpperLower:
        d = db.desc_general(N, N, NB, NB)
    else:
        d = db.desc_sym(N, NB, region)
    buf = np.zeros(db.desc_elems(d))
    db.attach(d, buf)
    assert gpu_ctx.dplgsy(float(N), region, d, SEED_A) == 0
    got = db.unpack(buf, d, fill=np.nan)
    mask = ~np.isnan(got)
    assert mask.any()
    assert np.array_equal(got[mask], ref[mask])


@pytest.mark.parametrize("M,N,MB,NB,diagdom", [(378, 367, 93, 93, 0), (1000, 64, 256, 256, 0), (300, 300, 128, 64, 1)])
def test_dplrnt_bitexact(gpu_ctx, M, N, MB, NB, diagdom):
    ref = oracle.dplrnt(M, N, MB, NB, 2354, diagdom)
    d = db.desc_general(M, N, MB, NB)
    buf = np.zeros(db.desc_elems(d))
    db.attach(d, buf)
    assert gpu_ctx.dplrnt(diagdom, d, 2354) == 0
    assert np.array_equal(db.unpack(buf, d), ref)


# ---------------------------------------------------------------------------
# factorization
# ---------------------------------------------------------------------------
SHAPES = [(378, 93), (874, 76), (1700, 320), (3200, 320), (4096, 256), (1, 1), (1, 64), (7, 64), (127, 128),
          (128, 128), (129, 128), (515, 256), (1024, 512), (1152, 384)]


@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
@pytest.mark.parametrize("N,NB", SHAPES)
def test_dpotrf_parity(gpu_ctx, N, NB, uplo):
    A0 = oracle.dplgsy(N, NB, SEED_A)
    d, buf = sym_desc_with(A0, NB, uplo)
    info = gpu_ctx.dpotrf(uplo, d)
    assert info == 0, gpu_ctx.last_error()
    got = db.unpack(buf, d)
    ref = A0.copy(order="F")
    assert oracle.dpotrf(uplo, ref, NB) == 0
    assert rel_fro(tri(got, uplo), tri(ref, uplo)) <= FACTOR_TOL
    assert oracle.check_dpotrf(uplo, np.asfortranarray(got), A0) < RATIO_TOL
    # the other triangle of the diagonal tiles is left as it was
    other = np.triu(np.ones((N, N), bool), 1) if uplo == db.Lower else np.tril(np.ones((N, N), bool), -1)
    blk = np.zeros((N, N), bool)
    for k in range(0, N, NB):
        blk[k:k + NB, k:k + NB] = True
    assert np.array_equal(got[other & blk], A0[other & blk])


@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
def test_dpotrf_lapack_storage(gpu_ctx, uplo):
    N, NB, lda = 777, 128, 800
    A0 = oracle.dplgsy(N, NB, SEED_A)
    d = db.desc_general(N, N, NB, NB, storage=db.STORAGE_LAPACK, lda=lda)
    buf = db.pack(A0, d)
    db.attach(d, buf)
    assert gpu_ctx.dpotrf(uplo, d) == 0
    got = db.unpack(buf, d)
    ref = A0.copy(order="F")
    oracle.dpotrf(uplo, ref, NB)
    assert rel_fro(tri(got, uplo), tri(ref, uplo)) <= FACTOR_TOL
    # the other triangle is untouched
    off = np.triu(np.ones((N, N), bool), 1) if uplo == db.Lower else np.tril(np.ones((N, N), bool), -1)
    assert np.array_equal(got[off], A0[off])


@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
def test_dpotrf_full_grid_storage(gpu_ctx, uplo):
    N, NB = 600, 128
    A0 = oracle.dplgsy(N, NB, SEED_A)
    d, buf = gen_desc(A0, NB, NB)
    assert gpu_ctx.dpotrf(uplo, d) == 0
    got = db.unpack(buf, d)
    ref = A0.copy(order="F")
    oracle.dpotrf(uplo, ref, NB)
    assert rel_fro(tri(got, uplo), tri(ref, uplo)) <= FACTOR_TOL


@pytest.mark.parametrize("N,NB,bad", [(700, 128, 333), (512, 256, 0), (1000, 256, 999), (378, 93, 200)])
@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
def test_dpotrf_not_spd_info(gpu_ctx, N, NB, bad, uplo):
    A0 = oracle.dplgsy(N, NB, SEED_A)
    A0[bad, bad] = -float(N)
    d, buf = sym_desc_with(A0, NB, uplo)
    info = gpu_ctx.dpotrf(uplo, d)
    ref = A0.copy(order="F")
    rinfo = oracle.dpotrf(uplo, ref, NB)
    assert rinfo == bad + 1
    assert info == rinfo


def test_dpotrf_taskpool_api(gpu_ctx):
    import ctypes
    N, NB = 500, 128
    A0 = oracle.dplgsy(N, NB, SEED_A)
    d, buf = sym_desc_with(A0, NB, db.Lower)
    info = ctypes.c_int(-7)
    L = db.lib()
    tp = L.dplasma_dpotrf_New(db.Lower, ctypes.byref(d), ctypes.byref(info))
    assert tp and info.value == 0
    assert L.dplasma_b200_taskpool_run(gpu_ctx.h, tp) == 0
    L.dplasma_dpotrf_Destruct(tp)
    assert info.value == 0
    ref = A0.copy(order="F")
    oracle.dpotrf(db.Lower, ref, NB)
    assert rel_fro(np.tril(db.unpack(buf, d)), np.tril(ref)) <= FACTOR_TOL
    assert L.dplasma_dpotrf_New(999, ctypes.byref(d), ctypes.byref(info)) is None


# ---------------------------------------------------------------------------
# solves
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
@pytest.mark.parametrize("N,NB,NRHS", [(378, 93, 367), (1700, 320, 16), (4096, 256, 64), (129, 128, 1),
                                       (1, 1, 1), (1000, 256, 40)])
def test_dposv_parity(gpu_ctx, N, NB, NRHS, uplo):
    A0 = oracle.dplgsy(N, NB, SEED_A)
    B0 = oracle.dplrnt(N, NRHS, NB, NB, SEED_B)
    dA, bufA = sym_desc_with(A0, NB, uplo)
    dB, bufB = gen_desc(B0, NB, NB)
    assert gpu_ctx.dposv(uplo, dA, dB) == 0, gpu_ctx.last_error()
    X = db.unpack(bufB, dB)
    Aref, Xref = A0.copy(order="F"), B0.copy(order="F")
    assert oracle.dposv(uplo, Aref, Xref, NB) == 0
    assert rel_fro(X, Xref) <= FACTOR_TOL
    assert oracle.check_daxmb(uplo, A0, B0, np.asfortranarray(X)) < RATIO_TOL


@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
def test_dpotrf_then_dpotrs(gpu_ctx, uplo):
    N, NB, NRHS = 1100, 256, 16
    A0 = oracle.dplgsy(N, NB, SEED_A)
    B0 = oracle.dplrnt(N, NRHS, NB, NB, SEED_B)
    dA, bufA = sym_desc_with(A0, NB, uplo)
    assert gpu_ctx.dpotrf(uplo, dA) == 0
    dB, bufB = gen_desc(B0, NB, NB)
    assert gpu_ctx.dpotrs(uplo, dA, dB) == 0
    X = db.unpack(bufB, dB)
    assert oracle.check_daxmb(uplo, A0, B0, np.asfortranarray(X)) < RATIO_TOL


@pytest.mark.parametrize("uplo", [db.Lower, db.Upper])
@pytest.mark.parametrize("trans", [db.NoTrans, db.Trans])
@pytest.mark.parametrize("diag", [db.NonUnit, db.Unit])
def test_dtrsm_left_parity(gpu_ctx, uplo, trans, diag):
    N, NB, NRHS, alpha = 600, 128, 24, 1.5
    A0 = oracle.dplgsy(N, NB, SEED_A)
    F = A0.copy(order="F")
    oracle.dpotrf(uplo, F, NB)
    B0 = oracle.dplrnt(N, NRHS, NB, NB, SEED_B)
    dA, bufA = sym_desc_with(F, NB, uplo)
    dB, bufB = gen_desc(B0, NB, NB)
    assert gpu_ctx.dtrsm(db.Left, uplo, trans, diag, alpha, dA, dB) == 0
    X = db.unpack(bufB, dB)
    Xref = B0.copy(order="F")
    oracle.dtrsm_left(uplo, trans, diag, alpha, F, Xref, NB)
    assert rel_fro(X, Xref) <= FACTOR_TOL


# ---------------------------------------------------------------------------
# device-resident descriptors (torch-owned HBM), in place
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("N,NB", [(2048, 256), (1000, 256)])
def test_device_resident(gpu_ctx, N, NB):
    torch = pytest.importorskip("torch")
    A0 = oracle.dplgsy(N, NB, SEED_A)
    d = db.desc_sym(N, NB, db.Lower)
    host = db.pack(A0, d)
    dev = torch.from_numpy(host).cuda()
    db.attach(d, dev)
    assert gpu_ctx.dpotrf(db.Lower, d) == 0
    got = db.unpack(dev.cpu().numpy(), d)
    ref = A0.copy(order="F")
    oracle.dpotrf(db.Lower, ref, NB)
    assert rel_fro(np.tril(got), np.tril(ref)) <= FACTOR_TOL
    # device generator gives the same bits as the host one
    d2 = db.desc_sym(N, NB, db.Lower)
    dev2 = torch.zeros(db.desc_elems(d2), dtype=torch.float64, device="cuda")
    db.attach(d2, dev2)
    assert gpu_ctx.dplgsy(float(N), db.Lower, d2, SEED_A) == 0
    assert np.array_equal(np.tril(db.unpack(dev2.cpu().numpy(), d2)), np.tril(A0))


def test_dlansy_inf(gpu_ctx):
    N, NB = 900, 256
    A0 = oracle.dplgsy(N, NB, SEED_A)
    for uplo in (db.Lower, db.Upper):
        d, buf = sym_desc_with(A0, NB, uplo)
        v = gpu_ctx.dlansy(db.InfNorm, uplo, d)
        assert abs(v - oracle.lib().orc_dlansy_inf(uplo, N, A0.ctypes.data, N)) <= 1e-12 * v


def test_fp64_peak_probe(gpu_ctx):
    tf = gpu_ctx.fp64_peak_tflops()
    assert 5.0 < tf < 100.0
