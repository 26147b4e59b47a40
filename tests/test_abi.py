"""CPU tests of the C ABI: the shared library loads, exports every function
declared in include/*.h, and its host-side logic (descriptors, tile offsets,
argument checks that return before any device work) behaves like the
reference wrappers.  No GPU is needed."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import dplasma_b200 as db

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\([^;{]*\)\s*;", src, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "return"):
                names.add(name)
    return names


def test_library_exports_every_declared_symbol():
    L = db.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    # and the python binding covers them
    assert not [n for n in names if n not in db.EXPORTS]


def test_enum_values_match_reference_constants():
    # src/include/dplasma/constants.h:78-99
    assert (db.NoTrans, db.Trans, db.ConjTrans) == (111, 112, 113)
    assert (db.Upper, db.Lower, db.UpperLower) == (121, 122, 123)
    assert (db.NonUnit, db.Unit, db.Left, db.Right, db.InfNorm) == (131, 132, 141, 142, 175)


def test_descriptor_fields():
    d = db.desc_sym(1000, 256, db.Lower)
    assert (d.m, d.n, d.mb, d.nb, d.mt, d.nt, d.lmt) == (1000, 1000, 256, 256, 4, 4, 4)
    assert d.bsiz == 256 * 256 and d.nb_local_tiles == 10
    g = db.desc_general(1000, 16, 256, 256)
    assert (g.mt, g.nt, g.nb_local_tiles, g.uplo) == (4, 1, 4, db.UpperLower)
    l = db.desc_general(100, 50, 32, 32, storage=db.STORAGE_LAPACK, lda=120)
    assert db.desc_elems(l) == 120 * 50


def test_tile_offset_rules():
    mt = 5
    lo = db.desc_sym(mt * 64, 64, db.Lower)
    up = db.desc_sym(mt * 64, 64, db.Upper)
    full = db.desc_general(mt * 64, mt * 64, 64, 64)
    seen_lo, seen_up = set(), set()
    for n in range(mt):
        for m in range(mt):
            assert db.tile_offset(full, m, n) == (m + n * mt) * 64 * 64
            o = db.tile_offset(lo, m, n)
            if m < n:
                assert o == -1
            else:
                assert o == (n * mt - n * (n - 1) // 2 + (m - n)) * 4096
                seen_lo.add(o)
            o = db.tile_offset(up, m, n)
            if m > n:
                assert o == -1
            else:
                seen_up.add(o)
    assert sorted(seen_lo) == [i * 4096 for i in range(15)]
    assert sorted(seen_up) == [i * 4096 for i in range(15)]


@pytest.mark.parametrize("kind", ["lower", "upper", "full", "lapack"])
def test_pack_unpack_roundtrip(kind):
    N, NB = 300, 64
    A = np.arange(N * N, dtype=np.float64).reshape(N, N, order="F")
    if kind == "lower":
        d = db.desc_sym(N, NB, db.Lower)
    elif kind == "upper":
        d = db.desc_sym(N, NB, db.Upper)
    elif kind == "full":
        d = db.desc_general(N, N, NB, NB)
    else:
        d = db.desc_general(N, N, NB, NB, storage=db.STORAGE_LAPACK, lda=N + 7)
    back = db.unpack(db.pack(A, d), d, fill=np.nan)
    m = ~np.isnan(back)
    assert np.array_equal(back[m], A[m])
    if kind == "lower":
        assert m[np.tril_indices(N)].all()
    if kind in ("full", "lapack"):
        assert m.all()


def test_argument_checks_without_a_device():
    L = db.lib()
    d = db.desc_sym(100, 32, db.Lower)
    b = db.desc_general(100, 4, 32, 32)
    buf = np.zeros(db.desc_elems(d))
    db.attach(d, buf)
    bb = np.zeros(db.desc_elems(b))
    db.attach(b, bb)
    pd = ctypes.byref
    # bad uplo first, as src/zpotrs_wrapper.c:63-66 and src/zposv_wrapper.c:72-75
    assert L.dplasma_dpotrf(None, 999, pd(d)) == -1
    assert L.dplasma_dpotrs(None, 999, pd(d), pd(b)) == -1
    assert L.dplasma_dposv(None, 999, pd(d), pd(b)) == -1
    info = ctypes.c_int(5)
    assert L.dplasma_dpotrf_New(999, pd(d), pd(info)) is None   # src/zpotrf_wrapper.c:207-210
    # dtrsm: -1..-4 for bad enums, -6 for shapes (src/ztrsm_wrapper.c:73-109)
    assert L.dplasma_dtrsm(None, 7, db.Lower, db.NoTrans, db.NonUnit, 1.0, pd(d), pd(b)) == -1
    assert L.dplasma_dtrsm(None, db.Left, 7, db.NoTrans, db.NonUnit, 1.0, pd(d), pd(b)) == -2
    assert L.dplasma_dtrsm(None, db.Left, db.Lower, 7, db.NonUnit, 1.0, pd(d), pd(b)) == -3
    assert L.dplasma_dtrsm(None, db.Left, db.Lower, db.NoTrans, 7, 1.0, pd(d), pd(b)) == -4
    b2 = db.desc_general(99, 4, 32, 32)
    assert L.dplasma_dtrsm(None, db.Left, db.Lower, db.NoTrans, db.NonUnit, 1.0, pd(d), pd(b2)) == -6
    assert L.dplasma_dtrsm(None, db.Right, db.Lower, db.NoTrans, db.NonUnit, 1.0, pd(d), pd(b)) == -6
    br = db.desc_general(4, 100, 32, 32)
    assert L.dplasma_dtrsm(None, db.Right, db.Lower, db.NoTrans, db.NonUnit, 1.0, pd(d), pd(br)) == db.ERR_NOT_SUPPORTED
    assert L.dplasma_dplgsy(None, 1.0, 999, pd(d), 1) == -3
    # mixed-precision solve: uplo first, then the options, then the context
    x = db.desc_general(100, 4, 32, 32)
    db.attach(x, np.zeros(db.desc_elems(x)))
    it = ctypes.c_int(7)
    assert L.dplasma_dsposv(None, 999, pd(d), pd(b), pd(x), pd(it)) == -1
    o = db.RefineOpts()
    L.dplasma_b200_refine_opts_default(pd(o))
    assert (o.fmt, o.solver, o.itermax, o.gmres_m, o.gmres_tol, o.bwdmax, o.escalate) == \
        (db.FP16, db.IR_AUTO, 30, 30, 1e-4, 1.0, 1)
    st = db.RefineStats()
    bad = db.RefineOpts()
    L.dplasma_b200_refine_opts_default(pd(bad))
    bad.fmt = 5
    assert L.dplasma_b200_dsposv_ex(None, db.Lower, pd(d), pd(b), pd(x), pd(bad), pd(st)) == db.ERR_ILLEGAL_VALUE
    assert L.dplasma_b200_dsposv_ex(None, db.Lower, pd(d), pd(b), pd(x), pd(o), pd(st)) == db.ERR_NOT_INITIALIZED
    assert L.dplasma_dsposv(None, db.Lower, pd(d), pd(b), pd(x), pd(it)) == db.ERR_NOT_INITIALIZED
    # valid arguments without a context
    assert L.dplasma_dpotrf(None, db.Lower, pd(d)) == db.ERR_NOT_INITIALIZED
    assert L.dplasma_dposv(None, db.Lower, pd(d), pd(b)) == db.ERR_NOT_INITIALIZED
    assert L.dplasma_b200_taskpool_run(None, None) == db.ERR_NOT_INITIALIZED


def test_pdpotrf_argument_checks_without_a_device():
    """ScaLAPACK PDPOTRF's INFO codes for illegal arguments (-i for scalar
    argument i, -(100 i + j) for entry j of array argument i), returned before
    any device work; N = 0 is a no-op."""
    N, NB = 64, 16
    a = np.asfortranarray(np.eye(N))
    good = [1, 0, N, N, NB, NB, 0, 0, N]

    def info(uplo="L", n=N, ia=1, ja=1, desc=None):
        return db.pdpotrf(uplo, n, a, ia, ja, good if desc is None else desc)

    def with_(j, v):
        d = list(good)
        d[j] = v
        return d

    assert info(desc=with_(0, 2)) == -601          # DTYPE
    assert info(uplo="X") == -1
    assert info(n=-1) == -2
    assert info(ia=0) == -4
    assert info(ja=0) == -5
    assert info(desc=with_(4, 0)) == -605          # MB
    assert info(desc=with_(5, 0)) == -606          # NB
    assert info(desc=with_(6, 1)) == -607          # RSRC: one process owns the matrix
    assert info(desc=with_(7, 1)) == -608          # CSRC
    assert info(desc=with_(8, N - 1)) == -609      # LLD < M
    assert info(ia=2, n=N - 1) == -4               # not on a block boundary
    assert info(ja=2, n=N - 1) == -5
    assert info(ia=NB + 1) == -603                 # IA + N - 1 > M
    assert info(ja=NB + 1) == -604
    assert info(desc=with_(4, 8)) == -606          # MB != NB
    assert np.array_equal(a, np.eye(N))
    assert info(n=0) == 0


def test_python_side_refuses_without_gpu_library_context():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError):
        db.Context(0)


def test_failure_hooks_check_arguments_without_a_context():
    L = db.lib()
    assert L.dplasma_b200_inject_fault(None, db.INJECT_TASK_FAILED, 0) == db.ERR_NOT_INITIALIZED
    assert L.dplasma_b200_set_wait_limits(None, 10, 10) == db.ERR_NOT_INITIALIZED
    assert L.dplasma_b200_set_selfcheck(None, 1) == db.ERR_NOT_INITIALIZED
    assert L.dplasma_b200_selfcheck(None, None, None, None) == db.ERR_NOT_INITIALIZED
