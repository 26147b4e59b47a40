"""ctypes binding of the CPU oracle (``oracle/liboracle.so``) and of the
reference-kernel build (``oracle/_ref/libdplasma_ref.so``).

TEST INFRASTRUCTURE ONLY.  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this package, and only as the
checker.  The product library (``dplasma_b200``) never imports it.

Arrays are numpy float64 in Fortran (column-major) order, i.e. the LAPACK
layout; the oracle's tile algorithms block them by NB internally.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
REF_PATH = os.path.join(_HERE, "_ref", "libdplasma_ref.so")

UPPER, LOWER, UPPERLOWER = 121, 122, 123
NOTRANS, TRANS = 111, 112
NONUNIT, UNIT = 131, 132

_c_int, _c_dbl, _c_u64 = ctypes.c_int, ctypes.c_double, ctypes.c_uint64
_p = ctypes.c_void_p


def build(force: bool = False) -> None:
    """Compile liboracle.so (and oracle/_ref when the dplasma sources exist)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", _HERE])


def _load(path):
    lib = ctypes.CDLL(path)
    return lib


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = _load(LIB_PATH)
        L = _lib
        L.orc_rnd64_jump.restype = _c_u64
        L.orc_rnd64_jump.argtypes = [_c_u64, _c_u64]
        L.orc_dplgsy_tile.argtypes = [_c_dbl, _c_int, _c_int, _p, _c_int, _c_int, _c_int, _c_int, _c_u64]
        L.orc_dplrnt_tile.argtypes = [_c_int, _c_int, _p, _c_int, _c_int, _c_int, _c_int, _c_u64]
        L.orc_dplgsy.argtypes = [_c_dbl, _c_int, _c_int, _c_int, _p, _c_int, _c_u64]
        L.orc_dplrnt.argtypes = [_c_int, _c_int, _c_int, _c_int, _c_int, _p, _c_int, _c_u64]
        L.orc_dpotrf.argtypes = [_c_int, _c_int, _c_int, _p, _c_int]
        L.orc_dpotrf_parallel.argtypes = [_c_int, _c_int, _c_int, _p, _c_int, _c_int]
        L.orc_dtrsm_left.argtypes = [_c_int, _c_int, _c_int, _c_dbl, _c_int, _c_int, _c_int, _p, _c_int, _p, _c_int]
        L.orc_dpotrs.argtypes = [_c_int, _c_int, _c_int, _c_int, _p, _c_int, _p, _c_int]
        L.orc_dposv.argtypes = [_c_int, _c_int, _c_int, _c_int, _p, _c_int, _p, _c_int]
        L.orc_check_dpotrf.restype = _c_dbl
        L.orc_check_dpotrf.argtypes = [_c_int, _c_int, _p, _c_int, _p, _c_int, _p, _p]
        L.orc_check_daxmb.restype = _c_dbl
        L.orc_check_daxmb.argtypes = [_c_int, _c_int, _c_int, _p, _c_int, _p, _c_int, _p, _c_int]
        L.orc_dlansy_inf.restype = _c_dbl
        L.orc_dlansy_inf.argtypes = [_c_int, _c_int, _p, _c_int]
        L.orc_eps.restype = _c_dbl
        L.orc_set_blas_threads.argtypes = [_c_int]
    return _lib


def ref_available() -> bool:
    if not os.path.exists(REF_PATH):
        try:
            build(force=True)
        except Exception:
            return False
    return os.path.exists(REF_PATH)


def ref():
    """The reference's own CORE kernels (built from its sources), or None."""
    global _ref
    if _ref is None and ref_available():
        _ref = _load(REF_PATH)
        R = _ref
        R.ref_dplgsy_tile.argtypes = [_c_dbl, _c_int, _c_int, _p, _c_int, _c_int, _c_int, _c_int, _c_u64]
        R.ref_dplrnt_tile.argtypes = [_c_int, _c_int, _p, _c_int, _c_int, _c_int, _c_int, _c_u64]
        R.ref_dpotrf.argtypes = [_c_int, _c_int, _c_int, _p, _c_int]
        R.ref_dpotrf_parallel.argtypes = [_c_int, _c_int, _c_int, _p, _c_int, _c_int]
    return _ref


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(_p)


def dplgsy(N: int, NB: int, seed: int, bump: float | None = None, uplo: int = UPPERLOWER) -> np.ndarray:
    """Dense N x N matrix of dplasma_dplgsy(bump (default N), uplo, seed)."""
    A = np.zeros((N, N), dtype=np.float64, order="F")
    lib().orc_dplgsy(float(N if bump is None else bump), uplo, N, NB, _ptr(A), N, seed)
    return A


def dplrnt(M: int, N: int, MB: int, NB: int, seed: int, diagdom: int = 0) -> np.ndarray:
    B = np.zeros((M, N), dtype=np.float64, order="F")
    lib().orc_dplrnt(diagdom, M, N, MB, NB, _ptr(B), max(M, 1), seed)
    return B


def dpotrf(uplo: int, A: np.ndarray, NB: int) -> int:
    """In-place tile Cholesky of the dense array A; returns INFO."""
    N = A.shape[0]
    return lib().orc_dpotrf(uplo, N, NB, _ptr(A), max(N, 1))


def dpotrf_parallel(uplo: int, A: np.ndarray, NB: int, nthreads: int) -> int:
    N = A.shape[0]
    return lib().orc_dpotrf_parallel(uplo, N, NB, _ptr(A), max(N, 1), nthreads)


def dpotrs(uplo: int, A: np.ndarray, B: np.ndarray, NB: int) -> int:
    N, NRHS = B.shape
    return lib().orc_dpotrs(uplo, N, NRHS, NB, _ptr(A), max(N, 1), _ptr(B), max(N, 1))


def dposv(uplo: int, A: np.ndarray, B: np.ndarray, NB: int) -> int:
    N, NRHS = B.shape
    return lib().orc_dposv(uplo, N, NRHS, NB, _ptr(A), max(N, 1), _ptr(B), max(N, 1))


def dtrsm_left(uplo: int, trans: int, diag: int, alpha: float, A: np.ndarray, B: np.ndarray, NB: int) -> int:
    N, NRHS = B.shape
    return lib().orc_dtrsm_left(uplo, trans, diag, alpha, N, NRHS, NB, _ptr(A), max(N, 1), _ptr(B), max(N, 1))


def check_dpotrf(uplo: int, L: np.ndarray, A0: np.ndarray) -> float:
    """||LL^T - A0||_inf / (||A0||_inf N eps) -- src/dplasma_zcheck.c:63-133."""
    N = A0.shape[0]
    return lib().orc_check_dpotrf(uplo, N, _ptr(L), max(N, 1), _ptr(A0), max(N, 1), None, None)


def check_daxmb(uplo: int, A0: np.ndarray, B: np.ndarray, X: np.ndarray) -> float:
    """||B - A0 X||_inf / ((||A0|| ||X|| + ||B||) N eps) -- src/dplasma_zcheck.c:179-224."""
    N, NRHS = B.shape
    return lib().orc_check_daxmb(uplo, N, NRHS, _ptr(A0), max(N, 1), _ptr(B), max(N, 1), _ptr(X), max(N, 1))


def eps() -> float:
    return lib().orc_eps()


def set_blas_threads(n: int) -> None:
    lib().orc_set_blas_threads(n)
