"""Python host side of the B200 tile-Cholesky library.

A thin ctypes layer over the C ABI in ``include/dplasma_b200.h``
(``dplasma_b200/libdplasma_b200.so``).  It mirrors the dplasma calls of the
Cholesky path -- ``dplasma_dpotrf``, ``dplasma_dpotrs``, ``dplasma_dposv``,
``dplasma_dtrsm``, ``dplasma_dplgsy``, ``dplasma_dplrnt`` -- with the same
argument meaning, enum values and return codes (INFO > 0 for a non positive
definite leading minor, negative values for bad arguments), and adds helpers
to lay numpy arrays out as dplasma tile descriptors.

Every numerical call runs on the GPU through the shared library; when the
library or a CUDA device is missing the calls raise instead of computing
anything on the host.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdplasma_b200.so")

# enum values: src/include/dplasma/constants.h:78-99
NoTrans, Trans, ConjTrans = 111, 112, 113
Upper, Lower, UpperLower = 121, 122, 123
NonUnit, Unit = 131, 132
Left, Right = 141, 142
OneNorm, FrobeniusNorm, InfNorm, MaxNorm = 171, 174, 175, 177
MATRIX_DOUBLE = 3
STORAGE_LAPACK, STORAGE_TILE = 0, 1
HOST, DEVICE = 0, 1
ERR_NOT_INITIALIZED, ERR_NOT_SUPPORTED, ERR_ILLEGAL_VALUE = -101, -103, -104


class Desc(ctypes.Structure):
    """parsec_tiled_matrix_t as declared in include/dplasma_b200.h."""

    _fields_ = [(n, ctypes.c_int) for n in (
        "mtype", "storage", "uplo", "mb", "nb", "lm", "ln", "i", "j", "m", "n", "mt", "nt", "lmt", "lnt", "lda",
        "location")] + [("bsiz", ctypes.c_size_t), ("nb_local_tiles", ctypes.c_size_t), ("mat", ctypes.c_void_p)]


class RefineOpts(ctypes.Structure):
    """dplasma_b200_refine_opts_t."""

    _fields_ = [("fmt", ctypes.c_int), ("solver", ctypes.c_int), ("itermax", ctypes.c_int), ("gmres_m", ctypes.c_int),
                ("gmres_tol", ctypes.c_double), ("bwdmax", ctypes.c_double), ("escalate", ctypes.c_int),
                ("shift", ctypes.c_double)]


class RefineStats(ctypes.Structure):
    """dplasma_b200_refine_stats_t."""

    _fields_ = [("iter", ctypes.c_int), ("inner_iters", ctypes.c_int), ("fallback", ctypes.c_int),
                ("solver_used", ctypes.c_int), ("fmt_used", ctypes.c_int), ("backward_error", ctypes.c_double), ("factor_ms", ctypes.c_double),
                ("refine_ms", ctypes.c_double), ("anorm", ctypes.c_double)]


FP16, BF16, FP16_SPLIT = 0, 1, 2
IR_AUTO, IR_PLAIN, IR_GMRES = 0, 1, 2

_lib = None

EXPORTS = (
    "dplasma_b200_tile_offset", "dplasma_b200_desc_init", "dplasma_b200_sym_desc_init", "dplasma_b200_init",
    "dplasma_b200_fini", "dplasma_b200_last_error", "dplasma_dpotrf", "dplasma_dpotrf_New",
    "dplasma_dpotrf_Destruct", "dplasma_b200_taskpool_run", "dplasma_dpotrf_rec", "dplasma_dpotrf_setrecursive",
    "dplasma_dpotrs", "dplasma_dposv", "dplasma_dtrsm", "dplasma_dplgsy", "dplasma_dplrnt", "dplasma_dlansy",
    "dplasma_b200_last_factor_ms", "dplasma_b200_last_solve_ms", "dplasma_b200_last_launches",
    "dplasma_b200_fp64_peak_tflops", "dplasma_b200_refine_opts_default", "dplasma_dsposv",
    "dplasma_b200_dsposv_ex", "dplasma_b200_dplgsy_cond", "dplasma_b200_dposv_batched",
    "dplasma_b200_sposv_batched", "dplasma_b200_batched_variant", "dplasma_dpotrf_adjoint",
    "dplasma_dtrtri", "dplasma_dlauum", "dplasma_dpotri", "dplasma_dpoinv", "dplasma_dpoinv_sync",
    "dplasma_b200_dpotri_batched", "pdpotrf_", "dplasma_b200_dpotrf_noalloc", "dplasma_b200_inject_fault",
    "dplasma_b200_set_wait_limits", "dplasma_b200_set_selfcheck", "dplasma_b200_selfcheck", "dplasma_dlange",
    "dplasma_dsymm", "dplasma_b200_dtd_new", "dplasma_b200_dtd_insert", "dplasma_b200_dtd_panel_received",
    "dplasma_b200_dtd_flush", "dplasma_b200_dtd_data_flush_all", "dplasma_b200_dtd_tiles",
    "dplasma_b200_dtd_tickets", "dplasma_b200_dtd_destruct", "dplasma_dpotrf_dtd",
)
TASK_POTRF, TASK_TRSM, TASK_SYRK, TASK_GEMM = 1, 2, 3, 4
INJECT_NONE, INJECT_TASK_FAILED, INJECT_WITHHOLD = 0, 1, 2


def lib():
    """Load the shared library (build it first if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(LIB_PATH)
    P, I, D, U64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong
    pd = ctypes.POINTER(Desc)
    L.dplasma_b200_tile_offset.restype = ctypes.c_int64
    L.dplasma_b200_tile_offset.argtypes = [pd, I, I]
    L.dplasma_b200_desc_init.argtypes = [pd, I, I, I, I, I, I, I, I, I, I]
    L.dplasma_b200_sym_desc_init.argtypes = [pd, I, I, I, I, I, I, I, I, I, I]
    L.dplasma_b200_init.restype = P
    L.dplasma_b200_init.argtypes = [I]
    L.dplasma_b200_fini.argtypes = [ctypes.POINTER(P)]
    L.dplasma_b200_last_error.restype = ctypes.c_char_p
    L.dplasma_b200_last_error.argtypes = [P]
    L.dplasma_dpotrf.argtypes = [P, I, pd]
    L.dplasma_dpotrf_New.restype = P
    L.dplasma_dpotrf_New.argtypes = [I, pd, ctypes.POINTER(I)]
    L.dplasma_dpotrf_Destruct.argtypes = [P]
    L.dplasma_b200_taskpool_run.argtypes = [P, P]
    L.dplasma_dpotrf_rec.argtypes = [P, I, pd, I]
    L.dplasma_dpotrf_setrecursive.argtypes = [P, I]
    L.dplasma_dpotrs.argtypes = [P, I, pd, pd]
    L.dplasma_dposv.argtypes = [P, I, pd, pd]
    L.dplasma_dtrsm.argtypes = [P, I, I, I, I, D, pd, pd]
    L.dplasma_dplgsy.argtypes = [P, D, I, pd, U64]
    L.dplasma_dplrnt.argtypes = [P, I, pd, U64]
    L.dplasma_dlansy.restype = D
    L.dplasma_dlansy.argtypes = [P, I, I, pd]
    for f in ("dplasma_b200_last_factor_ms", "dplasma_b200_last_solve_ms"):
        getattr(L, f).restype = D
        getattr(L, f).argtypes = [P]
    L.dplasma_b200_last_launches.argtypes = [P]
    L.dplasma_b200_fp64_peak_tflops.restype = D
    L.dplasma_b200_fp64_peak_tflops.argtypes = [P]
    L.dplasma_b200_dplgsy_cond.argtypes = [P, D, I, I, pd, U64]
    for f in ("dplasma_b200_dposv_batched", "dplasma_b200_sposv_batched"):
        getattr(L, f).argtypes = [P, I, P, P, P, P, I, P, P]
    L.dplasma_dpotrf_adjoint.argtypes = [P, I, pd, pd]
    L.dplasma_dtrtri.argtypes = [P, I, I, pd]
    for f in ("dplasma_dlauum", "dplasma_dpotri", "dplasma_dpoinv", "dplasma_dpoinv_sync"):
        getattr(L, f).argtypes = [P, I, pd]
    L.dplasma_b200_dpotri_batched.argtypes = [P, I, P, P, P, P]
    pi = ctypes.POINTER(I)
    L.pdpotrf_.restype = None
    L.pdpotrf_.argtypes = [ctypes.c_char_p, pi, P, pi, pi, pi, pi]
    L.dplasma_b200_batched_variant.restype = ctypes.c_char_p
    L.dplasma_b200_batched_variant.argtypes = [P]
    L.dplasma_b200_refine_opts_default.argtypes = [ctypes.POINTER(RefineOpts)]
    L.dplasma_dsposv.argtypes = [P, I, pd, pd, pd, ctypes.POINTER(I)]
    L.dplasma_b200_dsposv_ex.argtypes = [P, I, pd, pd, pd, ctypes.POINTER(RefineOpts), ctypes.POINTER(RefineStats)]
    L.dplasma_dlange.restype = D
    L.dplasma_dlange.argtypes = [P, I, pd]
    L.dplasma_dsymm.argtypes = [P, I, I, D, pd, pd, D, pd]
    L.dplasma_b200_dtd_new.restype = P
    L.dplasma_b200_dtd_new.argtypes = [P, I, pd]
    L.dplasma_b200_dtd_insert.argtypes = [P, I, I, I, I]
    L.dplasma_b200_dtd_panel_received.argtypes = [P, I]
    for f in ("dplasma_b200_dtd_flush", "dplasma_b200_dtd_data_flush_all", "dplasma_b200_dtd_destruct"):
        getattr(L, f).argtypes = [P]
    L.dplasma_b200_dtd_tiles.restype = P
    L.dplasma_b200_dtd_tiles.argtypes = [P]
    L.dplasma_b200_dtd_tickets.restype = ctypes.c_longlong
    L.dplasma_b200_dtd_tickets.argtypes = [P]
    L.dplasma_dpotrf_dtd.argtypes = [P, I, pd]
    L.dplasma_b200_inject_fault.argtypes = [P, I, I]
    L.dplasma_b200_set_wait_limits.argtypes = [P, I, I]
    L.dplasma_b200_set_selfcheck.argtypes = [P, I]
    pll = ctypes.POINTER(ctypes.c_longlong)
    L.dplasma_b200_selfcheck.argtypes = [P, pll, pll, pll]
    _lib = L
    return L


# ---------------------------------------------------------------------------
# descriptors over numpy / device buffers
# ---------------------------------------------------------------------------
def desc_general(m: int, n: int, mb: int, nb: int, storage: int = STORAGE_TILE, lda: int | None = None) -> Desc:
    d = Desc()
    lib().dplasma_b200_desc_init(ctypes.byref(d), MATRIX_DOUBLE, storage, mb, nb, m, n, 0, 0, m, n)
    if storage == STORAGE_LAPACK and lda is not None:
        d.lda = lda
        d.lm = lda
    return d


def desc_sym(n: int, nb: int, uplo: int) -> Desc:
    d = Desc()
    lib().dplasma_b200_sym_desc_init(ctypes.byref(d), MATRIX_DOUBLE, nb, nb, n, n, 0, 0, n, n, uplo)
    return d


def desc_elems(d: Desc) -> int:
    return d.lda * d.ln if d.storage == STORAGE_LAPACK else d.bsiz * d.nb_local_tiles


def tile_offset(d: Desc, m: int, n: int) -> int:
    return lib().dplasma_b200_tile_offset(ctypes.byref(d), m, n)


def _tiles(d: Desc):
    for n in range(d.nt):
        for m in range(d.mt):
            off = tile_offset(d, m, n)
            if off < 0:
                continue
            tm = d.m - m * d.mb if m == d.mt - 1 else d.mb
            tn = d.n - n * d.nb if n == d.nt - 1 else d.nb
            yield m, n, off, tm, tn


def pack(dense: np.ndarray, d: Desc, buf: np.ndarray | None = None) -> np.ndarray:
    """Lay a dense (m x n) array out in descriptor d's storage (tiles of the
    stored triangle only for symmetric storage); returns the flat buffer."""
    if buf is None:
        buf = np.zeros(desc_elems(d), dtype=np.float64)
    if d.storage == STORAGE_LAPACK:
        v = buf[: d.lda * d.n].reshape(d.n, d.lda).T
        v[: d.m, : d.n] = dense
        return buf
    for m, n, off, tm, tn in _tiles(d):
        t = buf[off: off + d.bsiz].reshape(d.nb, d.mb).T
        t[:tm, :tn] = dense[m * d.mb: m * d.mb + tm, n * d.nb: n * d.nb + tn]
    return buf


def unpack(buf: np.ndarray, d: Desc, fill: float = 0.0) -> np.ndarray:
    """Inverse of pack: dense (m x n) array; entries of unstored tiles = fill."""
    out = np.full((d.m, d.n), fill, dtype=np.float64, order="F")
    if d.storage == STORAGE_LAPACK:
        out[:, :] = buf[: d.lda * d.n].reshape(d.n, d.lda).T[: d.m, : d.n]
        return out
    for m, n, off, tm, tn in _tiles(d):
        t = buf[off: off + d.bsiz].reshape(d.nb, d.mb).T
        out[m * d.mb: m * d.mb + tm, n * d.nb: n * d.nb + tn] = t[:tm, :tn]
    return out


# ---------------------------------------------------------------------------
# context and calls
# ---------------------------------------------------------------------------
class Context:
    """One GPU, one stream and its device workspace (the parsec_context_t
    argument of the dplasma calls)."""

    def __init__(self, device: int = 0):
        self.h = lib().dplasma_b200_init(device)
        if not self.h:
            raise RuntimeError("dplasma_b200_init failed: no usable CUDA device")

    def close(self):
        if self.h:
            h = ctypes.c_void_p(self.h)
            lib().dplasma_b200_fini(ctypes.byref(h))
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- instrumentation
    def last_error(self) -> str:
        return lib().dplasma_b200_last_error(self.h).decode()

    def last_factor_ms(self) -> float:
        return lib().dplasma_b200_last_factor_ms(self.h)

    def last_solve_ms(self) -> float:
        return lib().dplasma_b200_last_solve_ms(self.h)

    def last_launches(self) -> int:
        return lib().dplasma_b200_last_launches(self.h)

    def fp64_peak_tflops(self) -> float:
        return lib().dplasma_b200_fp64_peak_tflops(self.h)

    # -- failure detection
    def inject_fault(self, kind: int, arg: int) -> int:
        return lib().dplasma_b200_inject_fault(self.h, kind, arg)

    def set_wait_limits(self, dep_ms: int, pipe_ms: int) -> int:
        return lib().dplasma_b200_set_wait_limits(self.h, dep_ms, pipe_ms)

    def set_selfcheck(self, on: bool) -> int:
        return lib().dplasma_b200_set_selfcheck(self.h, 1 if on else 0)

    def selfcheck(self):
        """(tickets, task runs, tickets not run exactly once) of the last
        factorization, or None when the self check is off."""
        t, r, b = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        rc = lib().dplasma_b200_selfcheck(self.h, ctypes.byref(t), ctypes.byref(r), ctypes.byref(b))
        return None if rc else (t.value, r.value, b.value)

    # -- the dplasma calls (descriptor `mat` must be set by the caller)
    def dpotrf(self, uplo: int, A: Desc) -> int:
        return lib().dplasma_dpotrf(self.h, uplo, ctypes.byref(A))

    def dpotrs(self, uplo: int, A: Desc, B: Desc) -> int:
        return lib().dplasma_dpotrs(self.h, uplo, ctypes.byref(A), ctypes.byref(B))

    def dposv(self, uplo: int, A: Desc, B: Desc) -> int:
        return lib().dplasma_dposv(self.h, uplo, ctypes.byref(A), ctypes.byref(B))

    def dtrsm(self, side: int, uplo: int, trans: int, diag: int, alpha: float, A: Desc, B: Desc) -> int:
        return lib().dplasma_dtrsm(self.h, side, uplo, trans, diag, alpha, ctypes.byref(A), ctypes.byref(B))

    def dplgsy(self, bump: float, uplo: int, A: Desc, seed: int) -> int:
        return lib().dplasma_dplgsy(self.h, bump, uplo, ctypes.byref(A), seed)

    def dplrnt(self, diagdom: int, A: Desc, seed: int) -> int:
        return lib().dplasma_dplrnt(self.h, diagdom, ctypes.byref(A), seed)

    def dlansy(self, ntype: int, uplo: int, A: Desc) -> float:
        return lib().dplasma_dlansy(self.h, ntype, uplo, ctypes.byref(A))

    def dpotrf_dtd(self, uplo: int, A: Desc) -> int:
        return lib().dplasma_dpotrf_dtd(self.h, uplo, ctypes.byref(A))

    def dtd(self, uplo: int, A: Desc) -> "TaskPool":
        return TaskPool(self, uplo, A)

    def dlange(self, ntype: int, A: Desc) -> float:
        return lib().dplasma_dlange(self.h, ntype, ctypes.byref(A))

    def dsymm(self, side: int, uplo: int, alpha: float, A: Desc, B: Desc, beta: float, C: Desc) -> int:
        return lib().dplasma_dsymm(self.h, side, uplo, alpha, ctypes.byref(A), ctypes.byref(B), beta, ctypes.byref(C))

    def check_daxmb(self, uplo: int, A: Desc, B: Desc, X: Desc, R: Desc) -> float:
        """The reference's check_zaxmb (src/dplasma_zcheck.c:179-224) on the GPU:
        ||B - A X||_inf / ((||A||_inf ||X||_inf + ||B||_inf) N eps).  R must be a
        descriptor shaped like B holding a copy of B; it receives B - A X."""
        an = self.dlansy(InfNorm, uplo, A)
        bn = self.dlange(InfNorm, B)
        xn = self.dlange(InfNorm, X)
        rc = self.dsymm(Left, uplo, -1.0, A, X, 1.0, R)
        if rc != 0 or min(an, bn, xn) < 0:
            raise RuntimeError(f"check_daxmb on the GPU failed (rc={rc}): {self.last_error()}")
        rn = self.dlange(InfNorm, R)
        return rn / ((an * xn + bn) * A.n * 2.0 ** -53)

    def posv_batched(self, mats, rhs=None, keep=None):
        """Batched Cholesky + solve + log-det (dplasma_b200_dposv_batched or
        _sposv_batched by dtype) of CUDA tensors.  mats: list of (n, n)
        symmetric float64 or float32 tensors (contiguous; the column-major lower
        triangle is the row-major upper one, so a symmetric matrix reads the
        same), overwritten by L^T in row-major view; rhs: None or a list of
        (nrhs, n) or (n,) tensors (column-major n x nrhs), overwritten by the
        solutions.  Returns (info, logdet) as CPU tensors.  `keep` receives the
        device argument arrays (to replay the recorded launch, pass the same
        ones again through posv_batched_arrays)."""
        import torch
        batch = len(mats)
        dt = mats[0].dtype if batch else torch.float64
        dev = mats[0].device if batch else torch.device("cuda")
        n = torch.tensor([m.shape[0] for m in mats], dtype=torch.int32, device=dev)
        A = torch.tensor([m.data_ptr() for m in mats], dtype=torch.int64, device=dev)
        B = None
        nrhs = 0
        if rhs is not None:
            B = torch.tensor([r.data_ptr() for r in rhs], dtype=torch.int64, device=dev)
            nrhs = 1 if rhs[0].dim() == 1 else rhs[0].shape[0]
        logdet = torch.empty(batch, dtype=torch.float64, device=dev)
        info = torch.empty(batch, dtype=torch.int32, device=dev)
        args = (n, n, A, B, nrhs, logdet, info)
        if keep is not None:
            keep.extend(args)
        torch_ready(*mats, *(rhs or []), n, A, B)
        rc = self.posv_batched_arrays(dt, batch, *args)
        if rc != 0:
            raise RuntimeError(f"posv_batched rc={rc}: {self.last_error()}")
        return info.cpu(), logdet.cpu()

    def posv_batched_arrays(self, dtype, batch, n, lda, A, B, nrhs, logdet, info) -> int:
        """The C call on prepared device arrays (torch tensors)."""
        import torch
        torch_ready(n, A)
        f = lib().dplasma_b200_dposv_batched if dtype == torch.float64 else lib().dplasma_b200_sposv_batched
        return f(self.h, batch, n.data_ptr(), lda.data_ptr(), A.data_ptr(), B.data_ptr() if B is not None else None,
                 nrhs, logdet.data_ptr(), info.data_ptr())

    def potri_batched(self, mats):
        """dplasma_b200_dpotri_batched on float64 CUDA tensors holding factors
        (column-major lower = row-major upper, as posv_batched leaves them):
        each becomes the inverse (column-major lower).  Returns info (CPU)."""
        import torch
        batch = len(mats)
        dev = mats[0].device if batch else torch.device("cuda")
        n = torch.tensor([m.shape[0] for m in mats], dtype=torch.int32, device=dev)
        A = torch.tensor([m.data_ptr() for m in mats], dtype=torch.int64, device=dev)
        info = torch.empty(batch, dtype=torch.int32, device=dev)
        torch_ready(*mats, n, A)
        rc = lib().dplasma_b200_dpotri_batched(self.h, batch, n.data_ptr(), n.data_ptr(), A.data_ptr(),
                                               info.data_ptr())
        if rc != 0:
            raise RuntimeError(f"potri_batched rc={rc}: {self.last_error()}")
        return info.cpu()

    def batched_variant(self) -> str:
        return lib().dplasma_b200_batched_variant(self.h).decode()

    def dtrtri(self, uplo: int, diag: int, A: Desc) -> int:
        return lib().dplasma_dtrtri(self.h, uplo, diag, ctypes.byref(A))

    def dlauum(self, uplo: int, A: Desc) -> int:
        return lib().dplasma_dlauum(self.h, uplo, ctypes.byref(A))

    def dpotri(self, uplo: int, A: Desc) -> int:
        return lib().dplasma_dpotri(self.h, uplo, ctypes.byref(A))

    def dpoinv(self, uplo: int, A: Desc) -> int:
        return lib().dplasma_dpoinv(self.h, uplo, ctypes.byref(A))

    def dpotrf_adjoint(self, uplo: int, L: Desc, Lbar: Desc) -> int:
        return lib().dplasma_dpotrf_adjoint(self.h, uplo, ctypes.byref(L), ctypes.byref(Lbar))

    def dplgsy_cond(self, kappa: float, nrefl: int, uplo: int, A: Desc, seed: int) -> int:
        return lib().dplasma_b200_dplgsy_cond(self.h, kappa, nrefl, uplo, ctypes.byref(A), seed)

    def dsposv(self, uplo: int, A: Desc, B: Desc, X: Desc, fmt: int = FP16, solver: int = IR_AUTO,
               itermax: int = 30, gmres_m: int = 30, gmres_tol: float = 1e-4, bwdmax: float = 1.0,
               escalate: bool = True, shift: float = 0.0):
        """Mixed-precision solve (dplasma_b200_dsposv_ex): returns (rc, stats dict)."""
        o = RefineOpts()
        lib().dplasma_b200_refine_opts_default(ctypes.byref(o))
        o.fmt, o.solver, o.itermax, o.gmres_m, o.gmres_tol, o.bwdmax = fmt, solver, itermax, gmres_m, gmres_tol, bwdmax
        o.escalate = 1 if escalate else 0
        o.shift = shift
        st = RefineStats()
        rc = lib().dplasma_b200_dsposv_ex(self.h, uplo, ctypes.byref(A), ctypes.byref(B), ctypes.byref(X),
                                          ctypes.byref(o), ctypes.byref(st))
        return rc, {f: getattr(st, f) for f, _ in RefineStats._fields_}


class TaskPool:
    """Task insertion on the tiles of one matrix (dplasma_b200_dtd_*): insert
    POTRF / TRSM / SYRK / GEMM tile tasks in a sequential program order, flush
    to run them on the GPU.  Keeps the descriptor alive."""

    def __init__(self, ctx: Context, uplo: int, A: Desc):
        self.ctx, self.A = ctx, A
        self.h = lib().dplasma_b200_dtd_new(ctx.h, uplo, ctypes.byref(A))
        if not self.h:
            raise RuntimeError(f"dplasma_b200_dtd_new failed: {ctx.last_error()}")

    def insert(self, op: int, k: int, m: int = 0, n: int = 0) -> int:
        return lib().dplasma_b200_dtd_insert(self.h, op, k, m, n)

    def panel_received(self, k: int) -> int:
        return lib().dplasma_b200_dtd_panel_received(self.h, k)

    def flush(self) -> int:
        return lib().dplasma_b200_dtd_flush(self.h)

    def data_flush_all(self) -> int:
        return lib().dplasma_b200_dtd_data_flush_all(self.h)

    def tiles(self) -> int:
        return lib().dplasma_b200_dtd_tiles(self.h) or 0

    def tickets(self) -> int:
        return lib().dplasma_b200_dtd_tickets(self.h)

    def destruct(self) -> int:
        r = 0
        if self.h:
            r = lib().dplasma_b200_dtd_destruct(self.h)
            self.h = None
        return r

    def __del__(self):
        try:
            self.destruct()
        except Exception:
            pass


def torch_ready(*tensors):
    """The library runs on its own CUDA stream: wait for the work torch has
    queued on the tensors' current streams (the producers of our inputs)
    before a call.  The library's calls return with their results complete."""
    import torch
    seen = set()
    for t in tensors:
        if t is not None and getattr(t, "is_cuda", False):
            dev = t.device.index if t.device.index is not None else torch.cuda.current_device()
            if dev not in seen:
                seen.add(dev)
                torch.cuda.current_stream(dev).synchronize()


def attach(d: Desc, buf) -> Desc:
    """Point descriptor d at `buf`: a numpy array (host) or a torch CUDA tensor
    (device).  The caller keeps `buf` alive."""
    if isinstance(buf, np.ndarray):
        assert buf.dtype == np.float64 and buf.flags.c_contiguous and buf.size >= desc_elems(d)
        d.mat = buf.ctypes.data
        d.location = HOST
    else:  # torch tensor on the GPU
        assert buf.is_cuda and str(buf.dtype) == "torch.float64" and buf.is_contiguous() and buf.numel() >= desc_elems(d)
        d.mat = buf.data_ptr()
        d.location = DEVICE
    return d


def pdpotrf(uplo: str, n: int, a, ia: int, ja: int, desca) -> int:
    """ScaLAPACK's PDPOTRF through the library's pdpotrf_ entry: `a` is the
    local (here: whole) column-major array as a Fortran-ordered float64 numpy
    array, `desca` the 9 descriptor integers; returns INFO."""
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.f_contiguous):
        raise ValueError("a must be a Fortran-ordered float64 array")
    L = lib()
    c = ctypes.c_int
    d = (c * 9)(*[int(v) for v in desca])
    info = c(0)
    L.pdpotrf_(uplo.encode()[:1], ctypes.byref(c(n)), a.ctypes.data_as(ctypes.c_void_p), ctypes.byref(c(ia)),
               ctypes.byref(c(ja)), d, ctypes.byref(info))
    return info.value
