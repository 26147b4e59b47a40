"""Failure detection of the device scheduler, tested without faulting the GPU.

The reference's failure paths are INFO > 0 for a non positive definite minor
(src/zpotrf_L.jdf:200-202) and PARSEC_HOOK_RETURN_ERROR from a task body
(src/zpotrf_L.jdf:136,261,390,530).  Here every device wait is bounded; the
failures are made on the host:
  * a task reported failed (dplasma_b200_inject_fault TASK_FAILED): the
    scheduler stops and the call returns DPLASMA_ERR_UNEXPECTED;
  * a withheld dependency (one ticket taken and dropped): the dependent tasks'
    waits run out after the short limit set here, the call returns
    DPLASMA_ERR_UNEXPECTED naming the dependency wait;
and after each, a clean call on the same context must give the oracle's
factor.  The self check counts the runs of every ticket on the device."""
import time

import numpy as np
import pytest

import oracle
import dplasma_b200 as db

pytestmark = pytest.mark.gpu
ERR_UNEXPECTED = -110
FACTOR_TOL = 1e-12


def _dev_matrix(torch, A0, NB):
    d = db.desc_sym(A0.shape[0], NB, db.Lower)
    buf = torch.from_numpy(db.pack(A0, d)).cuda()
    db.attach(d, buf)
    return d, buf


def _oracle_factor(A0, NB):
    L = A0.copy(order="F")
    assert oracle.dpotrf(oracle.LOWER, L, NB) == 0
    return np.tril(L)


def _clean_call_matches(ctx, torch, A0, NB, Lref):
    d, buf = _dev_matrix(torch, A0, NB)
    assert ctx.dpotrf(db.Lower, d) == 0, ctx.last_error()
    L = np.tril(db.unpack(buf.cpu().numpy(), d))
    assert np.linalg.norm(L - Lref) / np.linalg.norm(Lref) <= FACTOR_TOL


@pytest.mark.parametrize("N,NB,k", [(2048, 256, 3), (1536, 128, 0)])
def test_injected_task_failure_is_an_error_not_a_hang(N, NB, k):
    torch = pytest.importorskip("torch")
    A0 = oracle.dplgsy(N, NB, 3872)
    Lref = _oracle_factor(A0, NB)
    with db.Context(0) as ctx:
        ctx.set_wait_limits(500, 3000)
        assert ctx.inject_fault(db.INJECT_TASK_FAILED, k) == 0
        d, _ = _dev_matrix(torch, A0, NB)
        t0 = time.perf_counter()
        rc = ctx.dpotrf(db.Lower, d)
        dt = time.perf_counter() - t0
        assert rc == ERR_UNEXPECTED
        assert "task reported failed" in ctx.last_error()
        assert dt < 10.0
        # the injection was consumed: the next call on the same context is clean
        _clean_call_matches(ctx, torch, A0, NB, Lref)


def test_withheld_dependency_times_out_and_context_recovers():
    torch = pytest.importorskip("torch")
    N, NB = 2048, 256
    A0 = oracle.dplgsy(N, NB, 3872)
    Lref = _oracle_factor(A0, NB)
    with db.Context(0) as ctx:
        ctx.set_wait_limits(200, 3000)
        # ticket 1 is TRSM(1,0), strip 0: every update of tile row 1 waits on it
        assert ctx.inject_fault(db.INJECT_WITHHOLD, 1) == 0
        d, _ = _dev_matrix(torch, A0, NB)
        t0 = time.perf_counter()
        rc = ctx.dpotrf(db.Lower, d)
        dt = time.perf_counter() - t0
        assert rc == ERR_UNEXPECTED
        msg = ctx.last_error()
        assert "dependency wait timed out" in msg and "site 7" in msg, msg
        assert dt < 10.0
        ctx.set_wait_limits(4000, 4000)
        _clean_call_matches(ctx, torch, A0, NB, Lref)


def test_mixed_factorization_task_failure_releases_tensor_memory():
    # the mixed kernel holds tensor memory; a stopped scheduler must free it and
    # leave the context able to run the mixed solve again
    torch = pytest.importorskip("torch")
    N, NB, NRHS = 2048, 256, 4
    A0 = oracle.dplgsy(N, NB, 3872)
    B0 = oracle.dplrnt(N, NRHS, NB, NB, 3873)
    with db.Context(0) as ctx:
        ctx.set_wait_limits(500, 3000)
        dA, bA = _dev_matrix(torch, A0, NB)
        dB = db.desc_general(N, NRHS, NB, NB)
        bB = torch.from_numpy(db.pack(B0, dB)).cuda()
        db.attach(dB, bB)
        dX = db.desc_general(N, NRHS, NB, NB)
        bX = torch.zeros(db.desc_elems(dX), dtype=torch.float64, device="cuda")
        db.attach(dX, bX)
        assert ctx.inject_fault(db.INJECT_TASK_FAILED, 2) == 0
        rc, st = ctx.dsposv(db.Lower, dA, dB, dX, fmt=db.FP16_SPLIT)
        assert rc == ERR_UNEXPECTED
        rc, st = ctx.dsposv(db.Lower, dA, dB, dX, fmt=db.FP16_SPLIT)
        assert rc == 0 and st["fallback"] == 0, (rc, st, ctx.last_error())
        X = db.unpack(bX.cpu().numpy(), dX)
        assert oracle.check_daxmb(oracle.LOWER, A0, B0, np.asfortranarray(X)) < 10.0


@pytest.mark.parametrize("N,NB", [(3000, 256), (2560, 512)])
def test_selfcheck_every_ticket_runs_once(N, NB):
    torch = pytest.importorskip("torch")
    A0 = oracle.dplgsy(N, NB, 3872)
    Lref = _oracle_factor(A0, NB)
    with db.Context(0) as ctx:
        assert ctx.selfcheck() is None
        assert ctx.set_selfcheck(True) == 0
        d, buf = _dev_matrix(torch, A0, NB)
        assert ctx.dpotrf(db.Lower, d) == 0, ctx.last_error()
        tickets, runs, bad = ctx.selfcheck()
        mt = (N + NB - 1) // NB
        nbs = (NB + 127) // 128
        # the FP64 ticket order's length, as built on the host
        expect = db.lib().dplasma_b200_debug_task_list(0, mt, nbs, 0, None, 0)
        assert tickets == expect and runs == tickets and bad == 0, (tickets, runs, bad, expect)
        L = np.tril(db.unpack(buf.cpu().numpy(), d))
        assert np.linalg.norm(L - Lref) / np.linalg.norm(Lref) <= FACTOR_TOL
