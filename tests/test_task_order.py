"""CPU tests of the persistent scheduler's ticket order.

CTAs take tickets in order and a task starts once its dependencies are met,
so the factorization makes progress without any co-residency assumption iff
every task's dependencies are produced by tasks earlier in the order.  The
rules replayed here are the ones the kernel waits on (the dataflow of
src/zpotrf_L.jdf as per-tile completion counts), for the FP64 list (one task
per 128x128 block and panel) and the mixed-precision list (one task per
tile and chunk of S panels)."""
import ctypes

import numpy as np
import pytest

import dplasma_b200 as db

T_POTRF, T_TRSM, T_GEMM = 1, 2, 3


def tasks(chunk, mt, nbs, delay):
    L = db.lib()
    f = L.dplasma_b200_debug_task_list
    f.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_int]
    n = f(chunk, mt, nbs, delay, None, 0)
    out = np.zeros(n, dtype=np.uint64)
    assert f(chunk, mt, nbs, delay, out.ctypes.data, n) == n
    return [(int(t) & 0xF, (int(t) >> 4) & 0xFFFF, (int(t) >> 20) & 0xFFFF, (int(t) >> 36) & 0xFFFF,
             (int(t) >> 52) & 0xF, (int(t) >> 56) & 0xF) for t in out]


def replay(tl, mt, nbs, S):
    potrf = np.zeros(mt, int)
    trsm = np.zeros((mt, mt), int)
    upd = np.zeros((mt, mt), int)

    def all_updates(m, n):
        if S:
            return -(-n // S)
        return n * (nbs * (nbs + 1) // 2 if m == n else nbs * nbs)

    for i, (ty, k, m, n, bi, bj) in enumerate(tl):
        if ty == T_POTRF:
            assert upd[k, k] == all_updates(k, k), (i, ty, k)
            potrf[k] += 1
        elif ty == T_TRSM:
            assert potrf[k] == 1 and upd[m, k] == all_updates(m, k), (i, ty, k, m)
            trsm[m, k] += 1
        else:
            assert ty == T_GEMM
            if S:
                kl = min(k * S + S, n) - 1
                assert trsm[m, kl] == nbs and trsm[n, kl] == nbs and upd[m, n] >= k, (i, k, m, n)
            else:
                assert trsm[m, k] == nbs and trsm[n, k] == nbs, (i, k, m, n)
                step = nbs * (nbs + 1) // 2 if m == n else nbs * nbs
                assert upd[m, n] >= k * step, (i, k, m, n)
            upd[m, n] += 1
    # everything factored exactly once
    assert (potrf == 1).all()
    for m in range(mt):
        for k in range(m):
            assert trsm[m, k] == nbs
        for n in range(m + 1):
            assert upd[m, n] == all_updates(m, n)


@pytest.mark.parametrize("mt,nbs,delay", [(1, 2, 0), (2, 1, 3), (7, 2, 5), (13, 1, 40), (20, 2, 444)])
def test_fp64_ticket_order(mt, nbs, delay):
    replay(tasks(0, mt, nbs, delay), mt, nbs, 0)


@pytest.mark.parametrize("mt,S,delay", [(1, 4, 0), (2, 4, 3), (5, 4, 0), (9, 4, 7), (17, 3, 100), (33, 4, 444),
                                        (12, 1, 10), (10, 16, 5), (65, 8, 444), (65, 16, 444)])
def test_mixed_ticket_order(mt, S, delay):
    replay(tasks(S, mt, 2, delay), mt, 2, S)


def test_mixed_steps_share_update_work():
    # every step between chunk closes carries update work (no idle steps)
    mt, S = 40, 4
    tl = tasks(S, mt, 2, 0)
    potrf_pos = [i for i, t in enumerate(tl) if t[0] == T_POTRF]
    for a, b in zip(potrf_pos[S:mt - 3 * S], potrf_pos[S + 1:mt - 3 * S + 1]):
        between = [t for t in tl[a:b] if t[0] == T_GEMM and t[3] != tl[b][1]]
        assert len(between) > 0


def tasks_blocked(chunk, mt, nbs, delay, bw, bh):
    L = db.lib()
    f = L.dplasma_b200_debug_task_list_blocked
    f.argtypes = [ctypes.c_int] * 6 + [ctypes.c_void_p, ctypes.c_int]
    n = f(chunk, mt, nbs, delay, bw, bh, None, 0)
    out = np.zeros(n, dtype=np.uint64)
    assert f(chunk, mt, nbs, delay, bw, bh, out.ctypes.data, n) == n
    return [(int(t) & 0xF, (int(t) >> 4) & 0xFFFF, (int(t) >> 20) & 0xFFFF, (int(t) >> 36) & 0xFFFF,
             (int(t) >> 52) & 0xF, (int(t) >> 56) & 0xF) for t in out]


@pytest.mark.parametrize("mt,S,bw,bh,delay", [(33, 4, 4, 8, 444), (65, 8, 4, 32, 444), (65, 8, 1, 1, 444),
                                              (40, 3, 7, 5, 444), (65, 8, 16, 16, 888)])
def test_mixed_blocked_ticket_order(mt, S, bw, bh, delay):
    # the blocked order permutes each step's share: same tasks, same dependency guarantees
    tl = tasks_blocked(S, mt, 2, delay, bw, bh)
    replay(tl, mt, 2, S)
    assert sorted(tl) == sorted(tasks(S, mt, 2, delay))
