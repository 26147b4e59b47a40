"""CPU tests of the multi-GPU column-cyclic factorization's host logic
(dplasma_b200.dist): tile ownership, the per-rank schedule (every rank takes
the same collectives in the same order), the panel exchange and the INFO
reduction, run as world_size 2 and 3 gloo process groups that exchange real
panel tiles.  The tile work is done here by a numpy engine (test code); the
assembled factor is compared with the oracle's, and INFO with the oracle's on a
matrix that is not positive definite.  The same schedule drives the GPU engine
(tests/test_gpu_dist.py)."""
import os
import socket

import numpy as np
import pytest
import scipy.linalg
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from dplasma_b200 import dist as ddist


class NumpyEngine:
    """Tile work on the packed lower-tile layout in a CPU tensor (test only)."""

    def __init__(self, A, nb, rank, nranks):
        n = A.shape[0]
        self.n, self.nb, self.mt = n, nb, n // nb
        self.rank, self.nranks = rank, nranks
        self.tiles = torch.zeros(self.mt * (self.mt + 1) // 2 * nb * nb, dtype=torch.float64)
        for c in range(self.mt):
            if ddist.owner(c, nranks) == rank:        # only the owned columns start with data
                for m in range(c, self.mt):
                    self.tile(m, c)[:, :] = A[m * nb:(m + 1) * nb, c * nb:(c + 1) * nb]

    def tile(self, m, n):
        idx = n * self.mt - n * (n - 1) // 2 + (m - n)
        t = self.nb * self.nb
        return self.tiles[idx * t:(idx + 1) * t].numpy().reshape(self.nb, self.nb).T   # column-major view

    def panel(self, k):
        T = np.asfortranarray(self.tile(k, k))
        info = oracle.dpotrf(oracle.LOWER, T, self.nb)
        if info:
            return k * self.nb + info
        self.tile(k, k)[:, :] = np.tril(T) + np.triu(self.tile(k, k), 1)
        Lkk = np.tril(T)
        for m in range(k + 1, self.mt):
            X = self.tile(m, k)
            X[:, :] = scipy.linalg.solve_triangular(Lkk, X.T, lower=True).T
        return 0

    def update(self, k, cols):
        for n in cols:
            for m in range(n, self.mt):
                C = self.tile(m, n)
                upd = self.tile(m, k) @ self.tile(n, k).T
                if m == n:
                    C[:, :] -= np.tril(upd)
                else:
                    C[:, :] -= upd

    def panel_tensor(self, k):
        first, count = ddist.panel_tiles(self.mt, k)
        t = self.nb * self.nb
        return self.tiles[first * t:(first + count) * t]

    def panel_received(self, k):
        pass

    def ready(self):
        pass


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, nranks, port, N, NB, bad, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        A = oracle.dplgsy(N, NB, 3872)
        if bad is not None:
            A[bad, bad] = -1.0
        eng = NumpyEngine(A, NB, rank, nranks)
        info = ddist.run_rank(eng, ddist.TorchComm(dist), nranks, rank)
        # assemble: every rank contributes its owned columns
        mine = torch.zeros_like(eng.tiles)
        t = NB * NB
        for c in ddist.local_columns(eng.mt, nranks, rank):
            first, count = ddist.panel_tiles(eng.mt, c)
            mine[first * t:(first + count) * t] = eng.tiles[first * t:(first + count) * t]
        dist.all_reduce(mine)
        if rank == 0:
            np.save(out + ".npy", mine.numpy())
            with open(out + ".info", "w") as f:
                f.write(str(info))
        infos = [None] * nranks
        dist.all_gather_object(infos, info)
        assert len(set(infos)) == 1, infos
    finally:
        dist.destroy_process_group()


def _run(nranks, N, NB, bad, tmp_path):
    out = str(tmp_path / f"res{nranks}")
    mp.spawn(_worker, args=(nranks, _free_port(), N, NB, bad, out), nprocs=nranks, join=True)
    return np.load(out + ".npy"), int(open(out + ".info").read())


def test_ownership_and_schedule_collectives_match():
    mt, P = 7, 3
    assert [ddist.owner(n, P) for n in range(mt)] == [0, 1, 2, 0, 1, 2, 0]
    assert ddist.local_columns(mt, P, 1) == [1, 4]
    scheds = [ddist.schedule(mt, P, r) for r in range(P)]
    coll = [[(o.kind, o.k, o.root) for o in s if o.kind.startswith("bcast")] for s in scheds]
    assert coll[0] == coll[1] == coll[2] and len(coll[0]) == 2 * mt
    # every tile column's panel is factored exactly once, by its owner
    panels = sorted((o.k, r) for r, s in enumerate(scheds) for o in s if o.kind == "panel")
    assert panels == [(k, k % P) for k in range(mt)]
    # every (step, owned column > step) update happens exactly once, on the owner
    ups = sorted((o.k, n, r) for r, s in enumerate(scheds) for o in s if o.kind == "update" for n in o.cols)
    assert ups == sorted((k, n, n % P) for k in range(mt) for n in range(k + 1, mt))
    # look-ahead: the owner of column k+1 updates it and factors panel k+1 before broadcasting it
    s1 = [(o.kind, o.k, o.cols) for o in scheds[1]]
    i = s1.index(("panel", 1, ()))
    assert s1[i - 1] == ("update", 0, (1,)) and s1[i + 1][0] == "bcast_start"
    assert ddist.panel_tiles(5, 2) == (9, 3)


@pytest.mark.parametrize("nranks", [2, 3])
def test_distributed_factor_matches_oracle(tmp_path, nranks):
    N, NB = 640, 64
    tiles, info = _run(nranks, N, NB, None, tmp_path)
    assert info == 0
    mt = N // NB
    L = np.zeros((N, N))
    for c in range(mt):
        for m in range(c, mt):
            idx = c * mt - c * (c - 1) // 2 + (m - c)
            L[m * NB:(m + 1) * NB, c * NB:(c + 1) * NB] = tiles[idx * NB * NB:(idx + 1) * NB * NB].reshape(NB, NB).T
    L = np.tril(L)
    ref = oracle.dplgsy(N, NB, 3872)
    assert oracle.dpotrf(oracle.LOWER, ref, NB) == 0
    ref = np.tril(ref)
    assert np.linalg.norm(L - ref) / np.linalg.norm(ref) <= 1e-12


def test_distributed_info_reduction(tmp_path):
    N, NB, bad = 512, 64, 300
    A = oracle.dplgsy(N, NB, 3872)
    A[bad, bad] = -1.0
    ref_info = oracle.dpotrf(oracle.LOWER, A, NB)
    assert ref_info == bad + 1
    _, info = _run(2, N, NB, bad, tmp_path)
    assert info == ref_info
