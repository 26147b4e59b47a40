"""Multi-GPU tile Cholesky: 1-D column-cyclic ownership of the tile columns.

The reference distributes the tiles of A 2-D block-cyclically over a P x Q
process grid (tests/common.c:470-490), PaRSEC moves remote tiles between
processes as the DAG asks for them (the remote inputs of TRSM, HERK and GEMM
in src/zpotrf_L.jdf:109,229,232) and the wrapper max-reduces INFO over the
processes (src/zpotrf_wrapper.c:364-368).

Here tile column n lives on rank n % P.  At step k the owner of column k
factors the panel (POTRF(k), TRSM(:,k)) and broadcasts it (the tiles
(k..mt-1, k), contiguous in the packed lower-tile layout) together with its
INFO; every rank then applies the panel to the tile columns it owns (SYRK of
the diagonal tile, GEMM of the tiles below).  One step of look-ahead: the
owner of column k+1 first updates that column with panel k and factors panel
k+1, so the broadcast of panel k+1 runs while every rank does the rest of
step k.  A remote panel always lands in the receiving GPU's own memory before
a kernel reads it.

The schedule (ownership, the per-step operations, the collectives) is plain
Python.  The tile work goes to an engine -- DeviceEngine runs it through the
library's task-insertion pool (dplasma_b200_dtd_*) on one GPU -- and the
exchange to a communicator: TorchComm (torch.distributed: NCCL between GPUs,
gloo between CPU processes) for one process per GPU, or run_lockstep, which
drives several engines from one process and copies the panels device to
device.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import Lower, TASK_GEMM, TASK_POTRF, TASK_SYRK, TASK_TRSM, attach, desc_elems, desc_sym


def owner(n: int, nranks: int) -> int:
    """Rank that owns tile column n (1-D cyclic)."""
    return n % nranks


def local_columns(mt: int, nranks: int, rank: int) -> list[int]:
    return [n for n in range(mt) if owner(n, nranks) == rank]


@dataclass(frozen=True)
class Op:
    """One operation of a rank's schedule.  kind: "panel" (POTRF(k) and
    TRSM(:,k)), "update" (step k applied to tile columns `cols`), "bcast_start"
    / "bcast_wait" (the panel of column k and its INFO from rank `root`)."""
    kind: str
    k: int
    root: int = -1
    cols: tuple = ()


def schedule(mt: int, nranks: int, rank: int) -> list[Op]:
    """The operations of `rank`, in issue order.  Every rank issues the same
    collectives (bcast_start / bcast_wait of every panel) in the same order."""
    ops: list[Op] = []
    if mt == 0:
        return ops
    o0 = owner(0, nranks)
    if o0 == rank:
        ops.append(Op("panel", 0))
    ops.append(Op("bcast_start", 0, o0))
    ops.append(Op("bcast_wait", 0, o0))
    for k in range(mt - 1):
        o = owner(k + 1, nranks)
        if o == rank:
            ops.append(Op("update", k, cols=(k + 1,)))
            ops.append(Op("panel", k + 1))
        ops.append(Op("bcast_start", k + 1, o))
        rest = tuple(n for n in range(k + 2, mt) if owner(n, nranks) == rank)
        if rest:
            ops.append(Op("update", k, cols=rest))
        ops.append(Op("bcast_wait", k + 1, o))
    return ops


def panel_tiles(mt: int, k: int) -> tuple[int, int]:
    """(first tile index, number of tiles) of panel k in the packed lower
    layout (tiles (k..mt-1, k) are consecutive)."""
    first = k * mt - (k * (k - 1)) // 2
    return first, mt - k


class DeviceEngine:
    """The tile work of one rank on its GPU.  `tiles` is a CUDA float64 tensor
    holding the whole matrix in the packed lower-tile layout (tile edge nb, a
    multiple of 128 dividing n); this rank's tile columns are meaningful, the
    others receive the broadcast panels.  The library's task-insertion pool
    runs each panel and update as one launch of the device scheduler."""

    def __init__(self, ctx, n: int, nb: int, tiles):
        if nb % 128 or n % nb:
            raise ValueError("the distributed factorization needs nb a multiple of 128 dividing n")
        self.ctx, self.n, self.nb, self.mt = ctx, n, nb, n // nb
        self.desc = desc_sym(n, nb, Lower)
        if tiles.numel() < desc_elems(self.desc):
            raise ValueError("tile buffer too small")
        self.tiles = tiles
        attach(self.desc, tiles)
        self.pool = ctx.dtd(Lower, self.desc)

    def panel(self, k: int) -> int:
        rc = self.pool.insert(TASK_POTRF, k)
        for m in range(k + 1, self.mt):
            rc = rc or self.pool.insert(TASK_TRSM, k, m)
        if rc:
            raise RuntimeError(f"panel {k}: insertion refused ({rc})")
        return self.pool.flush()

    def update(self, k: int, cols) -> int:
        for n in cols:
            rc = self.pool.insert(TASK_SYRK, k, n)
            for m in range(n + 1, self.mt):
                rc = rc or self.pool.insert(TASK_GEMM, k, m, n)
            if rc:
                raise RuntimeError(f"update {k} of column {n}: insertion refused ({rc})")
        r = self.pool.flush()
        if r < 0:
            raise RuntimeError(f"update {k}: flush failed ({r}): {self.ctx.last_error()}")
        return r

    def panel_tensor(self, k: int):
        first, count = panel_tiles(self.mt, k)
        t = self.nb * self.nb
        return self.tiles[first * t:(first + count) * t]

    def panel_received(self, k: int) -> None:
        rc = self.pool.panel_received(k)
        if rc:
            raise RuntimeError(f"panel {k} marked twice or after local work ({rc})")

    def ready(self) -> None:
        """Wait for the work torch queued on this GPU (a received panel)."""
        import torch
        torch.cuda.current_stream(self.tiles.device).synchronize()

    def close(self) -> int:
        return self.pool.destruct()


class TorchComm:
    """Collectives of one process per GPU (torch.distributed)."""

    def __init__(self, dist, device=None):
        self.dist, self.device = dist, device
        self._pending = {}

    def bcast_start(self, key, tensor, info: int, root: int):
        import torch
        it = torch.tensor([info], dtype=torch.int64, device=tensor.device)
        h1 = self.dist.broadcast(tensor, src=root, async_op=True)
        h2 = self.dist.broadcast(it, src=root, async_op=True)
        self._pending[key] = (h1, h2, it)

    def bcast_wait(self, key) -> int:
        h1, h2, it = self._pending.pop(key)
        h1.wait()
        h2.wait()
        return int(it.item())

    def allreduce_max(self, v: int) -> int:
        import torch
        dev = self.device if self.device is not None else "cpu"
        t = torch.tensor([v], dtype=torch.int64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return int(t.item())


def run_rank(engine, comm, nranks: int, rank: int) -> int:
    """The factorization on this rank (every rank calls it).  Returns INFO:
    0, or the 1-based index of the first non positive definite leading minor
    (the same value on every rank)."""
    mt = engine.mt
    info = 0
    stopped = False
    for op in schedule(mt, nranks, rank):
        if op.kind == "panel":
            if not stopped:
                r = engine.panel(op.k)
                if r:
                    info = r
        elif op.kind == "bcast_start":
            # the panel and the owner's INFO travel together; after a failure
            # the ranks still take part in every collective, with no tile work
            comm.bcast_start(op.k, engine.panel_tensor(op.k), info if rank == op.root else 0, op.root)
        elif op.kind == "bcast_wait":
            r = comm.bcast_wait(op.k)
            if r and not info:
                info = r
            stopped = stopped or info != 0
            if rank != op.root and not stopped:
                engine.ready()
                engine.panel_received(op.k)
        elif op.kind == "update":
            if not stopped:
                engine.update(op.k, op.cols)
    return comm.allreduce_max(info)


def run_lockstep(engines) -> int:
    """The same schedule for len(engines) ranks driven from one process: the
    local work of every rank up to the next collective, then the collective
    as device-to-device copies of the owner's panel.  Engines may share a GPU
    (nothing waits across ranks inside a kernel: each launch is complete
    before the next collective).  Returns INFO."""
    P = len(engines)
    mt = engines[0].mt
    ops = [schedule(mt, P, r) for r in range(P)]
    pos = [0] * P
    info = [0] * P
    stopped = False
    box = {}
    while any(pos[r] < len(ops[r]) for r in range(P)):
        # local work of every rank up to its next collective
        for r in range(P):
            while pos[r] < len(ops[r]) and ops[r][pos[r]].kind in ("panel", "update"):
                op = ops[r][pos[r]]
                if not stopped:
                    if op.kind == "panel":
                        v = engines[r].panel(op.k)
                        if v:
                            info[r] = v
                    else:
                        engines[r].update(op.k, op.cols)
                pos[r] += 1
        heads = {(ops[r][pos[r]].kind, ops[r][pos[r]].k) for r in range(P) if pos[r] < len(ops[r])}
        if len(heads) != 1:
            raise RuntimeError(f"ranks disagree on the next collective: {sorted(heads)}")
        kind, k = heads.pop()
        root = ops[0][pos[0]].root
        if kind == "bcast_start":
            box[k] = info[root]
            if not stopped and not box[k]:
                src = engines[root].panel_tensor(k)
                for r in range(P):
                    if r != root:
                        engines[r].panel_tensor(k).copy_(src)
        else:  # bcast_wait
            v = box.pop(k)
            stopped = stopped or v != 0
            for r in range(P):
                if v and not info[r]:
                    info[r] = v
                if r != root and not stopped:
                    engines[r].ready()
                    engines[r].panel_received(k)
        for r in range(P):
            pos[r] += 1
    return max(info)


def pdpotrf(ctx, n: int, nb: int, tiles, dist, device=None) -> int:
    """One process per GPU: factor the matrix whose tile columns this rank
    owns (n % P == rank) in `tiles` (CUDA tensor, packed lower tiles, the
    global layout), with torch.distributed as the communicator.  The owned
    columns of `tiles` hold L on return.  Returns INFO."""
    P, rank = dist.get_world_size(), dist.get_rank()
    eng = DeviceEngine(ctx, n, nb, tiles)
    try:
        return run_rank(eng, TorchComm(dist, device if device is not None else tiles.device), P, rank)
    finally:
        eng.close()
