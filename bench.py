#!/usr/bin/env python
"""Benchmark of the B200 tile-Cholesky path (one JSON line on stdout).

Workload (one "step"): plain FP64 dplasma_dposv, lower, N=65536, NB=256,
NRHS=16, on the dplgsy matrix (seed 3872, diagonal += N) and dplrnt
right-hand sides (seed 3873) -- the matrix and sizes dplasma's own testers
use, generated on the GPU bit-identically to the reference's generators.

  value : TFLOP/s of the step with inputs resident in HBM (the matrix is
          restored from a pristine device copy before every step, inside the
          timed region; 17 GB per step, larger than L2);
  e2e   : the same metric through the C ABI with caller-owned pinned HOST
          buffers: host->device copy of A and B, factor, solve, copy back;
  roofline : the persistent factorization kernel against the measured FP64
          tensor-core (DMMA) peak of this GPU;
  cpu_baseline : the reference's own CORE kernels (compiled from its sources)
          run as the tile DAG on all host cores, on a bounded N.

--impl reference runs only that CPU path (the reference's kernels) on a
bounded sample and prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "TFLOP/s & time-to-FP64-accuracy dposv N=65536: mixed+IR vs plain FP64 on 1 B200"
SEED_A, SEED_B = 3872, 3873


def potrf_flops(n):
    return n ** 3 / 3.0


def posv_flops(n, nrhs):
    return n ** 3 / 3.0 + 2.0 * nrhs * n * n


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                mx.append(float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[4:8]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU side (reference kernels) -- only the baseline legs touch oracle/
# ---------------------------------------------------------------------------
def cpu_reference_tflops(n, nb, threads, reps=1):
    import ctypes
    import oracle
    R = oracle.ref()
    kind = "reference"
    if R is None:
        kind = "port"
    A0 = oracle.dplgsy(n, nb, SEED_A)
    best = None
    for _ in range(reps):
        A = A0.copy(order="F")
        t = time.perf_counter()
        if R is not None:
            info = R.ref_dpotrf_parallel(oracle.LOWER, n, nb, A.ctypes.data_as(ctypes.c_void_p), n, threads)
        else:
            info = oracle.dpotrf_parallel(oracle.LOWER, A, nb, threads)
        dt = time.perf_counter() - t
        assert info == 0
        best = dt if best is None else min(best, dt)
    return potrf_flops(n) / best / 1e12, best, kind


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n, nb = args.cpu_n, 256
    for _ in range(args.warmup if args.warmup < 1 else 1):
        cpu_reference_tflops(min(n, 4096), nb, threads)
    vals, times = [], []
    for _ in range(args.steps):
        v, t, kind = cpu_reference_tflops(n, nb, threads)
        vals.append(v)
        times.append(t)
    value = sum(potrf_flops(n) for _ in times) / sum(times) / 1e12
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"dpotrf FP64 lower N={n} NB={nb} (bounded CPU sample of the N=65536 workload), "
                               "dplgsy seed 3872", "host_threads": threads},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": kind,
                         "sample": f"dpotrf N={n} NB={nb} lower, {args.steps} runs; reference CORE_d* kernels "
                                   "(compiled from the dplasma sources) run as the tile DAG with OpenMP tasks "
                                   "over OpenBLAS, one BLAS thread per task"},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import torch
    import dplasma_b200 as db

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    dev = local
    torch.cuda.set_device(dev)
    N, NB, NRHS = args.n, args.nb, args.nrhs
    ctx = db.Context(dev)

    # device-resident descriptors (sym lower tiles, general tiles for B)
    dA = db.desc_sym(N, NB, db.Lower)
    dB = db.desc_general(N, NRHS, NB, NB)
    A_pristine = torch.empty(db.desc_elems(dA), dtype=torch.float64, device="cuda")
    A = torch.empty_like(A_pristine)
    B_pristine = torch.empty(db.desc_elems(dB), dtype=torch.float64, device="cuda")
    B = torch.empty_like(B_pristine)
    db.attach(dA, A_pristine)
    db.attach(dB, B_pristine)
    assert ctx.dplgsy(float(N), db.Lower, dA, SEED_A) == 0
    assert ctx.dplrnt(0, dB, SEED_B) == 0
    db.attach(dA, A)
    db.attach(dB, B)
    peak = ctx.fp64_peak_tflops()

    def step():
        A.copy_(A_pristine)
        B.copy_(B_pristine)
        torch.cuda.current_stream().synchronize()
        info = ctx.dposv(db.Lower, dA, dB)
        if info != 0:
            raise RuntimeError(f"dposv info={info}: {ctx.last_error()}")

    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    fac_ms, sol_ms, launches = [], [], 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
            fac_ms.append(ctx.last_factor_ms())
            sol_ms.append(ctx.last_solve_ms())
            launches += ctx.last_launches()
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if dist:
        dist.barrier()
    total_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / args.steps
    value = world * posv_flops(N, NRHS) / (ms_step * 1e-3) / 1e12
    fac = statistics.median(fac_ms)
    achieved = potrf_flops(N) / (fac * 1e-3) / 1e12

    # end to end through the C ABI with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        hA = torch.empty(db.desc_elems(dA), dtype=torch.float64, pin_memory=True)
        hB = torch.empty(db.desc_elems(dB), dtype=torch.float64, pin_memory=True)
        hA_np, hB_np = hA.numpy(), hB.numpy()
        A0h, B0h = A_pristine.cpu().numpy(), B_pristine.cpu().numpy()
        hdA = db.desc_sym(N, NB, db.Lower)
        hdB = db.desc_general(N, NRHS, NB, NB)
        db.attach(hdA, hA_np)
        db.attach(hdB, hB_np)
        times = []
        for i in range(args.e2e_steps + 1):
            np.copyto(hA_np, A0h)
            np.copyto(hB_np, B0h)
            t = time.perf_counter()
            info = ctx.dposv(db.Lower, hdA, hdB)
            dt = time.perf_counter() - t
            assert info == 0, ctx.last_error()
            if i > 0:
                times.append(dt)
        e2e_s = sum(times) / len(times)
        e2e = {"value": world * posv_flops(N, NRHS) / e2e_s / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(hA_np.nbytes + hB_np.nbytes),
               "d2h_bytes_per_step": int(hA_np.nbytes + hB_np.nbytes), "s_per_step": e2e_s,
               "steps": len(times)}
        del hA, hB

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v, t, kind = cpu_reference_tflops(args.cpu_n, 256, threads)
        cpu = {"value": v, "unit": "TFLOP/s", "cores": threads, "kind": kind,
               "sample": f"dpotrf N={args.cpu_n} NB=256 lower, one run of {t:.2f} s: the reference's CORE_d* kernels "
                         "(compiled from its sources) as the tile DAG, OpenMP tasks over OpenBLAS on all host cores"}

    # DRAM bytes of one factorization launch: an ncu capture at a smaller N
    # (profiles/potrf_traffic_N16384.txt), scaled by (N/n)^3 at the same NB.
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "potrf_traffic_N16384.txt")
    if os.path.exists(tpath) and NB == 256:
        for line in open(tpath):
            if line.startswith("dram_bytes_per_launch"):
                _, b, _, n0 = line.split()
                traffic = float(b) * (N / float(n0)) ** 3

    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"dposv FP64 lower N={N} NB={NB} NRHS={NRHS}: dplgsy(seed 3872, bump N) and "
                               f"dplrnt(seed 3873); step = restore A,B in HBM + dpotrf + dpotrs",
                   "l2": "inputs larger than L2 (A is %.1f GB per step)" % (A.numel() * 8 / 1e9),
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "dpotrf_tflops": achieved, "dpotrf_ms": fac, "dpotrs_ms": statistics.median(sol_ms),
        "dpotrs_gbs": 2 * (N * (N + 1) / 2 * 8 + 2 * N * NRHS * 8) / (statistics.median(sol_ms) * 1e-3) / 1e9,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None, "traffic": traffic,
                     "kernel": "potrf_persistent_kernel",
                     "peak_source": "measured FP64 DMMA (mma.sync m16n8k4 f64) probe on this GPU; "
                                    "MEASURED_PEAKS.json carries no FP64 figure"},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks, "wall_s": wall,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--n", type=int, default=65536)
    p.add_argument("--nb", type=int, default=256)
    p.add_argument("--nrhs", type=int, default=16)
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--cpu-n", type=int, default=16384)
    p.add_argument("--no-cpu", action="store_true")
    args = p.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
