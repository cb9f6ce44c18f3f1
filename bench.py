#!/usr/bin/env python3
"""Benchmark of the B200 dposv path (one JSON line on rank 0).

Workload (the large single-solve configuration): N = 32768 symmetric positive
definite matrix made by dplgsy (seed 51, bump = N), NB = 512 tiles, nrhs = 64
right-hand sides from dplrnt (seed 5673), solved to FP64 accuracy by the
mixed-precision solver (BF16x3 tensor-core factorization + FP64 iterative
refinement).  One step = one complete solve with A and B resident in HBM.
`value` is dposv TFLOP/s counted with the reference's FP64 flop model
(include/chameleon/flops.h: potrf + potrs) over device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

`--impl reference` times the reference's own CPU implementation (the
reference library built from its sources, OpenMP runtime + OpenBLAS) on the
host cores.  Multi-GPU runs are independent replicas (the path is one solve
per GPU; nothing is exchanged), launched one process per GPU by torchrun.
"""
import argparse
import ctypes
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

METRIC = "dposv TFLOP/s & batched solves/s at FP64 accuracy, mixed vs plain FP64; p99"
N_DEF, NB_DEF, NRHS_DEF = 32768, 512, 64
SEED_A, SEED_B = 51, 5673


def dposv_flops(N, nrhs):
    """FMULS+FADDS of potrf + potrs, include/chameleon/flops.h:101-108,298-311."""
    n = float(N)
    potrf = n * (n / 6.0 * n + n / 2.0 + 1.0 / 3.0) + n * (n * n / 6.0 - 1.0 / 6.0)
    potrs = nrhs * n * (n + 1.0) + nrhs * n * (n - 1.0)
    return potrf + potrs


def peaks():
    p = {}
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    return p


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# Reference arm: the reference's own CPU dposv (oracle/_ref/libchamref.so)
# ---------------------------------------------------------------------------
def reference_arm(args, world, rank):
    if rank != 0:
        return None
    from oracle import oracle as O
    if not O.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libchamref.so not built"}))
        return None
    cores = os.cpu_count() or 1
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    L = O.reference(cores)
    N = args.ref_n
    NB, nrhs = NB_DEF, NRHS_DEF
    A0 = np.zeros((N, N), order="F")
    B0 = np.zeros((N, nrhs), order="F")
    L.chamref_dplgsy(float(N), 123, N, O._ptr(A0), N, NB, SEED_A)
    L.chamref_dplrnt(N, nrhs, O._ptr(B0), N, NB, SEED_B)
    times = []
    for it in range(args.warmup + args.steps):
        A = A0.copy(order="F")
        B = B0.copy(order="F")
        t = ctypes.c_double()
        rc = L.chamref_dposv(122, N, nrhs, NB, O._ptr(A), N, O._ptr(B), N, ctypes.byref(t))
        assert rc == 0, rc
        if it >= args.warmup:
            times.append(t.value)
    tsum = sum(times)
    val = dposv_flops(N, nrhs) * len(times) / tsum / 1e12
    sample = "N=%d NB=%d nrhs=%d dplgsy/dplrnt seeds %d/%d, Lower, full dposv per step (%.1f s/step)" % (
        N, NB, nrhs, SEED_A, SEED_B, tsum / len(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tsum / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "dposv (reference CPU: OpenMP runtime + coreblas + OpenBLAS 0.3.30)",
                   "N": N, "NB": NB, "nrhs": nrhs},
        "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return line


def cpu_baseline_sample():
    """The reference's dposv on the host cores on a bounded sample (N=8192)."""
    try:
        from oracle import oracle as O
        if not O.reference_available():
            return None
        cores = os.cpu_count() or 1
        os.environ["OPENBLAS_NUM_THREADS"] = "1"
        L = O.reference(cores)
        N, NB, nrhs = 8192, NB_DEF, NRHS_DEF
        A0 = np.zeros((N, N), order="F")
        B0 = np.zeros((N, nrhs), order="F")
        L.chamref_dplgsy(float(N), 123, N, O._ptr(A0), N, NB, SEED_A)
        L.chamref_dplrnt(N, nrhs, O._ptr(B0), N, NB, SEED_B)
        best = None
        t_total = 0.0
        for _ in range(3):
            A = A0.copy(order="F")
            B = B0.copy(order="F")
            t = ctypes.c_double()
            L.chamref_dposv(122, N, nrhs, NB, O._ptr(A), N, O._ptr(B), N, ctypes.byref(t))
            best = t.value if best is None else min(best, t.value)
            t_total += t.value
            if t_total > 30:
                break
        val = dposv_flops(N, nrhs) / best / 1e12
        return {"value": val, "unit": "TFLOP/s", "cores": cores, "kind": "reference",
                "sample": "reference dposv N=%d NB=%d nrhs=%d (best of <=3, %.1f s CPU); reference OpenMP runtime "
                          "+ OpenBLAS, all host cores" % (N, NB, nrhs, t_total)}
    except Exception as e:   # the baseline is reported, not required
        return {"value": None, "unit": "TFLOP/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "failed: %s" % e}


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def b200_arm(args, world, rank, local):
    import torch
    import chameleon_b200 as cb
    cb.init()
    L = cb.lib()
    N, NB, nrhs = args.n, args.nb, args.nrhs
    prec = {"bf16x3": cb.PREC_BF16X3, "fp32": cb.PREC_FP32, "fp64": cb.PREC_FP64}[args.precision]
    dA = cb.Desc.create(N, N, NB)
    dB = cb.Desc.create(N, nrhs, NB)
    dX = cb.Desc.create(N, nrhs, NB)
    assert cb.dplgsy_Tile(float(N), cb.ChamUpperLower, dA, SEED_A + rank) == 0
    assert cb.dplrnt_Tile(dB, SEED_B + rank) == 0
    flops = dposv_flops(N, nrhs)

    def step():
        rc, info = cb.dposv_mixed_Tile(cb.ChamLower, prec, dA, dB, dX)
        assert rc == 0, rc
        return info

    for _ in range(args.warmup):
        info = step()
    stats_acc = np.zeros(7)
    barrier(world)
    L.CHAM_B200_Device_Sync()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    n0 = L.CHAM_B200_Launch_Count()
    L.CHAM_B200_Event_Record(0)
    iters = []
    berrs = []
    st = (ctypes.c_double * 7)()
    for _ in range(args.steps):
        info = step()
        L.CHAM_B200_Mixed_Stats(st)
        stats_acc += np.array(st[:])
        iters.append(info.iterations)
        berrs.append(info.backward_error)
    L.CHAM_B200_Event_Record(1)
    ms = L.CHAM_B200_Event_Elapsed(0, 1)
    launches = int(L.CHAM_B200_Launch_Count() - n0)
    clk = clocks.stop()
    barrier(world)
    ms_max = allreduce_max(ms, world)
    value = flops * args.steps * world / (ms_max * 1e-3) / 1e12
    stats = stats_acc / args.steps

    # roofline of the dominant kernel: the FP32 factorization DAG launch
    pk = peaks()
    fact_ms = stats[0]
    mult = 3.0 if args.precision in ("bf16x3", "fp32") else 1.0
    fact_flops = N ** 3 / 3.0
    if args.precision == "bf16x3":
        peak, peak_src = pk.get("bf16_tflops"), "bf16_tflops (measured, burst)"
    elif args.precision == "fp32":
        peak, peak_src = (pk.get("bf16_tflops") or 1666.5) / 2.0, "bf16_tflops/2 (tf32 rate, measured bf16)"
    else:
        peak, peak_src = pk.get("fp64_tflops"), "fp64"
    achieved = mult * fact_flops / (fact_ms * 1e-3) / 1e12 if fact_ms > 0 else None
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if (achieved and peak) else None, "traffic": None,
                "kernel": "cholesky_dag_kernel<float,%s> (factorization + first solve)" % args.precision,
                "flops_per_launch": mult * fact_flops,
                "peak_source": peak_src + (" of measured" if peak else "")}

    # plain FP64 path on the same problem (reported beside the mixed number)
    fp64 = None
    if args.compare_fp64 and rank == 0:
        dA2 = cb.Desc.create(N, N, NB)
        dB2 = cb.Desc.create(N, nrhs, NB)
        cb.dplgsy_Tile(float(N), cb.ChamUpperLower, dA2, SEED_A)
        cb.dplrnt_Tile(dB2, SEED_B)
        L.CHAM_B200_Event_Record(2)
        assert cb.dposv_Tile(cb.ChamLower, dA2, dB2) == 0
        L.CHAM_B200_Event_Record(3)
        fms = L.CHAM_B200_Event_Elapsed(2, 3)
        fp64 = {"tflops": flops / (fms * 1e-3) / 1e12, "ms": fms}
        dA2.destroy()
        dB2.destroy()

    # end to end: LAPACK-layout CHAMELEON_dsposv from pinned host memory
    e2e = None
    if args.e2e and rank == 0:
        hA = torch.empty((N, N), dtype=torch.float64, pin_memory=True)
        hB = torch.empty((nrhs, N), dtype=torch.float64, pin_memory=True)
        hX = torch.empty((nrhs, N), dtype=torch.float64, pin_memory=True)
        assert L.CHAMELEON_Desc2Lap(cb.ChamUpperLower, dA.ptr, ctypes.c_void_p(hA.data_ptr()), N) == 0
        assert L.CHAMELEON_Desc2Lap(cb.ChamUpperLower, dB.ptr, ctypes.c_void_p(hB.data_ptr()), N) == 0
        cb.set_param(cb.CHAMELEON_TILE_SIZE, NB)
        cb.set_param(cb.CHAMELEON_B200_PRECISION, prec if prec != cb.PREC_FP64 else cb.PREC_BF16X3)
        it = ctypes.c_int()

        def e2e_step():
            rc = L.CHAMELEON_dsposv(cb.ChamLower, N, nrhs, ctypes.c_void_p(hA.data_ptr()), N,
                                    ctypes.c_void_p(hB.data_ptr()), N, ctypes.c_void_p(hX.data_ptr()), N,
                                    ctypes.byref(it))
            assert rc == 0, rc

        e2e_step()
        L.CHAM_B200_Event_Record(4)
        ne = max(1, min(args.steps, 3))
        for _ in range(ne):
            e2e_step()
        L.CHAM_B200_Event_Record(5)
        ems = L.CHAM_B200_Event_Elapsed(4, 5) / ne
        e2e = {"value": flops / (ems * 1e-3) / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": 8 * N * N + 8 * N * nrhs,
               "d2h_bytes_per_step": 8 * N * nrhs, "ms_per_step": ems,
               "api": "CHAMELEON_dsposv (LAPACK layout, pinned host A/B/X)"}
        del hA

    cpu = cpu_baseline_sample() if (rank == 0 and not args.no_cpu) else None
    line = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (bf16x3 factor + f64 refinement)" if args.precision == "bf16x3" else args.precision,
        "data": "synthetic (dplgsy seed %d + rank, dplrnt seed %d + rank)" % (SEED_A, SEED_B),
        "config": {"workload": "dposv N=%d NB=%d nrhs=%d, %s factorization + FP64 iterative refinement to FP64 "
                               "backward error (dsposv test), Lower" % (N, NB, nrhs, args.precision),
                   "N": N, "NB": NB, "nrhs": nrhs, "precision": args.precision,
                   "l2": "inputs larger than L2 (A is %.1f GB FP64)" % (8 * N * N / 1e9),
                   "parallelism": "replicas x%d" % world},
        "refine": {"iterations": iters, "backward_error_max": max(berrs) if berrs else None,
                   "phases_ms": {"factor+solve": stats[0], "refine_solves": stats[1], "residuals": stats[2],
                                 "casts+norm": stats[3], "total": stats[4]}},
        "fp64_plain": fp64,
        "speedup_vs_fp64_plain": (fp64["ms"] / (ms_max / args.steps)) if fp64 else None,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clk,
        "gpu_launches": launches,
    }
    if rank == 0:
        print(json.dumps(line))
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N_DEF)
    ap.add_argument("--nb", type=int, default=NB_DEF)
    ap.add_argument("--nrhs", type=int, default=NRHS_DEF)
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "fp32", "fp64"])
    ap.add_argument("--ref-n", type=int, default=16384, help="order of the reference arm's per-step sample")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-fp64", dest="compare_fp64", action="store_false")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        else:
            b200_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
