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


def cpu_baseline_sample(N, NB, nrhs):
    """The reference's dposv on the host cores, on the bench's own problem
    (one or more complete solves, stopping once 30 s of CPU time are spent)."""
    try:
        from oracle import oracle as O
        if not O.reference_available():
            return None
        cores = os.cpu_count() or 1
        os.environ["OPENBLAS_NUM_THREADS"] = "1"
        L = O.reference(cores)
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
            if t_total + t.value > 30:   # the next solve would pass the 30 s bound
                break
        val = dposv_flops(N, nrhs) / best / 1e12
        return {"value": val, "unit": "TFLOP/s", "cores": cores, "kind": "reference",
                "sample": "reference dposv N=%d NB=%d nrhs=%d, the bench's workload (best of <=3 solves, stopped "
                          "after 30 s: %.1f s CPU); reference OpenMP runtime + OpenBLAS, all host cores"
                          % (N, NB, nrhs, t_total)}
    except Exception as e:   # the baseline is reported, not required
        return {"value": None, "unit": "TFLOP/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "failed: %s" % e}


# ---------------------------------------------------------------------------
# Ill-conditioned systems: A = Q diag(s) Q^T, s geometric from 1 to 1/cond
# ---------------------------------------------------------------------------
COND_SEED = 1234


def conditioning_section(args, cb, rank):
    """C3: refinement convergence vs condition number and the FP64 fallback.
    Inputs are built on the GPU (input setup, outside any timed region): Q from
    the QR factorization of a seeded Gaussian matrix, B = A x_true."""
    if rank != 0:
        return None
    import torch
    N, nrhs, NB = args.cond_n, 16, 512
    g = torch.Generator(device="cuda").manual_seed(COND_SEED)
    Q, _ = torch.linalg.qr(torch.randn(N, N, dtype=torch.float64, device="cuda", generator=g))
    xt = torch.randn(nrhs, N, dtype=torch.float64, device="cuda", generator=g)   # column-major N x nrhs
    out = []
    for cond in args.conds:
        sv = torch.logspace(0.0, -np.log10(cond), N, dtype=torch.float64, device="cuda")
        A0 = (Q * sv) @ Q.T
        A0 = 0.5 * (A0 + A0.T)
        B0 = (A0 @ xt.T).T.contiguous()
        row = {"cond": cond}
        for arm in ("mixed", "fp64"):
            A = A0.clone()
            B = B0.clone()
            X = torch.zeros_like(B0)
            dA = cb.Desc.create(N, N, NB, mat=A)
            dB = cb.Desc.create(N, nrhs, NB, mat=B)
            dX = cb.Desc.create(N, nrhs, NB, mat=X)
            torch.cuda.synchronize()
            t0 = time.perf_counter()   # both calls end synchronized
            if arm == "mixed":
                rc, info = cb.dposv_mixed_Tile(cb.ChamLower, cb.PREC_BF16X3, dA, dB, dX)
            else:
                rc = cb.dposv_Tile(cb.ChamLower, dA, dB)
                X = B
            ms = (time.perf_counter() - t0) * 1e3
            torch.cuda.synchronize()
            ferr = float((X - xt).abs().max() / xt.abs().max())
            R = B0 - (A0 @ X.T).T
            berr = float((R.abs().amax(dim=1) / (A0.abs().sum(dim=1).max() * X.abs().amax(dim=1))).max())
            entry = {"rc": rc, "ms_wall": ms, "forward_error": ferr, "backward_error": berr}
            if arm == "mixed":
                entry.update({"iterations": info.iterations, "fallback": bool(info.fallback)})
            row[arm] = entry
            del dA, dB, dX
        out.append(row)
    return {"workload": "N=%d nrhs=%d, A = Q diag(s) Q^T (Q from QR of a Gaussian matrix, seed %d), s geometric "
                        "from 1 to 1/cond, B = A x_true; mixed BF16x3 + FP64 refinement (dsposv rules, 30 "
                        "iterations max, then FP64) vs plain FP64" % (N, nrhs, COND_SEED),
            "cases": out}


# ---------------------------------------------------------------------------
# Uneven batch: 8192 systems, n ~ U{16..512}, nrhs ~ U{1..8}
# ---------------------------------------------------------------------------
BATCH_COUNT, BATCH_SEED, BATCH_NMIN, BATCH_NMAX = 8192, 2024, 16, 512


def batch_workload(count=BATCH_COUNT, seed=BATCH_SEED):
    rng = np.random.default_rng(seed)
    n = rng.integers(BATCH_NMIN, BATCH_NMAX + 1, size=count).astype(np.int32)
    k = rng.integers(1, 9, size=count).astype(np.int32)
    a_off = np.zeros(count, np.int64)
    b_off = np.zeros(count, np.int64)
    a_off[1:] = np.cumsum(n.astype(np.int64) ** 2)[:-1]
    b_off[1:] = np.cumsum(n.astype(np.int64) * k)[:-1]
    return n, k, a_off, b_off


def batch_section(args, cb, world, rank):
    """C4: one uneven batch per step through CHAM_B200_dposv_batch vs one
    CHAMELEON_dposv call per matrix (the plain per-matrix launch path)."""
    import torch
    L = cb.lib()
    n, k, a_off, b_off = batch_workload(args.batch_count)
    count = len(n)
    na = int(a_off[-1] + int(n[-1]) ** 2)
    nb_ = int(b_off[-1] + int(n[-1]) * int(k[-1]))
    A0 = torch.empty(na, dtype=torch.float64, device="cuda")
    B0 = torch.empty(nb_, dtype=torch.float64, device="cuda")
    h = ctypes.c_void_p()
    assert L.CHAM_B200_Handle_Create(ctypes.byref(h), None) == 0
    for i in range(count):
        ni, ki = int(n[i]), int(k[i])
        bump = ctypes.c_double(float(ni))
        pa = ctypes.c_void_p(A0.data_ptr() + 8 * int(a_off[i]))
        pb = ctypes.c_void_p(B0.data_ptr() + 8 * int(b_off[i]))
        assert L.CUDA_dplgsy(ctypes.byref(bump), ni, ni, pa, ni, ni, 0, 0, BATCH_SEED + i, h) == 0
        assert L.CUDA_dplrnt(ni, ki, pb, ni, ni, 0, 0, BATCH_SEED + 7 * count + i, h) == 0
    torch.cuda.synchronize()
    L.CHAM_B200_Handle_Destroy(h)
    A, B = A0.clone(), B0.clone()
    dn = torch.from_numpy(n).cuda()
    dk = torch.from_numpy(k).cuda()
    da = torch.from_numpy(a_off).cuda()
    db = torch.from_numpy(b_off).cuda()
    info = torch.zeros(count, dtype=torch.int32, device="cuda")
    flops = sum(dposv_flops(int(a), int(b)) for a, b in zip(n, k))
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())

    def step():
        rc = L.CHAM_B200_dposv_batch(cb.ChamLower, count, ptr(dn), ptr(dk), ptr(A), ptr(da), ptr(B), ptr(db),
                                     ptr(info), None)
        assert rc == 0, rc

    times = []
    for it in range(args.warmup + args.steps):
        A.copy_(A0)
        B.copy_(B0)
        torch.cuda.synchronize()
        L.CHAM_B200_Event_Record(6)
        step()
        L.CHAM_B200_Event_Record(7)
        if it >= args.warmup:
            times.append(L.CHAM_B200_Event_Elapsed(6, 7))
    assert int(info.abs().sum()) == 0
    # accuracy on a sample: FP64 backward error against the generated inputs
    Ah, Bh, Xh = A0.cpu().numpy(), B0.cpu().numpy(), B.cpu().numpy()
    worst = 0.0
    for i in list(range(0, count, max(1, count // 24))):
        ni, ki = int(n[i]), int(k[i])
        Ai = Ah[a_off[i]:a_off[i] + ni * ni].reshape(ni, ni).T
        Ai = np.tril(Ai) + np.tril(Ai, -1).T
        Bi = Bh[b_off[i]:b_off[i] + ni * ki].reshape(ki, ni).T
        Xi = Xh[b_off[i]:b_off[i] + ni * ki].reshape(ki, ni).T
        r = np.abs(Bi - Ai @ Xi).max() / (np.abs(Ai).sum(1).max() * np.abs(Xi).max() * ni * 1.1102230246251565e-16)
        worst = max(worst, float(r))
    ms = statistics.median(times)
    ms_max = allreduce_max(ms, world)
    # plain path: one CHAMELEON_dposv (FP64 tile DAG) launch per matrix, device arrays
    plain_ms = None
    if rank == 0 and args.batch_plain:
        A.copy_(A0)
        B.copy_(B0)
        torch.cuda.synchronize()
        m = min(count, args.batch_plain)
        t0 = time.perf_counter()
        for i in range(m):
            ni, ki = int(n[i]), int(k[i])
            rc = L.CHAMELEON_dposv(cb.ChamLower, ni, ki, ctypes.c_void_p(A.data_ptr() + 8 * int(a_off[i])), ni,
                                   ctypes.c_void_p(B.data_ptr() + 8 * int(b_off[i])), ni)
            assert rc == 0, rc
        torch.cuda.synchronize()
        plain_ms = (time.perf_counter() - t0) * 1e3 * count / m
    # second plain path: the tile ABI per matrix (CUDA_dpotrf + two CUDA_dtrsm,
    # all on one stream, device arrays), every matrix of the batch
    A.copy_(A0)
    B.copy_(B0)
    torch.cuda.synchronize()
    hh = ctypes.c_void_p()
    assert L.CHAM_B200_Handle_Create(ctypes.byref(hh), None) == 0
    dinfo = torch.zeros(1, dtype=torch.int32, device="cuda")
    one = ctypes.c_double(1.0)
    L.CHAM_B200_Event_Record(6)
    for i in range(count):
        ni, ki = int(n[i]), int(k[i])
        pa = ctypes.c_void_p(A.data_ptr() + 8 * int(a_off[i]))
        pb = ctypes.c_void_p(B.data_ptr() + 8 * int(b_off[i]))
        assert L.CUDA_dpotrf(cb.ChamLower, ni, pa, ni, None, 0, ptr(dinfo), hh) == 0
        assert L.CUDA_dtrsm(cb.ChamLeft, cb.ChamLower, cb.ChamNoTrans, cb.ChamNonUnit, ni, ki, ctypes.byref(one),
                            pa, ni, pb, ni, hh) == 0
        assert L.CUDA_dtrsm(cb.ChamLeft, cb.ChamLower, cb.ChamTrans, cb.ChamNonUnit, ni, ki, ctypes.byref(one),
                            pa, ni, pb, ni, hh) == 0
    L.CHAM_B200_Event_Record(7)
    tile_abi_ms = L.CHAM_B200_Event_Elapsed(6, 7)
    L.CHAM_B200_Handle_Destroy(hh)
    tune = (ctypes.c_double * 28)()
    L.CHAM_B200_Batch_Tuning(cb.ChamRealDouble, tune)
    # FP32 systems: the same batch cast to FP32 through CHAM_B200_sposv_batch
    A32, B32 = A0.float(), B0.float()
    A, B = A32.clone(), B32.clone()
    t32 = []
    for it in range(args.warmup + args.steps):
        A.copy_(A32)
        B.copy_(B32)
        torch.cuda.synchronize()
        L.CHAM_B200_Event_Record(6)
        rc = L.CHAM_B200_sposv_batch(cb.ChamLower, count, ptr(dn), ptr(dk), ptr(A), ptr(da), ptr(B), ptr(db),
                                     ptr(info), None)
        assert rc == 0, rc
        L.CHAM_B200_Event_Record(7)
        if it >= args.warmup:
            t32.append(L.CHAM_B200_Event_Elapsed(6, 7))
    ms32 = allreduce_max(statistics.median(t32), world)
    del A0, B0, A, B, A32, B32
    sps = count * world / (ms_max * 1e-3)
    return {
        "workload": "%d SPD systems, n~U{%d..%d}, nrhs~U{1..8} (seed %d), dplgsy(bump=n, seed=%d+i, bigM=n), "
                    "FP64, Lower, one CHAM_B200_dposv_batch call per step" % (count, BATCH_NMIN, BATCH_NMAX,
                                                                              BATCH_SEED, BATCH_SEED),
        "solves_per_s": sps, "ms_per_step": ms_max, "tflops": flops * world / (ms_max * 1e-3) / 1e12,
        "backward_error_max_sampled": worst,
        "plain_per_matrix": ({"solves_per_s": count / (plain_ms * 1e-3), "ms": plain_ms,
                              "sampled_matrices": min(count, args.batch_plain),
                              "api": "CHAMELEON_dposv per matrix (device arrays)"} if plain_ms else None),
        "speedup_vs_plain": (plain_ms / ms_max) if plain_ms else None,
        "plain_tile_abi": {"solves_per_s": count / (tile_abi_ms * 1e-3), "ms": tile_abi_ms,
                           "api": "CUDA_dpotrf + 2 x CUDA_dtrsm per matrix on one stream (device arrays)"},
        "speedup_vs_tile_abi": tile_abi_ms / ms_max,
        "fp32": {"solves_per_s": count * world / (ms32 * 1e-3), "ms_per_step": ms32,
                 "api": "CHAM_B200_sposv_batch (FP32 systems)"},
        "size_bins": {"ranges": ["n<=64", "65..128", "129..256", "257+"],
                      "shape_per_range": [int(tune[r]) for r in range(4)],
                      "shape_ms_per_range": [[round(tune[4 + 6 * r + j], 4) for j in range(6)] for r in range(4)],
                      "shapes": ["generic x1", "small x1", "small x2", "small x3", "lean x2", "lean x3"],
                      "note": "autotuner: each size range runs the shape (kernel and CTAs per SM) that was "
                              "fastest on a synthetic batch of that range (-1: not admissible); adjacent "
                              "ranges with the same shape run as one launch"},
        "roofline": {"bound": "fp64", "achieved": flops / (ms_max * 1e-3) / 1e12, "peak": 40.0,
                     "unit": "TFLOP/s", "frac": flops / (ms_max * 1e-3) / 1e12 / 40.0,
                     "peak_source": "FP64 spec 40 TFLOP/s (fallback: no FP64 entry in the measured peaks)"},
    }


# ---------------------------------------------------------------------------
# Serving: Poisson arrivals, N = floor(exp(U(ln 64, ln 8192))), nrhs ~ U{1..32},
# 30% of requests reuse a kept factor with new right-hand sides
# ---------------------------------------------------------------------------
SERVE_NMIN, SERVE_NMAX, SERVE_SEED = 64, 8192, 77


class ServeLoad:
    """Host inputs of the serving workload: every request's matrix is the
    leading N x N block of one dplgsy(bump = 8192) matrix in pinned memory."""

    def __init__(self, cb):
        import torch
        self.cb = cb
        N = SERVE_NMAX
        self.A = torch.empty((N, N), dtype=torch.float64, pin_memory=True)   # column-major view: A[j, i] = a_ij
        self.B = torch.empty((32, N), dtype=torch.float64, pin_memory=True)
        dA = cb.Desc.create(N, N, 512)
        dB = cb.Desc.create(N, 32, 512)
        assert cb.dplgsy_Tile(float(N), cb.ChamUpperLower, dA, SEED_A) == 0
        assert cb.dplrnt_Tile(dB, SEED_B) == 0
        L = cb.lib()
        assert L.CHAMELEON_Desc2Lap(cb.ChamUpperLower, dA.ptr, ctypes.c_void_p(self.A.data_ptr()), N) == 0
        assert L.CHAMELEON_Desc2Lap(cb.ChamUpperLower, dB.ptr, ctypes.c_void_p(self.B.data_ptr()), N) == 0
        dA.destroy()
        dB.destroy()
        self.An = self.A.numpy()
        self.Bn = self.B.numpy()

    def draw(self, rng, count, reuse_frac=0.3):
        lo, hi = np.log(SERVE_NMIN), np.log(SERVE_NMAX)
        out = []
        for _ in range(count):
            Nr = int(np.floor(np.exp(rng.uniform(lo, hi))))
            Nr = min(max(Nr, SERVE_NMIN), SERVE_NMAX)
            out.append((Nr, int(rng.integers(1, 33)), bool(rng.random() < reuse_frac)))
        return out


NOT_FOUND = -105   # CHAMELEON_ERR_NOT_FOUND: the kept factor was released or replaced


def serve_run(cb, load, reqs, arrivals, slots, key_pool=32):
    """Submit `reqs` at `arrivals` (seconds from start; None: all at once).
    Returns per-request (N, latency s, status, reuse, X) and the elapsed time.
    A solve with a kept factor that the server has released or replaced in the
    meantime (NOT_FOUND) is resubmitted with its matrix, as a client would; its
    latency still counts from the original arrival."""
    sv = cb.Server(slots=slots)
    N0 = SERVE_NMAX
    kept = {}      # key -> (N, Request) of the request that made it
    next_key = 0
    done = []
    t0 = cb.Server.now()
    pending = []
    resubmitted = [0]

    def resubmit_not_found():
        for j, (Nk, kr, reuse, r, X, tarr) in enumerate(pending):
            if reuse and r.status == NOT_FOUND:
                r2 = sv.submit(load.An, load.Bn, X, N=Nk, nrhs=kr, factor_key=-1, lda=N0, ldb=N0, ldx=Nk)
                pending[j] = (Nk, kr, False, r2, X, tarr)
                resubmitted[0] += 1

    for i, (Nr, kr, reuse) in enumerate(reqs):
        if arrivals is not None:
            while cb.Server.now() - t0 < arrivals[i]:
                time.sleep(min(0.0005, max(0.0, arrivals[i] - (cb.Server.now() - t0))))
        resubmit_not_found()
        X = np.empty((kr, Nr))   # column-major N x nrhs
        ready = [key for key, (nk, r) in kept.items() if r.status == 0]
        if reuse and ready:
            key = ready[int(i * 2654435761) % len(ready)]
            Nk = kept[key][0]
            X = np.empty((kr, Nk))
            r = sv.submit(None, load.Bn, X, N=Nk, nrhs=kr, factor_key=key, ldb=N0, ldx=Nk)
            pending.append((Nk, kr, True, r, X, t0 + (arrivals[i] if arrivals is not None else 0.0)))
            continue
        key = -1
        if Nr > 512 and reuse is False and (i % 3 == 0):
            key = next_key % key_pool
            next_key += 1
        r = sv.submit(load.An, load.Bn, X, N=Nr, nrhs=kr, factor_key=key, lda=N0, ldb=N0, ldx=Nr)
        if key >= 0:
            kept[key] = (Nr, r)
        pending.append((Nr, kr, False, r, X, t0 + (arrivals[i] if arrivals is not None else 0.0)))
    while True:
        sv.drain()
        before = resubmitted[0]
        resubmit_not_found()
        if resubmitted[0] == before:
            break
    t1 = cb.Server.now()
    st = sv.stats()
    st["resubmitted"] = resubmitted[0]
    sv.close()
    for (Nr, kr, reuse, r, X, tarr) in pending:
        done.append((Nr, kr, reuse, r.t_done - tarr, r.status, X, r.iterations, r.t_done - r.t_start,
                     r.t_start - r.t_submit, r.t_submit - tarr))
    return done, t1 - t0, st


def serve_section(args, cb, rank):
    if rank != 0:
        return None
    load = ServeLoad(cb)
    rng = np.random.default_rng(SERVE_SEED)
    slots = args.serve_slots
    # capacity: closed loop, everything submitted at once
    cap_reqs = load.draw(rng, args.serve_cap_requests)
    serve_run(cb, load, cap_reqs[:16], None, slots)   # warm-up (schedules, workspaces)
    done, el, st = serve_run(cb, load, cap_reqs, None, slots)
    capacity = len(done) / el
    bad = [d for d in done if d[4] != 0]
    assert not bad, bad[:3]
    # accuracy on a sample of the capacity run
    worst = 0.0
    buckets = {}
    for d in done:
        key = "reuse" if d[2] else ("N<=512" if d[0] <= 512 else ("N<=2048" if d[0] <= 2048 else "N>2048"))
        buckets.setdefault(key, []).append(d[7] * 1e3)
    service = {k: {"count": len(v), "mean_ms": float(np.mean(v)), "p99_ms": float(np.percentile(v, 99))}
               for k, v in sorted(buckets.items())}
    for (Nr, kr, reuse, lat, status, X, it, svc, _q, _lag) in done[::max(1, len(done) // 12)]:
        Ai = load.An[:Nr, :Nr].T
        Ai = np.tril(Ai) + np.tril(Ai, -1).T
        Bi = load.Bn[:kr, :Nr].T
        Xi = X.T
        r = np.abs(Bi - Ai @ Xi).max() / (np.abs(Ai).sum(1).max() * np.abs(Xi).max() * Nr * 1.1102230246251565e-16)
        worst = max(worst, float(r))
    # plain path: one CHAMELEON_dsposv call per request, one after another
    L = cb.lib()
    plain_rate = None
    if args.serve_plain:
        m = min(len(cap_reqs), args.serve_plain)
        it = ctypes.c_int()
        cb.set_param(cb.CHAMELEON_TILE_SIZE, 512)
        t0 = time.perf_counter()
        for (Nr, kr, reuse) in cap_reqs[:m]:
            X = np.empty((kr, Nr))
            rc = L.CHAMELEON_dsposv(cb.ChamLower, Nr, kr, ctypes.c_void_p(load.A.data_ptr()), SERVE_NMAX,
                                    ctypes.c_void_p(load.B.data_ptr()), SERVE_NMAX, X.ctypes.data_as(ctypes.c_void_p),
                                    Nr, ctypes.byref(it))
            assert rc == 0, rc
        plain_rate = m / (time.perf_counter() - t0)
    loads = []
    for frac in args.serve_loads:
        rate = frac * capacity
        n_req = max(20, int(rate * args.serve_window))
        reqs = load.draw(rng, n_req)
        gaps = rng.exponential(1.0 / rate, size=n_req)
        arr = np.cumsum(gaps) - gaps[0]
        done, el, st = serve_run(cb, load, reqs, arr, slots)
        warm = int(0.1 * len(done))
        lat = np.array([d[3] for d in done[warm:]]) * 1e3
        failed = {}
        for d in done:
            if d[4] != 0:
                failed[str(d[4])] = failed.get(str(d[4]), 0) + 1
        slow = sorted(done[warm:], key=lambda d: -d[3])[:6]
        loads.append({"load_frac": frac, "offered_per_s": rate, "requests": len(done),
                      "slowest": [{"N": d[0], "nrhs": d[1], "reuse": d[2], "latency_ms": round(d[3] * 1e3, 2),
                                   "queue_ms": round(d[8] * 1e3, 2), "service_ms": round(d[7] * 1e3, 2),
                                   "submit_lag_ms": round(d[9] * 1e3, 2)} for d in slow],
                      "solves_per_s": len(done) / el, "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99)), "batches": st["batches"],
                      "batched_requests": st["batched_requests"], "max_batch": st["max_batch"],
                      "reused_factors": st["reused_factors"], "resubmitted_not_found": st["resubmitted"],
                      "failed_by_status": failed})
    return {
        "workload": "serving: N=floor(exp(U(ln 64, ln 8192))), nrhs~U{1..32}, 30%% reuse of a kept factor, "
                    "Poisson arrivals; mixed BF16x3 + FP64 refinement for N>512, batched FP64 for N<=512; host "
                    "pinned inputs, latency = arrival -> result in host memory; %d slots" % slots,
        "capacity_solves_per_s": capacity, "capacity_requests": len(cap_reqs),
        "capacity_service_ms": service,
        "backward_error_max_sampled": worst,
        "plain_per_request_solves_per_s": plain_rate,
        "speedup_vs_plain": (capacity / plain_rate) if plain_rate else None,
        "window_s": args.serve_window, "loads": loads,
    }


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
TRAFFIC_PROFILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles",
                               "cholesky_dag_f32_bf16x3_tcgen05_launch_traffic.md")


def traffic_capture():
    """(n0, bytes per launch, file) from the profile summary's key lines
    `order: <n0>` and `dram_bytes_per_launch: <bytes>`, or None."""
    try:
        kv = {}
        for line in open(TRAFFIC_PROFILE):
            if ":" in line and line.split(":", 1)[0].strip() in ("order", "dram_bytes_per_launch"):
                k, v = line.split(":", 1)
                kv[k.strip()] = float(v.split()[0])
        return int(kv["order"]), kv["dram_bytes_per_launch"], os.path.basename(TRAFFIC_PROFILE)
    except (OSError, KeyError, ValueError, IndexError):
        return None


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
    # DRAM bytes of the factor+solve launch: read from the committed summary of
    # a one-kernel ncu capture (dram__bytes_read.sum + dram__bytes_write.sum of
    # the launch at a smaller order n0), scaled to N by (N/n0)^3 -- the traffic
    # is dominated by the trailing updates' operand and C traffic
    traffic, traffic_src = None, None
    if args.precision == "bf16x3":
        cap = traffic_capture()
        if cap:
            n0, b0, fname = cap
            traffic = b0 * (N / float(n0)) ** 3
            traffic_src = "ncu dram__bytes_read.sum + dram__bytes_write.sum of the launch at N=%d (%s)%s" % (
                n0, fname, "" if N == n0 else ", scaled by (N/%d)^3" % n0)
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if (achieved and peak) else None, "traffic": traffic,
                "traffic_source": traffic_src,
                "kernel": "cholesky_dag_kernel<float,%s> (factorization + first solve)" % args.precision,
                "flops_per_launch": mult * fact_flops,
                "peak_source": peak_src + (" of measured" if peak else "")}

    # plain FP64 path on the same problem (reported beside the mixed number)
    fp64 = None
    ferr = None
    if args.compare_fp64 and rank == 0:
        dA2 = cb.Desc.create(N, N, NB)
        dB2 = cb.Desc.create(N, nrhs, NB)
        # one untimed call first (the task list of this shape is built and
        # cached on the first call, as for the mixed arm's warm-up steps)
        for timed in (False, True):
            cb.dplgsy_Tile(float(N), cb.ChamUpperLower, dA2, SEED_A)
            cb.dplrnt_Tile(dB2, SEED_B)
            if timed:
                L.CHAM_B200_Event_Record(2)
            assert cb.dposv_Tile(cb.ChamLower, dA2, dB2) == 0
        L.CHAM_B200_Event_Record(3)
        fms = L.CHAM_B200_Event_Elapsed(2, 3)
        fp64 = {"tflops": flops / (fms * 1e-3) / 1e12, "ms": fms}
        # forward error of the mixed solution against the plain FP64 one (same
        # inputs on rank 0)
        X64 = dB2.to_numpy()
        Xm = dX.to_numpy()
        ferr = float(np.abs(Xm - X64).max() / np.abs(X64).max())
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
        # the referenced triangle of A moves, one tile column of the FP32
        # factor's tiling at a time, while the factorization runs
        fnb = cb.get_param(cb.CHAMELEON_B200_FACTOR_NB)
        fnb = fnb if (0 < fnb < NB and NB % fnb == 0) else NB
        tri_bytes = sum(8 * (N - q * fnb) * min(fnb, N - q * fnb) for q in range((N + fnb - 1) // fnb))
        e2e = {"value": flops / (ems * 1e-3) / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": tri_bytes + 8 * N * nrhs,
               "d2h_bytes_per_step": 8 * N * nrhs, "ms_per_step": ems,
               "api": "CHAMELEON_dsposv (LAPACK layout, pinned host A/B/X; the lower triangle of A streams in "
                      "tile column by tile column while the factorization casts and factors the columns that "
                      "have landed)"}
        del hA

    cond = conditioning_section(args, cb, rank) if args.cond else None
    batch = batch_section(args, cb, world, rank) if args.batch else None
    serving = serve_section(args, cb, rank) if args.serve else None
    cpu = cpu_baseline_sample(N, NB, nrhs) if (rank == 0 and not args.no_cpu) else None
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
                   "backward_error_def": "max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf) of the returned x",
                   "forward_error_vs_fp64": ferr,
                   "phases_ms": {"factor+solve": stats[0], "refine_solves": stats[1], "residuals": stats[2],
                                 "casts+norm": stats[3], "total": stats[4]}},
        "fp64_plain": fp64,
        "speedup_vs_fp64_plain": (fp64["ms"] / (ms_max / args.steps)) if fp64 else None,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clk,
        "gpu_launches": launches,
        "conditioning": cond,
        "batch": batch,
        "serving": serving,
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
    ap.add_argument("--ref-n", type=int, default=None,
                    help="order of the reference arm's per-step solve (default: --n, the same workload)")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-fp64", dest="compare_fp64", action="store_false")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-cond", dest="cond", action="store_false")
    ap.add_argument("--cond-n", type=int, default=16384)
    ap.add_argument("--conds", type=float, nargs="+", default=[1e4, 1e6, 1e8, 1e12])
    ap.add_argument("--no-batch", dest="batch", action="store_false")
    ap.add_argument("--batch-count", type=int, default=BATCH_COUNT)
    ap.add_argument("--batch-plain", type=int, default=BATCH_COUNT,
                    help="matrices timed through the plain per-matrix path (0: skip)")
    ap.add_argument("--no-serve", dest="serve", action="store_false")
    ap.add_argument("--serve-slots", type=int, default=4)
    ap.add_argument("--serve-window", type=float, default=10.0, help="seconds of arrivals per load level")
    ap.add_argument("--serve-loads", type=float, nargs="+", default=[0.5, 0.8, 0.95])
    ap.add_argument("--serve-cap-requests", type=int, default=300)
    ap.add_argument("--serve-plain", type=int, default=100, help="requests timed through CHAMELEON_dsposv")
    args = ap.parse_args()
    if args.ref_n is None:
        args.ref_n = args.n
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
