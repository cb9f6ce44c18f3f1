"""Multi-GPU dispatch of independent systems, host logic on CPU.

The planner (CHAM_B200_Dispatch_Plan) is checked directly; the dispatcher and
its workers run as world_size-2 gloo ranks in child processes, with a numpy
Cholesky solve standing in for each GPU's solver (the transport, routing,
factor affinity and failure handling are what is under test here; the GPU
solvers have their own parity tests).  Failures are made on the host: a rank
that exits between requests without a word, and a rank whose solve raises.
"""
import multiprocessing as mp
import os
import socket
import time
import traceback

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# ---- planner ------------------------------------------------------------------

def test_plan_balances_longest_first():
    from chameleon_b200 import dist as cd
    n = [4096, 64, 2048, 4096, 128, 1024, 64, 3000, 512, 8192]
    nrhs = [8, 1, 4, 2, 1, 16, 3, 1, 5, 32]
    owner, wave, nw = cd.plan(n, nrhs, [1e12] * 3, [1, 1, 1])
    assert nw == 1 and set(wave) == {0}
    load = [0.0] * 3
    for i, o in enumerate(owner):
        load[o] += cd.cost(n[i], nrhs[i])
    costs = sorted((cd.cost(a, b) for a, b in zip(n, nrhs)), reverse=True)
    # LPT bound: max load <= optimal + largest item <= total/3 + largest
    assert max(load) <= sum(costs) / 3 + costs[0] + 1e-12
    # the largest system is placed first, on rank 0 (ties go to the lowest rank)
    assert owner[n.index(8192)] == 0


def test_plan_respects_liveness_memory_pins_and_waves():
    from chameleon_b200 import dist as cd
    from chameleon_b200 import lib
    n = [1000] * 6
    nrhs = [1] * 6
    b = lib().CHAM_B200_Dispatch_Bytes(1000, 1)
    # rank 1 dead: everything on 0 and 2
    owner, _, _ = cd.plan(n, nrhs, [1e12] * 3, [1, 0, 1])
    assert set(owner) == {0, 2}
    # each GPU admits two systems at once: 6 systems on 2 live GPUs = 2 waves
    owner, wave, nw = cd.plan(n, nrhs, [2.5 * b, 2.5 * b, 0.0], [1, 1, 1])
    assert nw == 2
    for w in range(nw):
        for r in (0, 1):
            assert sum(1 for o, wv in zip(owner, wave) if o == r and wv == w) <= 2
    assert all(o in (0, 1) for o in owner)
    # pins win over balance when the pinned GPU is alive
    owner, _, _ = cd.plan(n, nrhs, [1e12] * 3, [1, 1, 1], pin=[2] * 6)
    assert owner == [2] * 6
    # a system that fits on no live GPU, and no live GPU at all
    with pytest.raises(Exception, match="-106"):
        cd.plan([1000], [1], [b / 2, b / 2], [1, 1])
    with pytest.raises(Exception, match="-101"):
        cd.plan([10], [1], [1e9, 1e9], [0, 0])
    # outstanding load steers new work away from a busy GPU
    owner, _, _ = cd.plan([200], [1], [1e12] * 2, [1, 1], load_s=[5.0, 0.0])
    assert owner == [1]


# ---- two ranks over gloo ------------------------------------------------------

def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class NumpySolver:
    """Stand-in for one GPU's solver: Cholesky in numpy, factors kept by key."""

    def __init__(self, raise_first=False):
        self.kept = {}
        self.raise_first = raise_first
        self.calls = 0

    def __call__(self, reqs):
        self.calls += 1
        if self.raise_first and self.calls == 1:
            raise RuntimeError("planted solver failure")
        for r in reqs:
            if r.A is None:
                L = self.kept.get(r.factor_key)
                if L is None:
                    r.status, r.X = -105, np.zeros((r.n, r.nrhs))
                    continue
            else:
                A = np.tril(r.A) + np.tril(r.A, -1).T
                L = np.linalg.cholesky(A)
                if r.factor_key >= 0:
                    self.kept[r.factor_key] = L
            Y = np.linalg.solve(L, r.B)
            r.X, r.status = np.linalg.solve(L.T, Y), 0
        return reqs


def _spd(rng, n):
    M = rng.standard_normal((n, n))
    return M @ M.T / n + np.eye(n)


def _check(req, A):
    Af = np.tril(A) + np.tril(A, -1).T
    assert req.status == 0, req.status
    assert np.abs(Af @ req.X - req.B).max() < 1e-9 * max(1.0, np.abs(req.B).max())


def _rank0_fail(d, cd, store):
    rng = np.random.default_rng(5)
    # 1. a batch spreads over both ranks and comes back correct
    mats = [_spd(rng, int(n)) for n in rng.integers(8, 160, size=40)]
    reqs = [cd.Request(A, rng.standard_normal((A.shape[0], int(rng.integers(1, 5))))) for A in mats]
    d.dposv_batch(reqs)
    for r, A in zip(reqs, mats):
        _check(r, A)
    assert d.systems_per_rank[0] > 0 and d.systems_per_rank[1] > 0
    # 2. serving: factors kept under keys, reuse requests follow their factor
    keyed = {}
    for k in range(6):
        A = _spd(rng, 50 + 10 * k)
        keyed[k] = A
        d.submit(cd.Request(A, rng.standard_normal((A.shape[0], 2)), factor_key=k))
    d.drain()
    owner_of = dict(d.key_owner)
    assert set(owner_of) == set(range(6))
    reuse = []
    for k in range(6):
        A = keyed[k]
        reuse.append((k, d.submit(cd.Request(None, rng.standard_normal((A.shape[0], 3)), factor_key=k))))
    d.drain()
    for k, r in reuse:
        _check(r, keyed[k])
        assert r.rank == owner_of[k]
    # 3. rank 1 dies between requests; the dispatcher notices from its heartbeat
    on1 = [k for k, o in owner_of.items() if o == 1]
    assert on1 and len(on1) < 6              # the keyed requests were spread
    store.set("test/die", "1")
    t0 = time.time()
    while d.alive(1):
        assert time.time() - t0 < 20, "dead rank not detected"
        time.sleep(0.05)
    mats = [_spd(rng, int(n)) for n in rng.integers(8, 120, size=20)]
    reqs = [cd.Request(A, rng.standard_normal((A.shape[0], 2))) for A in mats]
    before = list(d.systems_per_rank)
    d.dposv_batch(reqs)
    for r, A in zip(reqs, mats):
        _check(r, A)
        assert r.rank == 0
    assert d.systems_per_rank[1] == before[1]
    # a factor kept on the dead rank is gone: NOT_FOUND, then a resubmission with A works
    k = on1[0]
    r = d.submit(cd.Request(None, rng.standard_normal((keyed[k].shape[0], 1)), factor_key=k))
    d.drain()
    assert r.status == -105
    r = d.submit(cd.Request(keyed[k], rng.standard_normal((keyed[k].shape[0], 1)), factor_key=k))
    d.drain()
    _check(r, keyed[k])
    assert r.rank == 0
    return {"on1": len(on1), "per_rank": d.systems_per_rank}


def _rank0_raise(d, cd, store):
    rng = np.random.default_rng(9)
    mats = [_spd(rng, int(n)) for n in rng.integers(8, 100, size=24)]
    reqs = [cd.Request(A, rng.standard_normal((A.shape[0], 2))) for A in mats]
    d.dposv_batch(reqs)
    for r, A in zip(reqs, mats):
        _check(r, A)
        assert r.rank == 0
    assert d.faulty[1] and not d.dead[1]
    assert d.systems_per_rank[1] == 0
    # serving keeps working on the remaining rank
    A = _spd(rng, 77)
    r = d.submit(cd.Request(A, rng.standard_normal((77, 4))))
    d.drain()
    _check(r, A)
    return {"per_rank": d.systems_per_rank}


def _rank_main(rank, world, port, scenario, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import sys
        sys.path.insert(0, ROOT)
        from datetime import timedelta
        import torch.distributed as dist
        from chameleon_b200 import dist as cd
        store = dist.TCPStore("127.0.0.1", port, world, rank == 0, timeout=timedelta(seconds=60))
        dist.init_process_group("gloo", store=store, rank=rank, world_size=world, timeout=timedelta(seconds=30))
        g = cd.make_group()
        if rank == 0:
            d = cd.Dispatcher(g, solve=NumpySolver(), free_fn=lambda: 4e9, dead_after_s=1.0, beat_s=0.05)
            out = (_rank0_fail if scenario == "fail" else _rank0_raise)(d, cd, store)
            d.close()
            q.put((rank, "ok", out))
        else:
            w = cd.Worker(g, solve=NumpySolver(raise_first=(scenario == "raise")), free_fn=lambda: 4e9, beat_s=0.05)
            if scenario == "fail":
                import threading

                def die():
                    while not store.check(["test/die"]):
                        time.sleep(0.02)
                    q.put((rank, "died", None))
                    q.close()
                    q.join_thread()         # the message is out before the process ends
                    os._exit(17)            # no goodbye: heartbeat stops, sockets close
                threading.Thread(target=die, daemon=True).start()
            w.serve_forever()
            q.put((rank, "ok", None))
        dist.destroy_process_group()
    except Exception:
        q.put((rank, "error", traceback.format_exc()))
        raise


def _run(scenario):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, scenario, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        msgs = {}
        deadline = time.time() + 120
        while len(msgs) < 2 and time.time() < deadline:
            try:
                r, how, out = q.get(timeout=1)
            except Exception:
                continue
            msgs[r] = (how, out)
            assert how != "error", out
        for p in procs:
            p.join(timeout=30)
        return msgs, [p.exitcode for p in procs]
    finally:
        for p in procs:
            if p.is_alive():
                p.kill()


def test_dispatch_two_ranks_with_rank_failure_between_requests():
    msgs, codes = _run("fail")
    assert msgs[0][0] == "ok" and msgs[1][0] == "died", msgs
    assert codes == [0, 17]


def test_dispatch_reroutes_a_share_whose_solve_raised():
    msgs, codes = _run("raise")
    assert msgs[0][0] == "ok" and msgs[1][0] == "ok", msgs
    assert codes == [0, 0]
