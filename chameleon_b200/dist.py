"""Multi-GPU dispatch of independent SPD systems: one process per GPU.

Batches of systems and serving requests shard over the GPUs of a node with
no collective: rank 0 plans which GPU solves which system
(``CHAM_B200_Dispatch_Plan``: longest-first list scheduling with per-GPU
free-HBM admission and factor affinity), ships each GPU its share, and the
results come back to rank 0's host memory.  Every rank, rank 0 included, runs
a worker that solves its shares on its own GPU through the library's serving
loop (batched FP64 for small orders, mixed BF16x3 + FP64 refinement for large
ones).  The reference distributes the tiles of one matrix over a P x Q grid
(control/descriptor_helpers.c:51-56) for one large solve; this is the split
that needs no exchange.

Transport and liveness are host-side ``torch.distributed`` plumbing:
point-to-point messages on a gloo group (host tensors; the inputs live in
host memory and each worker copies its share to its GPU), and a heartbeat
counter per rank in the rendezvous store.  A rank is dead when its counter
stops moving for ``dead_after_s`` or when a message to or from it fails; a
rank whose solve raised is marked faulty.  Neither receives work again, and a
share that was lost with it is planned again over the ranks that remain.
Factors kept on a dead rank are gone: a request that names one completes with
CHAMELEON_ERR_NOT_FOUND, as with the single-GPU server.
"""
import ctypes
import os
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from datetime import timedelta

import numpy as np
import torch
import torch.distributed as dist

from . import ChamLower, ChameleonError, lib

OP_STOP, OP_SOLVE, OP_RESULT, OP_ERROR = 0, 1, 2, 3
HDR = 6                     # int64 header: op, batch id, count, payload doubles, meta ints, spare
META_IN = 4                 # per system in: n, nrhs, factor key, has A
META_OUT = 2                # per system out: status, iterations
ERR_NOT_FOUND = -105        # CHAMELEON_ERR_NOT_FOUND
ERR_UNEXPECTED = -110


def plan(n, nrhs, free_bytes, alive, load_s=None, pin=None):
    """CHAM_B200_Dispatch_Plan on Python lists; returns (owner, wave, nwaves)."""
    count, nranks = len(n), len(alive)
    i32 = lambda v: (ctypes.c_int * max(len(v), 1))(*[int(x) for x in v])
    f64 = lambda v: (ctypes.c_double * max(len(v), 1))(*[float(x) for x in v])
    owner = (ctypes.c_int * max(count, 1))()
    wave = (ctypes.c_int * max(count, 1))()
    rc = lib().CHAM_B200_Dispatch_Plan(count, i32(n), i32(nrhs), i32(pin) if pin is not None else None, nranks,
                                       i32(alive), f64(free_bytes), f64(load_s) if load_s is not None else None,
                                       owner, wave)
    if rc < 0:
        raise ChameleonError("CHAM_B200_Dispatch_Plan returned %d" % rc)
    return list(owner[:count]), list(wave[:count]), rc


def cost(n, nrhs):
    return lib().CHAM_B200_Dispatch_Cost(int(n), int(nrhs))


class Request:
    """One system: A (n x n, column-major, `uplo` triangle read; None to reuse
    the factor kept under `factor_key`) and B (n x nrhs).  After completion:
    X, status (0, LAPACK info > 0, or CHAMELEON_ERR_*), iterations, rank."""

    def __init__(self, A, B, factor_key=-1):
        B = np.asarray(B, dtype=np.float64)
        self.B = B.reshape(B.shape[0], -1)
        self.n, self.nrhs = self.B.shape
        self.A = None if A is None else np.asarray(A, dtype=np.float64)
        if self.A is not None and self.A.shape != (self.n, self.n):
            raise ValueError("A must be n x n with n = B.shape[0]")
        self.factor_key = int(factor_key)
        self.X = None
        self.status = None
        self.iterations = 0
        self.rank = -1
        self.done = False


def _pack(reqs):
    meta = np.zeros((len(reqs), META_IN), dtype=np.int64)
    parts = []
    for i, r in enumerate(reqs):
        meta[i] = (r.n, r.nrhs, r.factor_key, 0 if r.A is None else 1)
        if r.A is not None:
            parts.append(np.ravel(r.A, order="F"))
        parts.append(np.ravel(r.B, order="F"))
    payload = np.concatenate(parts) if parts else np.zeros(0)
    return torch.from_numpy(meta.ravel()), torch.from_numpy(np.ascontiguousarray(payload))


def _unpack(meta, payload):
    meta = meta.numpy().reshape(-1, META_IN)
    pay = payload.numpy()
    out, o = [], 0
    for n, nrhs, key, has_a in meta:
        n, nrhs = int(n), int(nrhs)
        A = None
        if has_a:
            A = pay[o:o + n * n].reshape((n, n), order="F")
            o += n * n
        B = pay[o:o + n * nrhs].reshape((n, nrhs), order="F")
        o += n * nrhs
        out.append(Request(A, B, int(key)))
    return out


class _ServerSolver:
    """A rank's solver on its own GPU: the library's serving loop (batched FP64
    for n <= small_n, the mixed solver on `slots` streams above)."""

    def __init__(self, uplo=ChamLower, slots=4):
        from . import Server
        self.uplo = uplo
        self.server = Server(slots=slots)

    def __call__(self, reqs):
        pending = []
        for r in reqs:
            X = np.zeros((r.n, r.nrhs), order="F")
            A = None if r.A is None else np.asfortranarray(r.A)
            B = np.asfortranarray(r.B)
            q = self.server.submit(A, B, X, nrhs=r.nrhs, N=r.n, uplo=self.uplo, factor_key=r.factor_key)
            pending.append((r, q, X, A, B))
        self.server.drain()
        for r, q, X, _, _ in pending:
            r.X, r.status, r.iterations = X, int(q.status), int(q.iterations)
        return reqs

    def close(self):
        self.server.close()


def _gpu_free_bytes():
    free, _ = torch.cuda.mem_get_info()
    return float(free)


class _Beat:
    """Heartbeat of one rank: a counter in the store, bumped every `period_s`
    from a thread with its own store connection; the rank's free device bytes
    beside it."""

    def __init__(self, host, port, rank, period_s, free_fn):
        self.store = dist.TCPStore(host, port, is_master=False, timeout=timedelta(seconds=30))
        self.rank, self.period, self.free_fn = rank, period_s, free_fn
        self.stop = threading.Event()
        self.lock = threading.Lock()        # one store connection, two threads
        self.publish_free()
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def publish_free(self):
        v = repr(float(self.free_fn()))
        with self.lock:
            self.store.set("chb/free/%d" % self.rank, v)

    def _run(self):
        while not self.stop.is_set():
            try:
                with self.lock:
                    self.store.add("chb/hb/%d" % self.rank, 1)
            except Exception:
                return
            self.stop.wait(self.period)

    def close(self, leave=True):
        self.stop.set()
        self.t.join(timeout=5)
        if leave:
            try:
                with self.lock:
                    self.store.add("chb/leave/%d" % self.rank, 1)
            except Exception:
                pass


def _store_addr(store_addr):
    if store_addr is not None:
        return store_addr
    return os.environ.get("MASTER_ADDR", "127.0.0.1"), int(os.environ["MASTER_PORT"])


def make_group():
    """The gloo group the dispatcher and the workers talk on (the default
    group itself when it is gloo).  Collective: every rank calls it once."""
    if dist.get_backend() == "gloo":
        return dist.group.WORLD
    return dist.new_group(backend="gloo")


class Worker:
    """The solving side of a rank other than 0: receive a share, solve it on
    this rank's GPU, send the results back; until rank 0 says stop."""

    def __init__(self, group, solve=None, free_fn=None, store_addr=None, beat_s=0.1):
        self.g = group
        self.rank = dist.get_rank()
        self.solve = solve if solve is not None else _ServerSolver()
        self.beat = _Beat(*_store_addr(store_addr), self.rank, beat_s, free_fn or _gpu_free_bytes)
        dist.barrier(group=self.g)          # every rank's free memory is published

    def serve_forever(self):
        try:
            while True:
                hdr = torch.zeros(HDR, dtype=torch.int64)
                dist.recv(hdr, src=0, group=self.g)
                op, bid, count, npay, nmeta = (int(x) for x in hdr[:5])
                if op == OP_STOP:
                    break
                meta = torch.zeros(nmeta, dtype=torch.int64)
                pay = torch.zeros(npay, dtype=torch.float64)
                dist.recv(meta, src=0, group=self.g)
                dist.recv(pay, src=0, group=self.g)
                reqs = _unpack(meta, pay)
                try:
                    reqs = self.solve(reqs)
                    om = np.array([(r.status, r.iterations) for r in reqs], dtype=np.int64).ravel()
                    op_out = OP_RESULT
                    xs = [np.ravel(r.X, order="F") for r in reqs]
                    op_pay = np.concatenate(xs) if xs else np.zeros(0)
                except Exception:
                    op_out, om, op_pay = OP_ERROR, np.zeros(0, dtype=np.int64), np.zeros(0)
                self.beat.publish_free()
                out_hdr = torch.tensor([op_out, bid, count, op_pay.size, om.size, 0], dtype=torch.int64)
                dist.send(out_hdr, dst=0, group=self.g)
                dist.send(torch.from_numpy(om), dst=0, group=self.g)
                dist.send(torch.from_numpy(np.ascontiguousarray(op_pay)), dst=0, group=self.g)
        finally:
            self.beat.close(leave=True)
            close = getattr(self.solve, "close", None)
            if close:
                close()


class _Channel:
    """Rank 0's link to one rank: start a share, poll for its results."""

    def __init__(self, disp, rank):
        self.d, self.rank = disp, rank
        self.share = None
        self.bid = -1

    @property
    def busy(self):
        return self.share is not None


class _LocalChannel(_Channel):
    def __init__(self, disp, solve):
        super().__init__(disp, 0)
        self.solve = solve
        self.pool = ThreadPoolExecutor(max_workers=1)
        self.fut = None

    def start(self, share, bid):
        self.share, self.bid = share, bid
        copies = [Request(r.A, r.B, r.factor_key) for r in share]
        self.fut = self.pool.submit(self.solve, copies)

    def poll(self):
        """None while running; ('ok', results) / ('error', None) when done."""
        if not self.fut.done():
            return None
        share, self.share = self.share, None
        try:
            res = self.fut.result()
        except Exception:
            return share, "error", None
        return share, "ok", res


class _RemoteChannel(_Channel):
    """Sends a share from the calling thread; a thread of its own blocks in the
    receive of the results (gloo's non-blocking receive reports completion
    only to a waiter), so poll() only looks at a future."""

    def __init__(self, disp, rank):
        super().__init__(disp, rank)
        self.pool = ThreadPoolExecutor(max_workers=1)
        self.fut = None

    def start(self, share, bid):
        self.share, self.bid = share, bid
        meta, pay = _pack(share)
        hdr = torch.tensor([OP_SOLVE, bid, len(share), pay.numel(), meta.numel(), 0], dtype=torch.int64)
        try:
            dist.send(hdr, dst=self.rank, group=self.d.g)
            dist.send(meta, dst=self.rank, group=self.d.g)
            dist.send(pay, dst=self.rank, group=self.d.g)
        except Exception:
            self.fut = None
            return False
        self.fut = self.pool.submit(self._receive)
        return True

    def _receive(self):
        hdr = torch.zeros(HDR, dtype=torch.int64)
        dist.recv(hdr, src=self.rank, group=self.d.g)
        op, bid, count, npay, nmeta = (int(x) for x in hdr[:5])
        meta = torch.zeros(nmeta, dtype=torch.int64)
        pay = torch.zeros(npay, dtype=torch.float64)
        dist.recv(meta, src=self.rank, group=self.d.g)
        dist.recv(pay, src=self.rank, group=self.d.g)
        return op, bid, count, meta, pay

    def poll(self):
        if self.fut is None:
            share, self.share = self.share, None
            return share, "dead", None
        if not self.fut.done():
            return None
        share, self.share = self.share, None
        try:
            op, bid, count, meta, pay = self.fut.result()
        except Exception:
            return share, "dead", None
        if op != OP_RESULT or bid != self.bid or count != len(share):
            return share, "error", None
        om = meta.numpy().reshape(-1, META_OUT)
        p = pay.numpy()
        res, o = [], 0
        for r, (st, it) in zip(share, om):
            c = Request(None, r.B, r.factor_key)
            c.X = p[o:o + r.n * r.nrhs].reshape((r.n, r.nrhs), order="F").copy()
            o += r.n * r.nrhs
            c.status, c.iterations = int(st), int(it)
            res.append(c)
        return share, "ok", res


class Dispatcher:
    """Rank 0: plans and ships shares of independent systems to every rank
    (itself included) and gathers the results.

    ``dposv_batch`` solves a list of systems (waves when they do not fit in
    the GPUs' free memory at once); ``submit`` / ``drain`` serve a stream of
    requests with continuous micro-batching: a request is routed on arrival to
    the live rank with the least outstanding estimated work that admits it (or
    to the rank that keeps its factor), and each idle rank receives everything
    queued for it as one share.
    """

    def __init__(self, group, solve=None, free_fn=None, store_addr=None, beat_s=0.1, dead_after_s=2.0,
                 hbm_fraction=0.8):
        self.g = group
        self.world = dist.get_world_size(group)
        if dist.get_rank() != 0:
            raise ChameleonError("the dispatcher runs on rank 0")
        host, port = _store_addr(store_addr)
        self.store = dist.TCPStore(host, port, is_master=False, timeout=timedelta(seconds=30))
        self.beat = _Beat(host, port, 0, beat_s, free_fn or _gpu_free_bytes)
        self.dead_after = dead_after_s
        self.hbm_fraction = hbm_fraction
        self.chan = [_LocalChannel(self, solve if solve is not None else _ServerSolver())]
        self.chan += [_RemoteChannel(self, r) for r in range(1, self.world)]
        self.dead = [False] * self.world
        self.faulty = [False] * self.world
        self._hb = [(-1, time.monotonic())] * self.world
        self.key_owner = {}
        self.queue = [[] for _ in range(self.world)]
        self.outstanding = [0.0] * self.world
        self.open = []
        self.bid = 0
        self.systems_per_rank = [0] * self.world
        dist.barrier(group=self.g)

    # ---- liveness ----------------------------------------------------------
    def alive(self, r):
        if self.dead[r] or self.faulty[r]:
            return False
        if r == 0:
            return True
        if self.store.add("chb/leave/%d" % r, 0) > 0:
            self._mark_dead(r)
            return False
        c = self.store.add("chb/hb/%d" % r, 0)
        last, t = self._hb[r]
        now = time.monotonic()
        if c != last:
            self._hb[r] = (c, now)
        elif now - t > self.dead_after:
            self._mark_dead(r)
            return False
        return True

    def _mark_dead(self, r):
        self.dead[r] = True
        self._drop_keys(r)

    def _drop_keys(self, r):
        for k in [k for k, v in self.key_owner.items() if v == r]:
            del self.key_owner[k]

    def _free(self, r):
        key = "chb/free/%d" % r
        if not self.store.check([key]):
            return 0.0
        return float(self.store.get(key).decode()) * self.hbm_fraction

    def _alive_vec(self):
        return [1 if self.alive(r) else 0 for r in range(self.world)]

    # ---- batch -------------------------------------------------------------
    def dposv_batch(self, reqs):
        """Solve every Request; returns them completed (X, status, rank)."""
        todo = list(reqs)
        while todo:
            alive = self._alive_vec()
            keep, pin = [], []
            for r in todo:
                p = -1
                if r.A is None and r.factor_key >= 0:
                    p = self.key_owner.get(r.factor_key, -1)
                    if p < 0 or not alive[p]:
                        self._complete_missing(r)
                        continue
                keep.append(r)
                pin.append(p)
            todo = keep
            if not todo:
                break
            free = [self._free(r) if alive[r] else 0.0 for r in range(self.world)]
            owner, wave, nw = plan([r.n for r in todo], [r.nrhs for r in todo], free, alive, pin=pin)
            retry = []
            for w in range(nw):
                shares = {}
                for r, o, wv in zip(todo, owner, wave):
                    if wv == w:
                        shares.setdefault(o, []).append(r)
                retry += self._run_shares(shares)
            todo = retry
        return reqs

    def _complete_missing(self, r):
        r.X = np.zeros((r.n, r.nrhs), order="F")
        r.status, r.done, r.rank = ERR_NOT_FOUND, True, -1

    def _run_shares(self, shares):
        """Start every share, wait for all; returns the requests to retry."""
        retry = []
        for rk, share in shares.items():
            if not self._start(rk, share):
                retry += share
        while any(c.busy for c in self.chan):
            retry += self._poll_all()
            time.sleep(0.0005)
        return retry

    def _start(self, rk, share):
        self.bid += 1
        for r in share:
            if r.A is not None and r.factor_key >= 0:
                self.key_owner[r.factor_key] = rk
        ok = self.chan[rk].start(share, self.bid)
        if ok is False:
            self._mark_dead(rk)
            self.chan[rk].share = None
            return False
        return True

    def _poll_all(self):
        retry = []
        for c in self.chan:
            if not c.busy:
                continue
            if c.rank != 0 and not self.alive(c.rank):
                retry += c.share
                c.share = None
                continue
            got = c.poll()
            if got is None:
                continue
            share, how, res = got
            if how == "ok":
                self.systems_per_rank[c.rank] += len(share)
                for r, x in zip(share, res):
                    r.X, r.status, r.iterations, r.rank, r.done = x.X, x.status, x.iterations, c.rank, True
                    self.outstanding[c.rank] = max(0.0, self.outstanding[c.rank] - cost(r.n, r.nrhs))
            else:
                if how == "dead":
                    self._mark_dead(c.rank)
                else:
                    self.faulty[c.rank] = True
                    self._drop_keys(c.rank)
                for r in share:
                    self.outstanding[c.rank] = max(0.0, self.outstanding[c.rank] - cost(r.n, r.nrhs))
                retry += share
        return retry

    # ---- serving -----------------------------------------------------------
    def submit(self, req):
        """Route one request; it completes during pump() / drain()."""
        alive = self._alive_vec()
        pin = -1
        if req.factor_key >= 0 and req.A is None:
            pin = self.key_owner.get(req.factor_key, -1)
            if pin < 0:
                self._complete_missing(req)
                return req
        free = [self._free(r) if alive[r] else 0.0 for r in range(self.world)]
        owner, _, _ = plan([req.n], [req.nrhs], free, alive, load_s=self.outstanding, pin=[pin])
        rk = owner[0]
        if req.A is not None and req.factor_key >= 0:
            self.key_owner[req.factor_key] = rk
        self.queue[rk].append(req)
        self.outstanding[rk] += cost(req.n, req.nrhs)
        self.open.append(req)
        return req

    def pump(self):
        """Start a share on every idle live rank with queued requests, collect
        finished shares; lost or failed shares are routed again."""
        for rk in range(self.world):
            if self.queue[rk] and not self.chan[rk].busy:
                if not self.alive(rk):
                    self._reroute(self.queue[rk])
                    self.queue[rk] = []
                    continue
                share, self.queue[rk] = self.queue[rk], []
                if not self._start(rk, share):
                    self._reroute(share)
        self._reroute(self._poll_all())
        self.open = [r for r in self.open if not r.done]

    def _reroute(self, reqs):
        for r in reqs:
            self.open = [q for q in self.open if q is not r]
            self.submit(r)

    def drain(self):
        while self.open or any(c.busy for c in self.chan) or any(self.queue):
            self.pump()
            time.sleep(0.0005)

    def close(self):
        """Stop every live remote worker and this rank's own solver."""
        self.drain()
        for rk in range(1, self.world):
            if not self.dead[rk]:
                try:
                    dist.send(torch.tensor([OP_STOP, 0, 0, 0, 0, 0], dtype=torch.int64), dst=rk, group=self.g)
                except Exception:
                    pass
        self.beat.close(leave=False)
        for c in self.chan[1:]:
            c.pool.shutdown(wait=False)
        loc = self.chan[0]
        loc.pool.shutdown(wait=True)
        close = getattr(loc.solve, "close", None)
        if close:
            close()
