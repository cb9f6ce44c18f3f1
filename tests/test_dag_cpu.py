"""Host-side checks of the persistent executor's task DAG (no GPU).

1. Deadlock freedom: walking the task list in order, every task's wait
   predicate -- the exact counter conditions the device kernel spins on -- is
   already satisfied by the tasks before it.  With dispatch by an atomic cursor
   this proves the launch always progresses, whatever the number of CTAs.
2. Data flow: executing the same list on the host with numpy (each task doing
   the device task's sub-block arithmetic) reproduces the Cholesky factor and
   the solution of the oracle.
"""
import numpy as np
import pytest
import scipy.linalg as sla

TK_POTRF, TK_TRSM, TK_UPD, TK_FWD_TRSM, TK_FWD_UPD, TK_BWD_TRSM, TK_BWD_UPD, TK_INV, TK_XINV, TK_CAST = range(1, 11)
SUBB = 128
SOLB = 64     # row block of the substitutions with full tile inverses (MODE_XINV)
FACT, SOLVE, XINV, NOINV, CAST = 1, 2, 4, 8, 16


def ngroups(n, G, tail=2):
    """Update groups of tile column n (upd_ngroups in executor.cuh): the last
    `tail` panels alone, the panels before them in groups of G aligned at the
    end (the first group takes the remainder)."""
    if n <= tail:
        return max(n, 0)
    return -(-(n - tail) // G) + tail


def geometry(N, NB, nrhs, NBB):
    NT = -(-N // NB)
    NTB = -(-nrhs // NBB) if nrhs else 0
    tm = lambda m: N - m * NB if m == NT - 1 else NB
    nbi = lambda m: -(-tm(m) // SUBB)
    S = lambda m, n: nbi(m) * (nbi(m) + 1) // 2 if m == n else nbi(m) * nbi(n)
    return NT, NTB, tm, nbi, S


def check_waits(tasks, mode, N, NB, nrhs, NBB, G=1):
    NT, NTB, tm, nbi, S = geometry(N, NB, nrhs, NBB)
    upd = np.zeros((NT, NT), int); pan = np.zeros((NT, NT), int)
    fwdB = np.zeros((NT, max(NTB, 1)), int); fwdD = np.zeros_like(fwdB)
    bwdB = np.zeros_like(fwdB); bwdD = np.zeros_like(fwdB)
    xinv = np.zeros(NT, int)
    fact = bool(mode & FACT)
    # with full tile inverses (XINV) each substitution is split into row blocks
    srb = SOLB if mode & XINV else SUBB
    nsb = lambda m: -(-tm(m) // srb)
    ns = (lambda k: nsb(k)) if mode & XINV else (lambda k: 1)
    applied = {}   # (m, n, bi, bj) -> panels applied so far, in order
    cast = np.zeros((NT, NT), int)
    ccast = bool(mode & CAST)   # the host's arrival flags are external: assumed set
    for kind, sub, m, n, k, bn, grp in tasks:
        if kind == TK_CAST:
            ok = m >= n and cast[m, n] == 0; cast[m, n] += 1
        elif kind == TK_POTRF:
            ok = upd[k, k] >= ngroups(k, G) * S(k, k) and (not ccast or k > 0 or cast[0, 0] == 1); pan[k, k] += 1
        elif kind == TK_INV:
            ok = True; pan[k, k] += 1
        elif kind == TK_XINV:
            ok = (not fact) or pan[k, k] >= 1; xinv[k] += 1
        elif kind == TK_TRSM:
            ok = pan[k, k] >= 1 and upd[m, k] >= ngroups(k, G) * S(m, k) and (not ccast or k > 0 or cast[m, 0] == 1)
            pan[m, k] += 1
        elif kind == TK_UPD:
            kl = k + bn - 1
            ok = pan[m, kl] >= nbi(m) and pan[n, kl] >= nbi(n) and upd[m, n] >= grp * S(m, n)
            ok = ok and (not ccast or grp > 0 or cast[m, n] == 1)
            upd[m, n] += 1
            # every sub-block sees each panel k < n exactly once, in order
            key = (m, n, sub)
            assert applied.get(key, 0) == k, (key, applied.get(key, 0), k)
            applied[key] = k + bn
        elif kind == TK_FWD_TRSM:
            if mode & XINV:
                inv_ok = bool(mode & NOINV) or xinv[k] >= 1
            else:
                inv_ok = pan[k, k] >= 1
            ok = inv_ok and fwdB[k, bn] >= k * nsb(k); fwdD[k, bn] += 1
        elif kind == TK_FWD_UPD:
            ok = fwdD[k, bn] >= ns(k) and (not fact or pan[m, k] >= nbi(m)) and fwdB[m, bn] >= k * nsb(m)
            fwdB[m, bn] += 1
        elif kind == TK_BWD_TRSM:
            ok = fwdD[k, bn] >= ns(k) and bwdB[k, bn] >= (NT - 1 - k) * nsb(k); bwdD[k, bn] += 1
        elif kind == TK_BWD_UPD:
            ok = bwdD[k, bn] >= ns(k) and bwdB[m, bn] >= (NT - 1 - k) * nsb(m); bwdB[m, bn] += 1
        else:
            raise AssertionError(kind)
        assert ok, (kind, sub, m, n, k, bn)
    # every tile got all of its updates / solves
    if fact:
        for m in range(NT):
            for n in range(m + 1):
                assert upd[m, n] == ngroups(n, G) * S(m, n)
        assert all(v == key[1] for key, v in applied.items())
        if ccast:
            assert (cast[np.tril_indices(NT)] == 1).all() and not np.triu(cast, 1).any()
    if mode & SOLVE:
        want = np.array([ns(k) for k in range(NT)])[:, None]
        assert (fwdD[:, :NTB] == want).all() and (bwdD[:, :NTB] == want).all()
    if (mode & XINV) and (mode & SOLVE) and not (mode & NOINV):
        assert (xinv == 1).all()
    else:
        assert (xinv == 0).all()


def emulate(tasks, A, B, uplo, N, NB, NBB, xinv=False):
    """Run the task list on host arrays with the device tasks' arithmetic.
    xinv: substitutions split into row blocks, forward results in a separate
    array Y (forward reads B writes Y, backward reads Y writes B)."""
    NT, NTB, tm, nbi, S = geometry(N, NB, B.shape[1] if B is not None else 0, NBB)
    M = A if uplo == 122 else A.T          # logical lower view (writes land in A)
    L = lambda m, n: M[m * NB:m * NB + tm(m), n * NB:n * NB + tm(n)]
    Bt = lambda m, bn: B[m * NB:m * NB + tm(m), bn * NBB:min((bn + 1) * NBB, B.shape[1])]
    Y = np.full_like(B, np.nan) if B is not None else None
    Yt = lambda m, bn: Y[m * NB:m * NB + tm(m), bn * NBB:min((bn + 1) * NBB, B.shape[1])]
    for kind, sub, m, n, k, bn, grp in tasks:
        if kind == TK_CAST:
            continue
        if kind == TK_POTRF:
            T = L(k, k)
            T[np.tril_indices(T.shape[0])] = np.linalg.cholesky(np.tril(T) + np.tril(T, -1).T)[
                np.tril_indices(T.shape[0])]
        elif kind == TK_TRSM:
            X = L(m, k)[sub * SUBB:(sub + 1) * SUBB]
            X[:] = sla.solve_triangular(np.tril(L(k, k)), X.T, lower=True).T
        elif kind == TK_UPD:
            bi, bj = sub & 0xFF, (sub >> 8) & 0xFF
            C = L(m, n)[bi * SUBB:(bi + 1) * SUBB, bj * SUBB:(bj + 1) * SUBB]
            upd = sum(L(m, kk)[bi * SUBB:(bi + 1) * SUBB] @ L(n, kk)[bj * SUBB:(bj + 1) * SUBB].T
                      for kk in range(k, k + bn))
            if m == n and bi == bj:
                upd = np.tril(upd)
            C -= upd
        elif kind in (TK_INV, TK_XINV):
            pass   # inverses of diagonal tiles: the emulation solves triangular systems directly
        elif kind == TK_FWD_TRSM and xinv:
            r = slice(sub * SOLB, (sub + 1) * SOLB)
            Yt(k, bn)[r] = np.linalg.inv(np.tril(L(k, k)))[r] @ Bt(k, bn)
        elif kind == TK_BWD_TRSM and xinv:
            r = slice(sub * SOLB, (sub + 1) * SOLB)
            Bt(k, bn)[r] = np.linalg.inv(np.tril(L(k, k))).T[r] @ Yt(k, bn)
        elif kind == TK_FWD_TRSM:
            X = Bt(k, bn); X[:] = sla.solve_triangular(np.tril(L(k, k)), X, lower=True)
        elif kind == TK_BWD_TRSM:
            X = Bt(k, bn); X[:] = sla.solve_triangular(np.tril(L(k, k)), X, lower=True, trans=1)
        elif kind == TK_FWD_UPD:
            src = Yt(k, bn) if xinv else Bt(k, bn)
            rb = SOLB if xinv else SUBB
            Bt(m, bn)[sub * rb:(sub + 1) * rb] -= L(m, k)[sub * rb:(sub + 1) * rb] @ src
        elif kind == TK_BWD_UPD:
            dst = Yt(m, bn) if xinv else Bt(m, bn)
            rb = SOLB if xinv else SUBB
            dst[sub * rb:(sub + 1) * rb] -= L(k, m)[:, sub * rb:(sub + 1) * rb].T @ Bt(k, bn)


SHAPES = [(15, 16, 1, 16), (37, 17, 22, 17), (300, 128, 5, 128), (700, 256, 70, 64), (1000, 384, 3, 384),
          (1100, 512, 64, 512), (513, 512, 1, 512), (2000, 128, 7, 128), (1500, 100, 3, 100)]


@pytest.mark.parametrize("N,NB,nrhs,NBB", SHAPES)
@pytest.mark.parametrize("workers", [1, 7, 148])
@pytest.mark.parametrize("prof", [0, 1, 2])
@pytest.mark.parametrize("G", [1, 3, 4])
def test_schedule_is_deadlock_free(cb_host, N, NB, nrhs, NBB, workers, prof, G):
    for mode in (FACT, SOLVE, FACT | SOLVE):
        t = cb_host.schedule(mode, N, NB, nrhs if mode & SOLVE else 0, NBB, workers, prof, G)
        check_waits(t, mode, N, NB, nrhs if mode & SOLVE else 0, NBB, G)


@pytest.mark.parametrize("N,NB,nrhs,NBB", SHAPES)
@pytest.mark.parametrize("workers", [1, 7, 148])
def test_schedule_casting_arriving_tiles_is_deadlock_free(cb_host, N, NB, nrhs, NBB, workers):
    """MODE_CAST: the FP32 tiles are cast inside the launch as their columns
    arrive; every tile is cast once, before its first reader (the panel solve
    of column 0 or the first update group), whatever the list order."""
    for mode in (FACT | SOLVE | XINV | CAST, FACT | CAST):
        t = cb_host.schedule(mode, N, NB, nrhs if mode & SOLVE else 0, NBB, workers, 2, 8)
        check_waits(t, mode, N, NB, nrhs if mode & SOLVE else 0, NBB, 8)
        assert (t[:, 0] == TK_CAST).sum() == (-(-N // NB)) * (-(-N // NB) + 1) // 2


@pytest.mark.parametrize("N,NB,nrhs,NBB", SHAPES)
@pytest.mark.parametrize("workers", [1, 148])
def test_schedule_with_full_tile_inverses_is_deadlock_free(cb_host, N, NB, nrhs, NBB, workers):
    """FP32 substitutions with full diagonal-tile inverses: TK_XINV after each
    POTRF in a factor+solve launch, instead of TK_INV in a solve launch, and no
    inversion task at all when the inverses are reused (NOINV)."""
    for mode in (FACT | SOLVE | XINV, SOLVE | XINV, SOLVE | XINV | NOINV):
        t = cb_host.schedule(mode, N, NB, nrhs, NBB, workers, 2, 4)
        check_waits(t, mode, N, NB, nrhs, NBB, 4)
        kinds = set(int(x) for x in t[:, 0])
        assert (TK_XINV in kinds) == (not mode & NOINV)
        assert TK_INV not in kinds


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs,NBB", SHAPES[:6] + SHAPES[7:])
@pytest.mark.parametrize("G", [1, 4])
def test_schedule_dataflow_reproduces_cholesky(cb_host, orc, uplo, N, NB, nrhs, NBB, G):
    A0 = orc.dplgsy(float(N), N, 51)
    B0 = orc.dplrnt(N, nrhs, 5673)
    A = A0.copy(); B = B0.copy()
    emulate(cb_host.schedule(FACT | SOLVE, N, NB, nrhs, NBB, 13, 0, G), A, B, uplo, N, NB, NBB)
    F = np.tril(A) if uplo == 122 else np.triu(A)
    assert orc.check_factorization(uplo, A0, F) < 60
    assert orc.check_solve(A0, B, B0) < 60
    Fo, _ = orc.dpotrf_tiled(uplo, A0, NB)
    assert np.allclose(F, np.tril(Fo) if uplo == 122 else np.triu(Fo), atol=1e-12)


@pytest.fixture(scope="module")
def cb_host():
    import chameleon_b200 as cb
    return cb


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs,NBB", SHAPES[:6])
def test_schedule_dataflow_with_full_tile_inverses(cb_host, orc, uplo, N, NB, nrhs, NBB):
    """The split substitutions (row blocks, forward results in Y) produce the
    solution, in a factor+solve launch and in a solve-only launch."""
    A0 = orc.dplgsy(float(N), N, 52)
    B0 = orc.dplrnt(N, nrhs, 5674)
    A = A0.copy(); B = B0.copy()
    emulate(cb_host.schedule(FACT | SOLVE | XINV, N, NB, nrhs, NBB, 13, 2, 4), A, B, uplo, N, NB, NBB, xinv=True)
    assert orc.check_solve(A0, B, B0) < 60
    B2 = B0.copy()
    emulate(cb_host.schedule(SOLVE | XINV | NOINV, N, NB, nrhs, NBB, 13, 2, 4), A, B2, uplo, N, NB, NBB, xinv=True)
    assert np.allclose(B2, B, rtol=1e-12, atol=1e-14)


def replay_two_lists(tasks, mode, N, NB, nrhs, NBB, G=1):
    """The executor's dedicated-CTA scheme: one worker runs the POTRF tasks in
    list order, the others run the remaining tasks in list order.  Replays the
    two sequences greedily (whichever head's wait predicate holds goes next)
    and asserts the run never stalls; returns the interleaved order."""
    pot = [t for t in tasks if t[0] == TK_POTRF]
    rest = [t for t in tasks if t[0] != TK_POTRF]
    order, i, j = [], 0, 0
    while i < len(pot) or j < len(rest):
        progressed = False
        for head_list, idx_name in ((pot, 'i'), (rest, 'j')):
            idx = i if idx_name == 'i' else j
            if idx < len(head_list):
                cand = order + [head_list[idx]]
                try:
                    check_waits_prefix(cand, mode, N, NB, nrhs, NBB, G)
                except AssertionError:
                    continue
                order = cand
                if idx_name == 'i':
                    i += 1
                else:
                    j += 1
                progressed = True
                break
        assert progressed, "stalled at POTRF %d / task %d" % (i, j)
    return order


def check_waits_prefix(prefix, mode, N, NB, nrhs, NBB, G=1):
    """check_waits on a prefix of a run (no completeness checks)."""
    NT, NTB, tm, nbi, S = geometry(N, NB, nrhs, NBB)
    upd = np.zeros((NT, NT), int); pan = np.zeros((NT, NT), int)
    fwdB = np.zeros((NT, max(NTB, 1)), int); fwdD = np.zeros_like(fwdB)
    bwdB = np.zeros_like(fwdB); bwdD = np.zeros_like(fwdB)
    xinv = np.zeros(NT, int)
    fact = bool(mode & FACT)
    srb = SOLB if mode & XINV else SUBB
    nsb = lambda m: -(-tm(m) // srb)
    ns = (lambda k: nsb(k)) if mode & XINV else (lambda k: 1)
    for kind, sub, m, n, k, bn, grp in prefix:
        if kind == TK_CAST:
            continue
        if kind == TK_POTRF:
            ok = upd[k, k] >= ngroups(k, G) * S(k, k); pan[k, k] += 1
        elif kind == TK_INV:
            ok = True; pan[k, k] += 1
        elif kind == TK_XINV:
            ok = (not fact) or pan[k, k] >= 1; xinv[k] += 1
        elif kind == TK_TRSM:
            ok = pan[k, k] >= 1 and upd[m, k] >= ngroups(k, G) * S(m, k); pan[m, k] += 1
        elif kind == TK_UPD:
            kl = k + bn - 1
            ok = pan[m, kl] >= nbi(m) and pan[n, kl] >= nbi(n) and upd[m, n] >= grp * S(m, n); upd[m, n] += 1
        elif kind == TK_FWD_TRSM:
            inv_ok = (bool(mode & NOINV) or xinv[k] >= 1) if mode & XINV else pan[k, k] >= 1
            ok = inv_ok and fwdB[k, bn] >= k * nsb(k); fwdD[k, bn] += 1
        elif kind == TK_FWD_UPD:
            ok = fwdD[k, bn] >= ns(k) and (not fact or pan[m, k] >= nbi(m)) and fwdB[m, bn] >= k * nsb(m)
            fwdB[m, bn] += 1
        elif kind == TK_BWD_TRSM:
            ok = fwdD[k, bn] >= ns(k) and bwdB[k, bn] >= (NT - 1 - k) * nsb(k); bwdD[k, bn] += 1
        else:
            ok = bwdD[k, bn] >= ns(k) and bwdB[m, bn] >= (NT - 1 - k) * nsb(m); bwdB[m, bn] += 1
        assert ok


@pytest.mark.parametrize("N,NB,nrhs,NBB", [(1000, 256, 3, 256), (1100, 512, 64, 512), (300, 128, 5, 128)])
def test_dedicated_potrf_worker_never_stalls(cb_host, N, NB, nrhs, NBB):
    for mode, prof, G in ((FACT, 0, 1), (FACT | SOLVE, 0, 1), (FACT | SOLVE | XINV, 2, 4)):
        t = cb_host.schedule(mode, N, NB, nrhs if mode & SOLVE else 0, NBB, 148, prof, G)
        order = replay_two_lists([tuple(int(v) for v in r) for r in t], mode, N, NB,
                                 nrhs if mode & SOLVE else 0, NBB, G)
        check_waits(np.array(order), mode, N, NB, nrhs if mode & SOLVE else 0, NBB, G)
