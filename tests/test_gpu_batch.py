"""GPU tests of the batch entry points.

Uniform batches (CHAMELEON_dpotrf_batch_Tile / dtrsm_batch_Tile) are compared
with the reference's own batch results (tests/golden/batch_*.npz, produced by
the reference library); the uneven-size batch (no reference equivalent) is
compared per matrix with the oracle and the reference's residual checks.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
EPS = 1.1102230246251565e-16


@pytest.mark.parametrize("uplo", [121, 122])
def test_potrf_trsm_batch_vs_reference_golden(cb, uplo):
    import torch
    g = np.load(os.path.join(GOLDEN, "batch_%d.npz" % uplo))
    n, count, nrhs, trans = int(g["n"]), int(g["count"]), int(g["nrhs"]), int(g["trans"])
    # caller matrices are column-major (count*n) x n / (count*n) x nrhs arrays on the device
    tA = torch.from_numpy(g["A"].T.copy()).cuda()
    tB = torch.from_numpy(g["B"].T.copy()).cuda()
    dA = cb.Desc.create(count * n, n, n, mat=tA)
    dB = cb.Desc.create(count * n, nrhs, n, nb=nrhs, mat=tB)
    assert cb.lib().CHAMELEON_dpotrf_batch_Tile(uplo, dA.ptr) == 0
    torch.cuda.synchronize()
    F = tA.cpu().numpy().T
    tri = np.triu if uplo == 121 else np.tril
    for i in range(count):
        blk = slice(i * n, (i + 1) * n)
        assert np.abs(tri(F[blk]) - tri(g["F"][blk])).max() < 1e-12
    assert cb.lib().CHAMELEON_dtrsm_batch_Tile(141, uplo, trans, 131, ctypes.c_double(1.0), dA.ptr, dB.ptr) == 0
    torch.cuda.synchronize()
    assert np.abs(tB.cpu().numpy().T - g["Y"]).max() < 1e-12


@pytest.mark.parametrize("side", [141, 142])
@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("trans", [111, 112])
def test_trsm_batch_all_variants(cb, side, uplo, trans):
    import torch
    n, w, count = 48, 20, 5
    rng = np.random.default_rng(side + uplo + trans)
    Ts = []
    for i in range(count):
        T = rng.standard_normal((n, n)) * 0.1 + 2 * np.eye(n)
        Ts.append(np.triu(T) if uplo == 121 else np.tril(T))
    A = np.asfortranarray(np.concatenate(Ts))
    bm, bn = (n, w) if side == 141 else (w, n)
    B = np.asfortranarray(rng.standard_normal((count * bm, bn)))
    tA = torch.from_numpy(A.T.copy()).cuda()
    tB = torch.from_numpy(B.T.copy()).cuda()
    dA = cb.Desc.create(count * n, n, n, mat=tA)
    dB = cb.Desc.create(count * bm, bn, bm, nb=bn, mat=tB)
    assert cb.lib().CHAMELEON_dtrsm_batch_Tile(side, uplo, trans, 131, ctypes.c_double(2.0), dA.ptr, dB.ptr) == 0
    torch.cuda.synchronize()
    X = tB.cpu().numpy().T
    for i in range(count):
        op = Ts[i] if trans == 111 else Ts[i].T
        Bi = B[i * bm:(i + 1) * bm]
        ref = np.linalg.solve(op, 2 * Bi) if side == 141 else np.linalg.solve(op.T, 2 * Bi.T).T
        assert np.abs(X[i * bm:(i + 1) * bm] - ref).max() < 1e-11


def _uneven_batch(orc, count, nmin, nmax, rmax, seed):
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, count)
    rs = rng.integers(1, rmax + 1, count)
    As = [orc.dplgsy(float(n), int(n), 1000 + i) for i, n in enumerate(ns)]
    Bs = [orc.dplrnt(int(n), int(r), 2000 + i) for i, (n, r) in enumerate(zip(ns, rs))]
    return ns, rs, As, Bs


@pytest.mark.parametrize("uplo", [121, 122])
def test_uneven_batch_dposv(cb, orc, uplo):
    import torch
    ns, rs, As, Bs = _uneven_batch(orc, 300, 16, 512, 8, 2024)
    a_off = np.cumsum([0] + [n * n for n in ns[:-1]]).astype(np.int64)
    b_off = np.cumsum([0] + [n * r for n, r in zip(ns[:-1], rs[:-1])]).astype(np.int64)
    As[17] = As[17].copy(); As[17][5, 5] = -1.0      # one matrix not SPD

    def poisoned(a):   # only the uplo triangle is referenced: NaN elsewhere
        a = np.array(a, order="F")
        a[np.tril_indices(a.shape[0], -1) if uplo == 121 else np.triu_indices(a.shape[0], 1)] = np.nan
        return a

    A = np.concatenate([poisoned(a).ravel(order="F") for a in As])
    B = np.concatenate([b.ravel(order="F") for b in Bs])
    dev = lambda x, dt=None: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    tA, tB = dev(A), dev(B)
    tn, tr = dev(ns.astype(np.int32)), dev(rs.astype(np.int32))
    ta, tb = dev(a_off), dev(b_off)
    info = torch.zeros(len(ns), dtype=torch.int32, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = cb.lib().CHAM_B200_dposv_batch(uplo, len(ns), p(tn), p(tr), p(tA), p(ta), p(tB), p(tb), p(info), None)
    assert rc == 0
    X = tB.cpu().numpy()
    inf = info.cpu().numpy()
    assert inf[17] == 6 and (np.delete(inf, 17) == 0).all()
    for i, (n, r) in enumerate(zip(ns, rs)):
        if i == 17:
            continue
        Xi = X[b_off[i]:b_off[i] + n * r].reshape((n, r), order="F")
        R = Bs[i] - As[i] @ Xi
        res = np.abs(R).sum(0).max() / (np.abs(As[i]).sum(0).max() * np.abs(Xi).sum(0).max() * n * EPS)
        assert res < 60, (i, n, res)


def _run_batch(cb, fn, uplo, ns, rs, As, Bs, dtype):
    import torch
    a_off = np.cumsum([0] + [n * n for n in ns[:-1]]).astype(np.int64)
    b_off = np.cumsum([0] + [n * r for n, r in zip(ns[:-1], rs[:-1])]).astype(np.int64)
    A = np.concatenate([a.ravel(order="F") for a in As]).astype(dtype)
    B = np.concatenate([b.ravel(order="F") for b in Bs]).astype(dtype)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    tA, tB = dev(A), dev(B)
    tn, tr, ta, tb = dev(ns.astype(np.int32)), dev(rs.astype(np.int32)), dev(a_off), dev(b_off)
    info = torch.full((len(ns),), 7, dtype=torch.int32, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = getattr(cb.lib(), fn)(uplo, len(ns), p(tn), p(tr), p(tA), p(ta), p(tB), p(tb), p(info), None)
    assert rc == 0
    X = tB.cpu().numpy()
    return [X[b_off[i]:b_off[i] + n * r].reshape((n, r), order="F") for i, (n, r) in enumerate(zip(ns, rs))], \
        info.cpu().numpy()


def _residual(A, X, B, eps):
    R = B - A @ X
    return np.abs(R).sum(0).max() / (np.abs(A).sum(0).max() * np.abs(X).sum(0).max() * A.shape[0] * eps)


@pytest.mark.parametrize("uplo", [121, 122])
def test_small_bin_systems(cb, orc, uplo):
    """n <= 64 runs in the small-system kernel (or wherever the autotuner put
    the small bin): every order from 1 to 64, the solve check per system."""
    ns = np.arange(1, 65)
    rs = (ns % 5) + 1
    As = [orc.dplgsy(float(n), int(n), 3000 + int(n)) for n in ns]
    Bs = [orc.dplrnt(int(n), int(r), 4000 + int(n)) for n, r in zip(ns, rs)]
    Xs, inf = _run_batch(cb, "CHAM_B200_dposv_batch", uplo, ns, rs, As, Bs, np.float64)
    assert (inf == 0).all()
    for A, X, B in zip(As, Xs, Bs):
        assert _residual(A, X, B, EPS) < 60


def test_batch_replay_is_identical(cb, orc):
    """The second call with the same batch replays the captured graph: same bits."""
    ns, rs, As, Bs = _uneven_batch(orc, 200, 16, 300, 6, 77)
    X1, i1 = _run_batch(cb, "CHAM_B200_dposv_batch", 122, ns, rs, As, Bs, np.float64)
    X2, i2 = _run_batch(cb, "CHAM_B200_dposv_batch", 122, ns, rs, As, Bs, np.float64)
    assert (i1 == 0).all() and (i2 == 0).all()
    for a, b in zip(X1, X2):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("uplo", [121, 122])
def test_sposv_batch_fp32(cb, orc, uplo):
    """FP32 systems: solve check at FP32 precision (eps = 2^-24)."""
    ns, rs, As, Bs = _uneven_batch(orc, 150, 16, 400, 8, 88)
    Xs, inf = _run_batch(cb, "CHAM_B200_sposv_batch", uplo, ns, rs, As, Bs, np.float32)
    assert (inf == 0).all()
    for A, X, B in zip(As, Xs, Bs):
        assert _residual(A.astype(np.float32).astype(np.float64), X.astype(np.float64),
                         B.astype(np.float32).astype(np.float64), 2.0 ** -24) < 60


def test_batch_autotuner_picked_the_fastest(cb, orc):
    ns, rs, As, Bs = _uneven_batch(orc, 40, 16, 300, 2, 99)
    _run_batch(cb, "CHAM_B200_dposv_batch", 122, ns, rs, As, Bs, np.float64)   # tunes the ranges on first use
    out = (ctypes.c_double * 28)()
    assert cb.lib().CHAM_B200_Batch_Tuning(cb.ChamRealDouble, out) == 0
    tuned = 0
    for r in range(4):
        mode = int(out[r])
        times = [out[4 + 6 * r + k] for k in range(6)]
        if mode < 0:
            continue
        tuned += 1
        admissible = [t for t in times if t >= 0]
        assert len(admissible) >= 2
        assert times[mode] == min(admissible)
        if r > 0:
            assert mode in (0, 4, 5)
    assert tuned >= 3                       # ranges 0..2 at least (n in 16..300)


@pytest.mark.parametrize("r,lo,hi", [(0, 8, 64), (1, 65, 128), (2, 129, 256), (3, 257, 400)])
def test_every_batch_shape_is_correct(cb, orc, r, lo, hi):
    """Each kernel shape the tuner may pick for a size range, forced in turn."""
    ns, rs, As, Bs = _uneven_batch(orc, 50, lo, hi, 9, 500 + r)
    L = cb.lib()
    try:
        ran = 0
        for shape in range(6):
            if L.CHAM_B200_Batch_SetShape(cb.ChamRealDouble, r, shape) != 0:
                continue
            ran += 1
            for uplo in (121, 122):
                Xs, inf = _run_batch(cb, "CHAM_B200_dposv_batch", uplo, ns, rs, As, Bs, np.float64)
                assert (inf == 0).all(), (shape, uplo)
                for A, X, B in zip(As, Xs, Bs):
                    assert _residual(A, X, B, 1.1102230246251565e-16) < 60, (shape, uplo)
        assert ran >= 2
    finally:
        L.CHAM_B200_Batch_SetShape(cb.ChamRealDouble, r, -1)
