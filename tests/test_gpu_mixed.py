"""GPU tests of the mixed-precision solver (FP32 / BF16x3 factor + FP64 refinement).

The reference has no mixed solver to compare with (zcposv is commented out of
its build), so parity is pinned on the FP64 answer: the refined solution must
pass the reference's solve check (threshold 60, testing/testing_zcheck_facto.c
:430-438) and match the FP64 oracle solution to near machine precision (forward
error), with LAPACK dsposv's ITER conventions for fallbacks.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EPS = 1.1102230246251565e-16


def np_check_solve(A0, X, B):
    R = B - A0 @ X
    return np.abs(R).sum(0).max() / (np.abs(A0).sum(0).max() * np.abs(X).sum(0).max() * A0.shape[0] * EPS)


def spd_with_condition(N, cond, seed):
    """Q diag(s) Q^T with s geometric from 1 down to 1/cond (seeded Gaussian QR)."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((N, N)))
    s = np.geomspace(1.0, 1.0 / cond, N)
    A = (Q * s) @ Q.T
    return np.asfortranarray((A + A.T) / 2)


def solve_mixed(cb, uplo, prec, A0, B0, NB):
    N, nrhs = B0.shape
    dA = cb.Desc.create(N, N, NB)
    dB = cb.Desc.create(N, nrhs, NB)
    dX = cb.Desc.create(N, nrhs, NB)
    dA.from_numpy(A0)
    dB.from_numpy(B0)
    rc, info = cb.dposv_mixed_Tile(uplo, prec, dA, dB, dX)
    return rc, info, dX.to_numpy(), dA.to_numpy()


@pytest.mark.parametrize("prec", [2, 1])          # BF16x3, FP32 (TF32x3)
@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs", [(1000, 256, 5), (2048, 320, 1), (3000, 512, 64), (37, 17, 3)])
def test_mixed_refines_to_fp64_accuracy(cb, orc, prec, uplo, N, NB, nrhs):
    A0 = orc.dplgsy(float(N), N, 51)
    B0 = orc.dplrnt(N, nrhs, 5673)
    rc, info, X, Aout = solve_mixed(cb, uplo, prec, A0, B0, NB)
    assert rc == 0
    assert 0 <= info.iterations <= 6 and info.fallback == 0
    assert np_check_solve(A0, X, B0) < 60
    Xr = np.linalg.solve(A0, B0)
    assert np.abs(X - Xr).max() / np.abs(Xr).max() < 1e-14
    assert np.array_equal(Aout, A0)          # A untouched when refinement succeeds


@pytest.mark.parametrize("cond", [1e3, 1e6])
def test_mixed_ill_conditioned_converges_or_falls_back(cb, cond):
    N, NB, nrhs = 512, 128, 4
    A0 = spd_with_condition(N, cond, 7)
    rng = np.random.default_rng(3)
    xt = rng.standard_normal((N, nrhs))
    B0 = np.asfortranarray(A0 @ xt)
    for prec in (2, 1):
        rc, info, X, _ = solve_mixed(cb, 122, prec, A0, B0, NB)
        assert rc == 0
        assert np_check_solve(A0, X, B0) < 60
        assert np.abs(X - xt).max() / np.abs(xt).max() < cond * 1e-13


def test_mixed_fallback_when_refinement_stalls(cb):
    N, NB = 400, 128
    A0 = spd_with_condition(N, 1e12, 11)
    B0 = np.asfortranarray(A0 @ np.ones((N, 2)))
    cb.set_param(cb.CHAMELEON_B200_REFINE_MAXITER, 30)
    rc, info, X, Aout = solve_mixed(cb, 122, 2, A0, B0, NB)
    assert rc == 0
    assert info.iterations < 0 and info.fallback == 1       # LAPACK dsposv: ITER < 0 on fallback
    assert np_check_solve(A0, X, B0) < 60
    L = np.tril(Aout)                                        # A holds the FP64 factor, as in dsposv
    assert np.abs(L @ L.T - A0).max() < 1e-12 * np.abs(A0).max() * N


def test_mixed_overflow_in_cast_falls_back(cb):
    N, NB = 300, 128
    A0 = np.asfortranarray(np.eye(N) * 1e39)
    B0 = np.asfortranarray(np.ones((N, 1)) * 1e39)
    rc, info, X, _ = solve_mixed(cb, 122, 2, A0, B0, NB)
    assert rc == 0 and info.iterations == -2
    assert np.allclose(X, 1.0)


@pytest.mark.parametrize("uplo", [121, 122])
def test_mixed_huge_values_outside_the_triangle_are_not_read(cb, orc, uplo):
    """Only the uplo triangle is referenced: values that do not fit FP32 in the
    other one neither trigger the overflow fallback nor change the norm."""
    N, NB = 700, 256
    A0 = orc.dplgsy(float(N), N, 61)
    B0 = orc.dplrnt(N, 3, 62)
    Ain = np.array(A0, order="F")
    other = np.triu_indices(N, 1) if uplo == 122 else np.tril_indices(N, -1)
    Ain[other] = 1e39
    rc, info, X, _ = solve_mixed(cb, uplo, 2, Ain, B0, NB)
    assert rc == 0
    assert 0 <= info.iterations <= 6 and info.fallback == 0
    assert np_check_solve(A0, X, B0) < 60


def test_mixed_not_spd_reports_info(cb, orc):
    N, NB = 300, 128
    A0 = orc.dplgsy(float(N), N, 2)
    A0[150, 150] = -5.0
    B0 = orc.dplrnt(N, 1, 3)
    rc, info, X, _ = solve_mixed(cb, 122, 2, A0, B0, NB)
    assert rc == 151


@pytest.mark.parametrize("uplo", [121, 122])
def test_dsposv_lapack_layout_host(cb, orc, uplo):
    N, nrhs, LDA = 777, 6, 800
    A0 = orc.dplgsy(float(N), N, 8)
    B0 = orc.dplrnt(N, nrhs, 9)
    A = np.zeros((LDA, N), order="F"); A[:N] = A0
    B = np.zeros((LDA, nrhs), order="F"); B[:N] = B0
    X = np.zeros((LDA, nrhs), order="F")
    rc, it = cb.dsposv(uplo, N, nrhs, A, LDA, B, LDA, X, LDA)
    assert rc == 0 and it >= 0
    assert np_check_solve(A0, X[:N], B0) < 60
    assert np.array_equal(A[:N], A0)


def test_dsposv_tile_api(cb, orc):
    N, NB, nrhs = 1500, 384, 3
    dA = cb.Desc.create(N, N, NB)
    dB = cb.Desc.create(N, nrhs, NB)
    dX = cb.Desc.create(N, nrhs, NB)
    cb.dplgsy_Tile(float(N), 122, dA, 51)
    cb.dplrnt_Tile(dB, 5673)
    rc, it = cb.dsposv_Tile(122, dA, dB, dX)
    assert rc == 0 and it >= 0
    A0 = orc.dplgsy(float(N), N, 51)
    assert np_check_solve(A0, dX.to_numpy(), dB.to_numpy()) < 60


def poison_other_triangle(A, uplo):
    """LAPACK convention: only the `uplo` triangle is referenced.  NaN in the
    other strict triangle must not reach any result."""
    P = np.asfortranarray(A.copy())
    if uplo == 121:
        P[np.tril_indices(A.shape[0], -1)] = np.nan
    else:
        P[np.triu_indices(A.shape[0], 1)] = np.nan
    return P


@pytest.mark.parametrize("prec", [2, 1])
@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs", [(513, 256, 4), (1000, 384, 3), (130, 64, 2)])
def test_mixed_reads_only_uplo_triangle(cb, orc, prec, uplo, N, NB, nrhs):
    A0 = orc.dplgsy(float(N), N, 61)
    B0 = orc.dplrnt(N, nrhs, 62)
    rc, info, X, Aout = solve_mixed(cb, uplo, prec, poison_other_triangle(A0, uplo), B0, NB)
    assert rc == 0 and info.iterations >= 0 and info.fallback == 0
    assert np.isfinite(X).all()
    assert np_check_solve(A0, X, B0) < 60


@pytest.mark.parametrize("uplo", [121, 122])
def test_dsposv_lapack_reads_only_uplo_triangle(cb, orc, uplo):
    N, nrhs = 700, 5
    A0 = orc.dplgsy(float(N), N, 63)
    B0 = orc.dplrnt(N, nrhs, 64)
    A = poison_other_triangle(A0, uplo)
    X = np.zeros((N, nrhs), order="F")
    rc, it = cb.dsposv(uplo, N, nrhs, A, N, np.asfortranarray(B0.copy()), N, X, N)
    assert rc == 0 and it >= 0
    assert np_check_solve(A0, X, B0) < 60


@pytest.mark.parametrize("rec", [1, 0])
@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs", [(1000, 512, 3), (777, 384, 5), (2048, 320, 2), (37, 17, 1), (1500, 1000, 2),
                                       (130, 64, 3), (600, 1100, 1)])
def test_recursive_tile_path_matches_blocked(cb, orc, rec, uplo, N, NB, nrhs):
    """FP32 factorization with recursive diagonal tiles + full tile inverses
    (CHAMELEON_B200_REC_TILE=1, tiles up to 1024) and the blocked one (=0,
    default) both refine to FP64 accuracy in a few iterations on dplgsy
    matrices."""
    A0 = orc.dplgsy(float(N), N, 81)
    B0 = orc.dplrnt(N, nrhs, 82)
    old = cb.get_param(cb.CHAMELEON_B200_REC_TILE)
    assert cb.lib().CHAMELEON_Set(cb.CHAMELEON_B200_REC_TILE, rec) == 0
    try:
        for prec in (2, 1):
            rc, info, X, _ = solve_mixed(cb, uplo, prec, A0, B0, NB)
            assert rc == 0 and info.fallback == 0 and 0 <= info.iterations <= 5, (prec, info.iterations)
            assert np_check_solve(A0, X, B0) < 60
    finally:
        cb.lib().CHAMELEON_Set(cb.CHAMELEON_B200_REC_TILE, old)


def test_recursive_tile_not_spd_reports_info(cb):
    """A non-positive pivot inside the recursion (second leaf of the second
    half) is reported with the same LAPACK order as the blocked path."""
    N, NB = 512, 512
    A0 = np.eye(N) * 4.0
    A0[300, 300] = -1.0
    B0 = np.ones((N, 1))
    import ctypes
    old = cb.get_param(cb.CHAMELEON_B200_REC_TILE)
    for rec in (1, 0):
        assert cb.lib().CHAMELEON_Set(cb.CHAMELEON_B200_REC_TILE, rec) == 0
        rc, info, X, _ = solve_mixed(cb, 122, 2, np.asfortranarray(A0), np.asfortranarray(B0), NB)
        assert rc == 301, (rec, rc)
        # the FP32 factorization alone reports the same order
        dA = cb.Desc.create(N, N, NB)
        dB = cb.Desc.create(N, 1, NB)
        dA.from_numpy(np.asfortranarray(A0))
        dB.from_numpy(np.asfortranarray(B0))
        ms = ctypes.c_float()
        assert cb.lib().CHAM_B200_Mixed_Factor_Only(122, 2, dA.ptr, dB.ptr, ctypes.byref(ms)) == 301
    cb.lib().CHAMELEON_Set(cb.CHAMELEON_B200_REC_TILE, old)


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs", [(3000, 512, 7), (2100, 256, 3), (1025, 512, 64)])
def test_dsposv_host_matrix_streams_while_factoring(cb, orc, uplo, N, NB, nrhs):
    """A host matrix is copied to the device one tile column at a time while
    the factorization casts the columns that have landed (only the referenced
    triangle moves).  The result equals the one from the same matrix already
    on the device (same FP32 factor; the norm is summed in another order, so
    agreement to the refinement's stopping accuracy), and NaN in the other
    triangle of the host matrix is never read."""
    import torch
    A0 = orc.dplgsy(float(N), N, 91)
    B0 = orc.dplrnt(N, nrhs, 92)
    cb.set_param(cb.CHAMELEON_TILE_SIZE, NB)
    try:
        A = poison_other_triangle(A0, uplo)
        Ah = torch.from_numpy(A.T.copy()).pin_memory()          # column-major N x N in pinned memory
        Bh = torch.from_numpy(np.asfortranarray(B0).T.copy()).pin_memory()
        Xh = torch.zeros_like(Bh).pin_memory()
        rc, it = cb.dsposv(uplo, N, nrhs, Ah, N, Bh, N, Xh, N)
        assert rc == 0 and it >= 0
        X = Xh.numpy().T
        assert np_check_solve(A0, X, B0) < 60
        Ad = torch.from_numpy(np.asfortranarray(A0).T.copy()).cuda()
        Bd = torch.from_numpy(np.asfortranarray(B0).T.copy()).cuda()
        Xd = torch.zeros_like(Bd)
        rc2, it2 = cb.dsposv(uplo, N, nrhs, Ad, N, Bd, N, Xd, N)
        assert rc2 == 0 and it2 >= 0
        Xdev = Xd.cpu().numpy().T
        assert np.abs(X - Xdev).max() / np.abs(Xdev).max() < 2 * np.sqrt(N) * EPS
        assert np.array_equal(Ah.numpy(), A.T, equal_nan=True)   # the host matrix is not written
    finally:
        cb.set_param(cb.CHAMELEON_TILE_SIZE, 384)
