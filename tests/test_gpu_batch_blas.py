"""GPU parity of the batched tile GEMM / SYRK (compute/zgemm_batch.c,
zherk_batch.c after z->d) against numpy and the reference's CPU batch run on
the same tiles (testing/testing_zgemm_batch.c / testing_zherk_batch.c build
the same stacked-tile descriptors)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EPS = 1.1102230246251565e-16
NOTRANS, TRANS = 111, 112
UPPER, LOWER = 121, 122


def stacked_desc(cb, T):
    """Desc whose tile i (of one tile column) is T[i] (count x r x c)."""
    cnt, r, c = T.shape
    d = cb.Desc.create(cnt * r, c, r, c)
    d.from_numpy(np.concatenate(list(T), axis=0))
    return d


def unstack(d, cnt, r, c):
    M = d.to_numpy()
    return np.stack([M[i * r:(i + 1) * r] for i in range(cnt)])


def op(X, t):
    return np.swapaxes(X, 1, 2) if t == TRANS else X


@pytest.mark.parametrize("ta", [NOTRANS, TRANS])
@pytest.mark.parametrize("tb", [NOTRANS, TRANS])
def test_gemm_batch_vs_numpy_and_reference(cb, orc, ta, tb):
    rng = np.random.default_rng(ta * 7 + tb)
    cnt, m, n, k = 9, 150, 70, 200          # ragged 128-blocks in every direction
    A = rng.standard_normal((cnt, k, m) if ta == TRANS else (cnt, m, k))
    B = rng.standard_normal((cnt, n, k) if tb == TRANS else (cnt, k, n))
    C = rng.standard_normal((cnt, m, n))
    alpha, beta = 1.5, -0.75
    dA, dB, dC = stacked_desc(cb, A), stacked_desc(cb, B), stacked_desc(cb, C)
    assert cb.lib().CHAMELEON_dgemm_batch_Tile(ta, tb, alpha, dA.ptr, dB.ptr, beta, dC.ptr) == 0
    out = unstack(dC, cnt, m, n)
    ref = alpha * op(A, ta) @ op(B, tb) + beta * C
    tol = 4 * k * EPS * (np.abs(A).max() * np.abs(B).max() * abs(alpha) + abs(beta) * np.abs(C).max())
    assert np.abs(out - ref).max() <= tol
    if orc.reference_available():
        r = orc.ref_dgemm_batch(ta, tb, alpha, A, B, beta, C)
        assert np.abs(out - r).max() <= tol


def test_gemm_batch_beta_zero_does_not_read_c(cb):
    rng = np.random.default_rng(3)
    A, B = rng.standard_normal((4, 64, 33)), rng.standard_normal((4, 33, 129))
    C = np.full((4, 64, 129), np.nan)
    dA, dB, dC = stacked_desc(cb, A), stacked_desc(cb, B), stacked_desc(cb, C)
    assert cb.lib().CHAMELEON_dgemm_batch_Tile(NOTRANS, NOTRANS, 2.0, dA.ptr, dB.ptr, 0.0, dC.ptr) == 0
    out = unstack(dC, 4, 64, 129)
    assert np.isfinite(out).all()
    assert np.abs(out - 2.0 * A @ B).max() <= 4 * 33 * EPS * 2.0 * np.abs(A).max() * np.abs(B).max()


def test_gemm_batch_on_a_tile_grid(cb):
    """A 2 x 3 grid of square tiles: tile (m, n) of C uses tiles (m, n) of A and B."""
    rng = np.random.default_rng(5)
    sq = 88
    A, B, C = (rng.standard_normal((2 * sq, 3 * sq)) for _ in range(3))
    dA, dB, dC = (cb.Desc.create(2 * sq, 3 * sq, sq, sq) for _ in range(3))
    dA.from_numpy(A)
    dB.from_numpy(B)
    dC.from_numpy(C)
    assert cb.lib().CHAMELEON_dgemm_batch_Tile(TRANS, NOTRANS, -1.0, dA.ptr, dB.ptr, 1.0, dC.ptr) == 0
    out = dC.to_numpy()
    for i in range(2):
        for j in range(3):
            sl = np.s_[i * sq:(i + 1) * sq, j * sq:(j + 1) * sq]
            ref = C[sl] - A[sl].T @ B[sl]
            assert np.abs(out[sl] - ref).max() <= 4 * sq * EPS * (np.abs(A).max() * np.abs(B).max() + 1.0) * 4


@pytest.mark.parametrize("uplo", [UPPER, LOWER])
@pytest.mark.parametrize("trans", [NOTRANS, TRANS])
def test_syrk_batch_vs_numpy_and_reference(cb, orc, uplo, trans):
    rng = np.random.default_rng(uplo + trans)
    cnt, n, k = 6, 150, 90
    A = rng.standard_normal((cnt, k, n) if trans == TRANS else (cnt, n, k))
    C = rng.standard_normal((cnt, n, n))
    alpha, beta = 0.5, 2.0
    dA, dC = stacked_desc(cb, A), stacked_desc(cb, C)
    assert cb.lib().CHAMELEON_dsyrk_batch_Tile(uplo, trans, alpha, dA.ptr, beta, dC.ptr) == 0
    out = unstack(dC, cnt, n, n)
    opA = op(A, trans)
    ref = alpha * opA @ np.swapaxes(opA, 1, 2) + beta * C
    tri = (lambda X: np.triu(X)) if uplo == UPPER else (lambda X: np.tril(X))
    oth = (lambda X: np.tril(X, -1)) if uplo == UPPER else (lambda X: np.triu(X, 1))
    tol = 4 * k * EPS * (abs(alpha) * np.abs(A).max() ** 2 + abs(beta) * np.abs(C).max())
    for i in range(cnt):
        assert np.abs(tri(out[i]) - tri(ref[i])).max() <= tol
        assert np.array_equal(oth(out[i]), oth(C[i]))       # the other triangle is not touched
    if orc.reference_available():
        r = orc.ref_dsyrk_batch(uplo, trans, alpha, A, beta, C)
        for i in range(cnt):
            assert np.abs(tri(out[i]) - tri(r[i])).max() <= tol
