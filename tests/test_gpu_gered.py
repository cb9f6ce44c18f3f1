"""GPU gered / gerst (compute/pzgered.c:160-260, pzgerst.c) against the
oracle's restatement of the same rule: identical precision decisions per tile
and bitwise identical rounded values (round to nearest even in both)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HALF, SINGLE, DOUBLE = 5, 6, 7   # ChamRealHalf / ChamRealFloat / ChamRealDouble


def graded(N, mb, seed):
    """SPD matrix whose off-diagonal tiles shrink geometrically away from the
    diagonal, so that some tiles fall under each threshold."""
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((N, N))
    A = (M + M.T) / 2
    mt = (N + mb - 1) // mb
    for m in range(mt):
        for n in range(mt):
            A[m * mb:(m + 1) * mb, n * mb:(n + 1) * mb] *= 10.0 ** (-4.0 * abs(m - n))
    A += N * np.eye(N)
    return A


@pytest.mark.parametrize("uplo", [121, 122, 123])
@pytest.mark.parametrize("prec", [-1.0, 1e-10, 1e-6])
def test_gered_matches_oracle(cb, orc, uplo, prec):
    N, mb = 700, 128
    A = graded(N, mb, 4)
    d = cb.Desc.create(N, N, mb)
    d.from_numpy(A)
    assert cb.lib().CHAMELEON_dgered_Tile(uplo, prec, d.ptr) == 0
    out = d.to_numpy()
    ref, tags = orc.gered(uplo, prec, A, mb)
    mt = tags.shape[0]
    code = {0: DOUBLE, 1: SINGLE, 2: HALF}
    for m in range(mt):
        for n in range(mt):
            got = cb.lib().CHAM_B200_Tile_Precision(d.ptr, m, n)
            assert got == code[int(tags[m, n])], (m, n)
    assert np.array_equal(out, ref, equal_nan=True)
    assert (tags > 0).any() and (tags == 0).any()          # both kinds of tiles occur
    # gerst: the tags go back to FP64, the values stay rounded
    assert cb.lib().CHAMELEON_dgerst_Tile(uplo, d.ptr) == 0
    assert all(cb.lib().CHAM_B200_Tile_Precision(d.ptr, m, n) == DOUBLE for m in range(mt) for n in range(mt))
    assert np.array_equal(d.to_numpy(), ref, equal_nan=True)


def test_gered_then_posv_still_solves(cb, orc):
    """The reduced matrix is a small perturbation (a few eps ||A||: FP16's
    unit roundoff is ~5 times the rule's 1e-4): the FP64 solve of the gered
    matrix stays within the requested accuracy of A's."""
    N, mb, nrhs = 640, 128, 3
    A = graded(N, mb, 9)
    B = np.random.default_rng(2).standard_normal((N, nrhs))
    d = cb.Desc.create(N, N, mb)
    d.from_numpy(A)
    assert cb.lib().CHAMELEON_dgered_Tile(122, 1e-8, d.ptr) == 0
    Ar = d.to_numpy()
    Ar = np.tril(Ar) + np.tril(Ar, -1).T
    assert np.linalg.norm(np.tril(Ar - A)) <= 1e-7 * np.linalg.norm(np.tril(A))
    dB = cb.Desc.create(N, nrhs, mb)
    dB.from_numpy(B)
    assert cb.dposv_Tile(122, d, dB) == 0
    X = dB.to_numpy()
    assert np.abs(A @ X - B).max() <= 1e-6 * np.abs(B).max()
