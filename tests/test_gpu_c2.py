"""Parity at the large single-solve configuration: N = 16384 (and the bench's
N = 32768), NB = 512, nrhs = 64, dplgsy seed 51 / dplrnt seed 5673.

Both triangles, the mixed solver (BF16x3 factor + FP64 refinement) and the plain
FP64 path.  The checks are the reference's own (testing/testing_zcheck_facto.c):

    check_dxxtrf   ||A - L L^T||_1 / (||A||_1 N eps)          < 60  (:198-300)
    check_dsolve   ||A X - B||_1 / (||A||_1 ||X||_1 N eps)      < 60  (:398-438)

computed in FP64 on the device by torch (cuBLAS), which is the checker here,
never the code under test.  The mixed solution must also agree with the plain
FP64 one: max|X_mixed - X_fp64| / max|X_fp64| < 2 sqrt(N) eps (these matrices
have condition numbers close to 1, and dsposv's rule stops refinement once the
backward error is below sqrt(N) eps), and the
solver's reported backward error ||b - A x||_inf / (||A||_inf ||x||_inf) must be
of the same size as the one computed here (two FP64 residuals at rounding
level, so within a factor 4 of each other) and satisfy dsposv's stopping rule
(<= sqrt(N) eps).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EPS = 1.1102230246251565e-16
NB, NRHS, SEED_A, SEED_B = 512, 64, 51, 5673


def _inputs(cb, N):
    """A (N x N) and B (N x nrhs) in column-major device tensors, made by the
    library's own generators (bit-exact with the reference's dplgsy/dplrnt)."""
    import torch
    A = torch.zeros((N, N), dtype=torch.float64, device="cuda")        # symmetric: row/col major agree
    B = torch.zeros((NRHS, N), dtype=torch.float64, device="cuda")     # B[j, i] = b_ij
    dA = cb.Desc.create(N, N, NB, mat=A)
    dB = cb.Desc.create(N, NRHS, NB, mat=B)
    assert cb.dplgsy_Tile(float(N), cb.ChamUpperLower, dA, SEED_A) == 0
    assert cb.dplrnt_Tile(dB, SEED_B) == 0
    torch.cuda.synchronize()
    dA.destroy()
    dB.destroy()
    return A, B


def _check_solve(A0, X, B0):
    """check_dsolve on column-major N x nrhs tensors stored transposed (nrhs, N)."""
    R = B0.T - A0 @ X.T
    N = A0.shape[0]
    return float(R.abs().sum(0).max() / (A0.abs().sum(0).max() * X.T.abs().sum(0).max() * N * EPS))


def _backward_inf(A0, X, B0):
    R = B0.T - A0 @ X.T
    return float((R.abs().amax(0) / (A0.abs().sum(1).max() * X.T.abs().amax(0))).max())


def _plain(cb, uplo, A0, B0):
    import torch
    N = A0.shape[0]
    A, B = A0.clone(), B0.clone()
    dA = cb.Desc.create(N, N, NB, mat=A)
    dB = cb.Desc.create(N, NRHS, NB, mat=B)
    rc = cb.dposv_Tile(uplo, dA, dB)
    torch.cuda.synchronize()
    dA.destroy()
    dB.destroy()
    return rc, A, B


def _mixed(cb, uplo, A0, B0):
    import torch
    N = A0.shape[0]
    A, B = A0.clone(), B0.clone()
    X = torch.zeros_like(B0)
    dA = cb.Desc.create(N, N, NB, mat=A)
    dB = cb.Desc.create(N, NRHS, NB, mat=B)
    dX = cb.Desc.create(N, NRHS, NB, mat=X)
    rc, info = cb.dposv_mixed_Tile(uplo, cb.PREC_BF16X3, dA, dB, dX)
    torch.cuda.synchronize()
    for d in (dA, dB, dX):
        d.destroy()
    assert bool((A == A0).all()), "A must be left untouched when refinement succeeds"
    return rc, info, X


@pytest.fixture(scope="module")
def c2_inputs(cb):
    import torch
    A0, B0 = _inputs(cb, 16384)
    yield A0, B0
    del A0, B0
    torch.cuda.empty_cache()


@pytest.mark.parametrize("uplo", [121, 122])
def test_c2_plain_fp64_reference_checks(cb, c2_inputs, uplo):
    import torch
    A0, B0 = c2_inputs
    N = A0.shape[0]
    rc, F, X = _plain(cb, uplo, A0, B0)
    assert rc == 0
    Fcm = F.T                      # the tensor is the row-major view of the column-major factor
    L = torch.tril(Fcm) if uplo == 122 else torch.triu(Fcm).T
    R = A0 - L @ L.T
    fact = float(R.abs().sum(0).max() / (A0.abs().sum(0).max() * N * EPS))
    del R, L, F, Fcm
    assert fact < 60, fact
    assert _check_solve(A0, X, B0) < 60


@pytest.mark.parametrize("uplo", [121, 122])
def test_c2_mixed_matches_fp64(cb, c2_inputs, uplo):
    A0, B0 = c2_inputs
    N = A0.shape[0]
    rc, info, X = _mixed(cb, uplo, A0, B0)
    assert rc == 0
    assert 0 <= info.iterations <= 6 and info.fallback == 0
    assert _check_solve(A0, X, B0) < 60
    berr = _backward_inf(A0, X, B0)
    assert berr <= 2 * np.sqrt(N) * EPS      # an independent FP64 residual: rounding level
    assert info.backward_error <= np.sqrt(N) * EPS
    assert berr / 4 <= info.backward_error <= 4 * berr, (info.backward_error, berr)
    rc64, _, X64 = _plain(cb, uplo, A0, B0)
    assert rc64 == 0
    assert float((X - X64).abs().max() / X64.abs().max()) < 2 * np.sqrt(N) * EPS


def test_c2_mixed_at_bench_size(cb):
    """The bench's own configuration (N = 32768, Lower): the solve check, the
    reported backward error and agreement with the plain FP64 solution."""
    import torch
    A0, B0 = _inputs(cb, 32768)
    try:
        rc, info, X = _mixed(cb, 122, A0, B0)
        assert rc == 0
        assert 0 <= info.iterations <= 6 and info.fallback == 0
        assert _check_solve(A0, X, B0) < 60
        berr = _backward_inf(A0, X, B0)
        assert berr <= 2 * np.sqrt(A0.shape[0]) * EPS
        assert info.backward_error <= np.sqrt(A0.shape[0]) * EPS
        assert berr / 4 <= info.backward_error <= 4 * berr, (info.backward_error, berr)
        rc64, _, X64 = _plain(cb, 122, A0, B0)
        assert rc64 == 0
        assert float((X - X64).abs().max() / X64.abs().max()) < 2 * np.sqrt(A0.shape[0]) * EPS
    finally:
        del A0, B0
        torch.cuda.empty_cache()
