"""The reference's CPU dpotri / dtrtri / dlauum (compute/zpotri.c, ztrtri.c,
zlauum.c, built from its sources into the oracle) agree with numpy, so that
the GPU parity tests may use them as the checker."""
import numpy as np
import pytest

EPS = 1.1102230246251565e-16


@pytest.fixture(scope="module")
def ref(orc):
    if not orc.reference_available():
        pytest.skip("reference CPU build absent")
    return orc


@pytest.mark.parametrize("uplo", [121, 122])
def test_reference_potri_trtri_lauum_vs_numpy(ref, uplo):
    N = 300
    tri = np.triu if uplo == 121 else np.tril
    A = ref.dplgsy(float(N), N, 51)
    L = np.linalg.cholesky(A)
    F = L.T if uplo == 121 else L
    Xr, info = ref.ref_dinverse("potri", uplo, F, 64)
    assert info == 0
    inv = np.linalg.inv(A)
    assert np.abs(tri(Xr) - tri(inv)).max() <= 64 * N * EPS * np.abs(inv).max()
    Tr, info = ref.ref_dinverse("trtri", uplo, F, 96)
    assert info == 0
    assert np.abs(tri(Tr) - np.linalg.inv(F)).max() <= 64 * N * EPS * np.abs(np.linalg.inv(F)).max() ** 2
    Pr, info = ref.ref_dinverse("lauum", uplo, F, 80)
    assert info == 0
    P = F.T @ F if uplo == 122 else F @ F.T
    assert np.abs(tri(Pr) - tri(P)).max() <= 4 * N * EPS * np.abs(P).max()


def test_reference_gemm_syrk_batch_vs_numpy(ref):
    rng = np.random.default_rng(1)
    A, B, C = rng.standard_normal((3, 20, 30)), rng.standard_normal((3, 30, 25)), rng.standard_normal((3, 20, 25))
    out = ref.ref_dgemm_batch(111, 111, 1.5, A, B, -0.5, C)
    assert np.abs(out - (1.5 * A @ B - 0.5 * C)).max() < 1e-12
    S = rng.standard_normal((3, 20, 20))
    out = ref.ref_dsyrk_batch(122, 111, 2.0, A, 1.0, S)
    exp = 2.0 * A @ np.swapaxes(A, 1, 2) + S
    for i in range(3):
        assert np.abs(np.tril(out[i]) - np.tril(exp[i])).max() < 1e-12
        assert np.array_equal(np.triu(out[i], 1), np.triu(S[i], 1))


@pytest.mark.parametrize("uplo", [121, 122])
def test_reference_potrimm_vs_numpy(ref, uplo):
    rng = np.random.default_rng(uplo)
    N = 150
    M = rng.standard_normal((N, N))
    A = M @ M.T / N + np.eye(N)
    B = rng.standard_normal((N, N))
    Aw, C, info = ref.ref_dpotrimm(uplo, A, B, 48)
    assert info == 0
    inv = np.linalg.inv(A)
    tri = np.triu if uplo == 121 else np.tril
    assert np.abs(tri(Aw) - tri(inv)).max() < 1e-12
    assert np.abs(C - B @ inv).max() < 1e-12
