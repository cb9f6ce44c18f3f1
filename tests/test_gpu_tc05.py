"""tcgen05 split-BF16 GEMM (the FP32 factorization's trailing update) on the GPU.

C = A B^T for 128 x K FP32 operands through the same path the factorization
uses (swizzled split chunks, bulk copies, tcgen05.mma into tensor memory,
tcgen05.ld).  Tolerance: BF16x3 keeps ~16 mantissa bits per operand, so the
error of a K-term dot product of O(1) values is a few 1e-5 * sqrt(K); a plain
BF16 product would be ~1e-2 -- the test requires the former.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("K", [64, 512, 1024])
def test_tc05_gemm_matches_fp64(cb, K):
    import torch
    rng = np.random.default_rng(K)
    A = rng.standard_normal((128, K)).astype(np.float32)
    B = rng.standard_normal((128, K)).astype(np.float32)
    tA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()   # column-major 128 x K
    tB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    tC = torch.zeros((128, 128), dtype=torch.float32, device="cuda")
    rc = cb.lib().CHAM_B200_Test_TC05(ctypes.c_void_p(tA.data_ptr()), ctypes.c_void_p(tB.data_ptr()), K,
                                      ctypes.c_void_p(tC.data_ptr()))
    assert rc == 0
    torch.cuda.synchronize()
    C = tC.cpu().numpy().T                                      # column-major result
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    err = np.abs(C - ref).max()
    assert err < 2e-4 * np.sqrt(K), err
    # a plain BF16 product is far less accurate: the split is really applied
    bf = lambda x: torch.from_numpy(x).bfloat16().float().numpy().astype(np.float64)
    assert err < 0.05 * np.abs(bf(A) @ bf(B).T - ref).max()


@pytest.mark.parametrize("uplo", [121, 122])
def test_mixed_solve_tcgen05_on_off(cb, orc, uplo):
    N, NB, nrhs = 2560, 512, 8
    A0 = orc.dplgsy(float(N), N, 77)
    B0 = orc.dplrnt(N, nrhs, 78)
    Xs = []
    for tc in (1, 0):
        cb.set_param(cb.CHAMELEON_B200_TCGEN05, tc)
        dA = cb.Desc.create(N, N, NB); dB = cb.Desc.create(N, nrhs, NB); dX = cb.Desc.create(N, nrhs, NB)
        dA.from_numpy(A0); dB.from_numpy(B0)
        rc, info = cb.dposv_mixed_Tile(uplo, cb.PREC_BF16X3, dA, dB, dX)
        assert rc == 0 and 0 <= info.iterations <= 6 and info.fallback == 0
        Xs.append(dX.to_numpy())
    cb.set_param(cb.CHAMELEON_B200_TCGEN05, 1)
    Xr = np.linalg.solve(A0, B0)
    for X in Xs:
        assert np.abs(X - Xr).max() / np.abs(Xr).max() < 1e-14
