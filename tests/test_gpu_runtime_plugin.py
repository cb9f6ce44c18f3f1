"""The reference's own CHAMELEON_dposv_Tile on the B200 runtime plugin (GPU).

compute/zposv.c (one chameleon_pdpotrf, two chameleon_pdtrsm) linked with
chameleon_b200/runtime/runtime_b200.c: its INSERT_TASK_* calls record one DAG
that RUNTIME_sequence_wait runs in one persistent executor launch on the
descriptors' tiles (CUDA managed memory).  The factor and the solution pass the
reference's checks (testing/testing_zcheck_facto.c, threshold 60) and agree
with this library's own dposv_Tile; a matrix that is not positive definite
reports LAPACK's info through the sequence status.
"""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN = os.path.join(ROOT, "oracle", "_ref", "libchamb200rt.so")
EPS = 1.1102230246251565e-16


def plugin_posv(uplo, A0, B0, NB):
    N, nrhs = B0.shape
    L = ctypes.CDLL(PLUGIN)
    A = np.asfortranarray(A0.copy())
    B = np.asfortranarray(B0.copy())
    n = ctypes.c_int()
    rc = L.harness_posv(uplo, N, NB, nrhs, A.ctypes.data_as(ctypes.c_void_p), N, B.ctypes.data_as(ctypes.c_void_p),
                        N, 0, None, 0, ctypes.byref(n))
    return rc, A, B


@pytest.mark.skipif(not os.path.exists(PLUGIN), reason="plugin test library not built")
@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs", [(2048, 320, 1), (3000, 512, 64), (700, 128, 9)])
def test_reference_dposv_runs_on_the_b200_runtime(cb, orc, uplo, N, NB, nrhs):
    A0 = orc.dplgsy(float(N), N, 51)
    B0 = orc.dplrnt(N, nrhs, 5673)
    rc, F, X = plugin_posv(uplo, A0, B0, NB)
    assert rc == 0
    Lf = np.tril(F) if uplo == 122 else np.triu(F).T
    assert np.abs(A0 - Lf @ Lf.T).sum(0).max() / (np.abs(A0).sum(0).max() * N * EPS) < 60
    R = B0 - A0 @ X
    assert np.abs(R).sum(0).max() / (np.abs(A0).sum(0).max() * np.abs(X).sum(0).max() * N * EPS) < 60
    # the same answer as this library's own dposv_Tile (same tile kernels)
    dA = cb.Desc.create(N, N, NB)
    dB = cb.Desc.create(N, nrhs, NB)
    dA.from_numpy(A0)
    dB.from_numpy(B0)
    assert cb.dposv_Tile(uplo, dA, dB) == 0
    assert np.abs(dB.to_numpy() - X).max() <= 1e-13 * np.abs(X).max()


@pytest.mark.skipif(not os.path.exists(PLUGIN), reason="plugin test library not built")
def test_reference_dposv_on_b200_runtime_reports_info(orc):
    N, NB = 600, 128
    A0 = orc.dplgsy(float(N), N, 3)
    A0[400, 400] = -1.0
    rc, _, _ = plugin_posv(122, A0, orc.dplrnt(N, 1, 4), NB)
    assert rc == 401
