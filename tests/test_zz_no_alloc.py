"""CUDA_dpotrf_noalloc: the diagonal-tile Cholesky for callers that cannot allocate.

Some callers cannot let the library call cudaMalloc -- a task runtime that owns
all device memory and forbids allocation inside its callbacks, or code that
must not block on an allocation.  CUDA_dpotrf_noalloc keeps its scratch in a
fixed device array instead (n <= 1024).  This test calls it through the C ABI
twice in a row and checks each result against the existing CUDA_dpotrf, with
the tolerance the other tile-kernel tests use, plus the size limit.  It must
pass alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.asfortranarray(a).T.copy()).cuda()


def _host(t, n):
    return t.cpu().numpy().T.reshape(n, n)


@pytest.mark.parametrize("uplo", [121, 122])
def test_noalloc_potrf_matches_cuda_dpotrf_twice(cb, orc, uplo):
    import torch
    L = cb.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    h = ctypes.c_void_p()
    assert L.CHAM_B200_Handle_Create(ctypes.byref(h), stream) == 0
    try:
        for call, (n, seed) in enumerate([(1000, 31), (512, 32)]):     # two calls in a row
            A = orc.dplgsy(float(n), n, seed)
            d_ref, d_new = _dev(A), _dev(A)
            i_ref = torch.full((1,), -7, dtype=torch.int32, device="cuda")
            i_new = torch.full((1,), -7, dtype=torch.int32, device="cuda")
            assert L.CUDA_dpotrf(uplo, n, ctypes.c_void_p(d_ref.data_ptr()), n, None, 0,
                                 ctypes.c_void_p(i_ref.data_ptr()), h) == 0
            assert L.CUDA_dpotrf_noalloc(uplo, n, ctypes.c_void_p(d_new.data_ptr()), n,
                                         ctypes.c_void_p(i_new.data_ptr()), stream) == 0
            torch.cuda.synchronize()
            assert int(i_ref.item()) == 0 and int(i_new.item()) == 0
            F_ref, F_new = _host(d_ref, n), _host(d_new, n)
            assert np.abs(F_new - F_ref).max() < 1e-12 * n, call
            tri = np.triu if uplo == 121 else np.tril
            U = tri(F_new)
            R = A - (U.T @ U if uplo == 121 else U @ U.T)
            assert np.abs(R).sum(0).max() / (np.abs(A).sum(0).max() * n * 1.11e-16) < 60
    finally:
        L.CHAM_B200_Handle_Destroy(h)


def _potrf_both(L, h, stream, uplo, A, n, lda):
    """Run CUDA_dpotrf and CUDA_dpotrf_noalloc on copies of the n x n matrix A
    stored with leading dimension lda; returns (factor, info) of each."""
    import torch
    Apad = np.zeros((lda, max(n, 1)), order="F")
    Apad[:n, :n] = A
    d_ref, d_new = _dev(Apad), _dev(Apad)
    i_ref = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    i_new = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    assert L.CUDA_dpotrf(uplo, n, ctypes.c_void_p(d_ref.data_ptr()), lda, None, 0,
                         ctypes.c_void_p(i_ref.data_ptr()), h) == 0
    assert L.CUDA_dpotrf_noalloc(uplo, n, ctypes.c_void_p(d_new.data_ptr()), lda,
                                 ctypes.c_void_p(i_new.data_ptr()), stream) == 0
    torch.cuda.synchronize()
    host = lambda t: t.cpu().numpy().T[:n, :n]
    return host(d_ref), int(i_ref.item()), host(d_new), int(i_new.item())


@pytest.mark.parametrize("uplo", [121, 122])
def test_noalloc_potrf_edge_cases_match_cuda_dpotrf(cb, orc, uplo):
    """A leading dimension larger than n, a matrix that is not positive
    definite (negative pivot inside the second 64-column block) and n = 0 give
    the same info and factor as CUDA_dpotrf."""
    import torch
    L = cb.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    h = ctypes.c_void_p()
    assert L.CHAM_B200_Handle_Create(ctypes.byref(h), stream) == 0
    try:
        n = 130
        A = orc.dplgsy(float(n), n, 41)
        F_ref, i_ref, F_new, i_new = _potrf_both(L, h, stream, uplo, A, n, n + 7)
        assert i_ref == 0 and i_new == 0
        assert np.abs(F_new - F_ref).max() < 1e-12 * n
        B = orc.dplgsy(float(n), n, 42)
        B[90, 90] = -3.0 * n
        F_ref, i_ref, F_new, i_new = _potrf_both(L, h, stream, uplo, B, n, n)
        assert i_ref == 91 and i_new == i_ref
        info0 = torch.full((1,), -7, dtype=torch.int32, device="cuda")
        dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
        assert L.CUDA_dpotrf_noalloc(uplo, 0, ctypes.c_void_p(dummy.data_ptr()), 1,
                                     ctypes.c_void_p(info0.data_ptr()), stream) == 0
        torch.cuda.synchronize()
        assert int(info0.item()) == 0
    finally:
        L.CHAM_B200_Handle_Destroy(h)


def test_noalloc_potrf_rejects_sizes_beyond_its_scratch(cb):
    import torch
    n = 1025
    d = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = cb.lib().CUDA_dpotrf_noalloc(122, n, ctypes.c_void_p(d.data_ptr()), n, ctypes.c_void_p(info.data_ptr()),
                                      stream)
    assert rc == -107       # CHAMELEON_ERR_INTERNAL_LIMIT, nothing launched
