"""GPU parity of the FP64 Cholesky path against the oracle, through the C ABI.

Cases follow the reference's own sweeps (testing/input/posv.in, potrf.in,
potrs.in: odd tile sizes 16/17, ragged edges, nrhs 1..33, both uplo) plus the
dposv configuration N=2048, NB=320.  Acceptance is the reference's testing
check (threshold 60, testing/testing_zcheck_facto.c:277-281, 430-438) and
element-wise agreement with the reference's factor / solution from the golden
fixtures.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

EPS = 1.1102230246251565e-16


def np_check_factorization(uplo, A0, F):
    L = np.tril(F) if uplo == 122 else np.triu(F).T
    R = A0 - L @ L.T
    return np.abs(R).sum(0).max() / (np.abs(A0).sum(0).max() * A0.shape[0] * EPS)


def np_check_solve(A0, X, B):
    R = B - A0 @ X
    return np.abs(R).sum(0).max() / (np.abs(A0).sum(0).max() * np.abs(X).sum(0).max() * A0.shape[0] * EPS)


def run_tile_posv(cb, uplo, A, B, NB):
    N, nrhs = B.shape
    dA = cb.Desc.create(N, N, NB)
    dB = cb.Desc.create(N, nrhs, NB)
    dA.from_numpy(A)
    dB.from_numpy(B)
    rc = cb.dposv_Tile(uplo, dA, dB)
    F = dA.to_numpy(uplo)
    X = dB.to_numpy()
    return rc, F, X


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "posv_*.npz"))))
def test_posv_tile_vs_reference_golden(cb, path):
    g = np.load(path)
    uplo, N, NB, nrhs = (int(x) for x in os.path.basename(path)[5:-4].split("_"))
    rc, F, X = run_tile_posv(cb, uplo, g["A"], g["B"], NB)
    assert rc == 0
    tri = np.triu if uplo == 121 else np.tril
    assert np.abs(tri(F) - g["F"]).max() <= 64 * N * EPS * np.abs(g["A"]).max()
    assert np.abs(X - g["X"]).max() <= 64 * N * EPS * max(1.0, np.abs(g["X"]).max())
    assert np_check_factorization(uplo, g["A"], F) < 60
    assert np_check_solve(g["A"], X, g["B"]) < 60


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs", [(2048, 320, 1), (1000, 256, 40), (777, 512, 3), (1500, 384, 130),
                                       (4096, 512, 64)])
def test_posv_tile_seeded_checks(cb, orc, uplo, N, NB, nrhs):
    """The testing driver's descriptor path: dplgsy/dplrnt on the device, then dposv_Tile."""
    dA = cb.Desc.create(N, N, NB)
    dB = cb.Desc.create(N, nrhs, NB)
    assert cb.dplgsy_Tile(float(N), 123, dA, 51) == 0
    assert cb.dplrnt_Tile(dB, 5673) == 0
    A0 = dA.to_numpy()
    B0 = dB.to_numpy()
    assert np.array_equal(A0, orc.dplgsy(float(N), N, 51))   # generator bit-exact on the GPU
    assert np.array_equal(B0, orc.dplrnt(N, nrhs, 5673))
    assert cb.dposv_Tile(uplo, dA, dB) == 0
    F = dA.to_numpy(uplo)
    X = dB.to_numpy()
    assert np_check_factorization(uplo, A0, F) < 60
    assert np_check_solve(A0, X, B0) < 60
    Xr = np.linalg.solve(A0, B0)
    assert np.abs(X - Xr).max() < 1e-12


@pytest.mark.parametrize("uplo", [121, 122])
def test_generator_uplo_skips_tiles_like_reference(cb, orc, uplo):
    N, NB = 100, 32
    dA = cb.Desc.create(N, N, NB)
    assert cb.dplgsy_Tile(float(N), uplo, dA, 7) == 0
    A = dA.to_numpy()
    full = orc.dplgsy(float(N), N, 7)
    for m in range(4):
        for n in range(4):
            blk = (slice(m * NB, min((m + 1) * NB, N)), slice(n * NB, min((n + 1) * NB, N)))
            skipped = (uplo == 122 and n > m) or (uplo == 121 and m > n)
            if skipped:
                assert not A[blk].any()
            else:
                assert np.array_equal(A[blk], full[blk])


@pytest.mark.parametrize("uplo", [121, 122])
def test_potrf_then_potrs(cb, orc, uplo):
    N, NB, nrhs = 700, 128, 9
    A0 = orc.dplgsy(float(N), N, 11)
    B0 = orc.dplrnt(N, nrhs, 12)
    dA = cb.Desc.create(N, N, NB)
    dB = cb.Desc.create(N, nrhs, NB)
    dA.from_numpy(A0)
    dB.from_numpy(B0)
    assert cb.dpotrf_Tile(uplo, dA) == 0
    F = dA.to_numpy(uplo)
    assert np_check_factorization(uplo, A0, F) < 60
    Fo, _ = orc.dpotrf_tiled(uplo, A0, NB)
    tri = np.triu if uplo == 121 else np.tril
    assert np.abs(tri(F) - tri(Fo)).max() < 1e-12 * N
    assert cb.dpotrs_Tile(uplo, dA, dB) == 0
    assert np_check_solve(A0, dB.to_numpy(), B0) < 60


@pytest.mark.parametrize("uplo", [121, 122])
def test_lapack_layout_host_and_device(cb, orc, uplo):
    import torch
    N, nrhs, LDA, LDB = 613, 17, 640, 650
    A0 = orc.dplgsy(float(N), N, 3)
    B0 = orc.dplrnt(N, nrhs, 4)
    A = np.zeros((LDA, N), order="F"); A[:N] = A0
    B = np.zeros((LDB, nrhs), order="F"); B[:N] = B0
    cb.set_param(cb.CHAMELEON_TILE_SIZE, 192)
    assert cb.dposv(uplo, N, nrhs, A, LDA, B, LDB) == 0
    assert np_check_solve(A0, B[:N], B0) < 60
    assert np_check_factorization(uplo, A0, A[:N]) < 60
    assert not A[N:].any()          # padding rows untouched
    # the same on device arrays (torch CUDA tensors in column-major storage)
    tA = torch.zeros((N, LDA), dtype=torch.float64, device="cuda"); tA[:, :N] = torch.from_numpy(A0.T.copy())
    tB = torch.zeros((nrhs, LDB), dtype=torch.float64, device="cuda"); tB[:, :N] = torch.from_numpy(B0.T.copy())
    assert cb.dposv(uplo, N, nrhs, tA, LDA, tB, LDB) == 0
    torch.cuda.synchronize()
    X = tB.cpu().numpy().T[:N]
    assert np_check_solve(A0, X, B0) < 60
    cb.set_param(cb.CHAMELEON_TILE_SIZE, 384)


@pytest.mark.parametrize("uplo", [121, 122])
def test_non_spd_reports_info(cb, orc, uplo):
    N, NB = 600, 128
    A0 = orc.dplgsy(float(N), N, 5)
    A0[300, 300] = -1.0            # leading minor 301 is not positive definite
    dA = cb.Desc.create(N, N, NB)
    dA.from_numpy(A0)
    info = cb.dpotrf_Tile(uplo, dA)
    _, info_o = orc.dpotrf_tiled(uplo, A0, NB)
    assert info == info_o == 301


def test_device_wait_budget_returns_error_and_context_survives(cb, orc):
    """A dependency wait that runs out of budget ends the launch with an error code, not a fault."""
    N, NB = 6144, 512
    dA = cb.Desc.create(N, N, NB)
    assert cb.dplgsy_Tile(float(N), 122, dA, 1) == 0
    old = cb.get_param(cb.CHAMELEON_B200_WAIT_BUDGET_US)
    cb.set_param(cb.CHAMELEON_B200_WAIT_BUDGET_US, 2)   # 2 us: the panel waits on POTRF(0) far longer
    try:
        rc = cb.dpotrf_Tile(122, dA)
    finally:
        cb.set_param(cb.CHAMELEON_B200_WAIT_BUDGET_US, old)
    assert rc == cb.CHAMELEON_ERR_DEVICE_TIMEOUT
    # the context is still usable
    N2, NB2 = 500, 128
    A0 = orc.dplgsy(float(N2), N2, 9)
    B0 = orc.dplrnt(N2, 2, 10)
    rc, F, X = run_tile_posv(cb, 122, A0, B0, NB2)
    assert rc == 0 and np_check_solve(A0, X, B0) < 60


# ---- gpucublas tile ABI -------------------------------------------------------

@pytest.fixture(scope="module")
def handle(cb):
    import torch
    h = ctypes.c_void_p()
    s = torch.cuda.current_stream().cuda_stream
    assert cb.lib().CHAM_B200_Handle_Create(ctypes.byref(h), ctypes.c_void_p(s)) == 0
    yield h
    cb.lib().CHAM_B200_Handle_Destroy(h)


def _dev(a):
    import torch
    return torch.from_numpy(np.asfortranarray(a).T.copy()).cuda()   # storage is column-major a


def _host(t, shape):
    return t.cpu().numpy().T.reshape(shape)


@pytest.mark.parametrize("ta,tb", [(111, 111), (111, 112), (112, 111), (112, 112)])
@pytest.mark.parametrize("m,n,k", [(128, 128, 512), (37, 45, 17), (300, 129, 257)])
def test_cuda_dgemm(cb, handle, ta, tb, m, n, k):
    import torch
    rng = np.random.default_rng(m * n + k)
    A = rng.standard_normal((m, k) if ta == 111 else (k, m))
    B = rng.standard_normal((k, n) if tb == 111 else (n, k))
    C = rng.standard_normal((m, n))
    al, be = ctypes.c_double(-1.5), ctypes.c_double(0.75)
    dA, dB, dC = _dev(A), _dev(B), _dev(C)
    rc = cb.lib().CUDA_dgemm(ta, tb, m, n, k, ctypes.byref(al), ctypes.c_void_p(dA.data_ptr()), A.shape[0],
                             ctypes.c_void_p(dB.data_ptr()), B.shape[0], ctypes.byref(be),
                             ctypes.c_void_p(dC.data_ptr()), m, handle)
    torch.cuda.synchronize()
    assert rc == 0
    opA = A if ta == 111 else A.T
    opB = B if tb == 111 else B.T
    ref = -1.5 * opA @ opB + 0.75 * C
    assert np.abs(_host(dC, (m, n)) - ref).max() < 1e-12 * k


@pytest.mark.parametrize("uplo,trans", [(121, 111), (121, 112), (122, 111), (122, 112)])
def test_cuda_dsyrk(cb, handle, uplo, trans):
    import torch
    n, k = 200, 77
    rng = np.random.default_rng(5)
    A = rng.standard_normal((n, k) if trans == 111 else (k, n))
    C = rng.standard_normal((n, n))
    al, be = ctypes.c_double(-1.0), ctypes.c_double(1.0)
    dA, dC = _dev(A), _dev(C)
    assert cb.lib().CUDA_dsyrk(uplo, trans, n, k, ctypes.byref(al), ctypes.c_void_p(dA.data_ptr()), A.shape[0],
                               ctypes.byref(be), ctypes.c_void_p(dC.data_ptr()), n, handle) == 0
    torch.cuda.synchronize()
    opA = A if trans == 111 else A.T
    ref = C - opA @ opA.T
    got = _host(dC, (n, n))
    mask = np.triu(np.ones((n, n), bool)) if uplo == 121 else np.tril(np.ones((n, n), bool))
    assert np.abs(got[mask] - ref[mask]).max() < 1e-12 * k
    assert np.array_equal(got[~mask], C[~mask])


@pytest.mark.parametrize("side", [141, 142])
@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("trans", [111, 112])
@pytest.mark.parametrize("diag", [131, 132])
def test_cuda_dtrsm(cb, handle, side, uplo, trans, diag):
    import torch
    m, n = 150, 70
    na = m if side == 141 else n
    rng = np.random.default_rng(side + uplo + trans + diag)
    T = rng.standard_normal((na, na)) * 0.1 + np.eye(na) * 2
    T = np.triu(T) if uplo == 121 else np.tril(T)
    Tf = T.copy()
    if diag == 132:
        np.fill_diagonal(Tf, 1.0)
    B = rng.standard_normal((m, n))
    al = ctypes.c_double(0.5)
    dT, dB = _dev(T), _dev(B)
    assert cb.lib().CUDA_dtrsm(side, uplo, trans, diag, m, n, ctypes.byref(al), ctypes.c_void_p(dT.data_ptr()),
                               na, ctypes.c_void_p(dB.data_ptr()), m, handle) == 0
    torch.cuda.synchronize()
    op = Tf if trans == 111 else Tf.T
    ref = np.linalg.solve(op, 0.5 * B) if side == 141 else np.linalg.solve(op.T, 0.5 * B.T).T
    assert np.abs(_host(dB, (m, n)) - ref).max() < 1e-11


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("n", [17, 64, 320, 512])
def test_cuda_dpotrf(cb, orc, handle, uplo, n):
    import torch
    A = orc.dplgsy(float(n), n, 21)
    dA = _dev(A)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert cb.lib().CUDA_dpotrf(uplo, n, ctypes.c_void_p(dA.data_ptr()), n, None, 0,
                                ctypes.c_void_p(info.data_ptr()), handle) == 0
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    F = _host(dA, (n, n))
    assert np_check_factorization(uplo, A, F) < 60
    tri = np.triu if uplo == 121 else np.tril
    assert np.array_equal(F - tri(F), A - tri(A))   # other triangle untouched


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("n", [1, 37, 64, 100, 200, 255, 256, 300, 512])
def test_cuda_spotrf(cb, orc, handle, uplo, n):
    """FP32 tile Cholesky (the mixed solver's diagonal-tile kernel: on chip for
    n <= 256, blocked above) against the FP64 factor, to FP32 accuracy, with
    the other triangle untouched; a non-positive pivot gives LAPACK's info."""
    import torch
    A = orc.dplgsy(float(n), n, 23)
    dA = torch.from_numpy(np.asfortranarray(A).T.astype(np.float32).copy()).cuda()
    info = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    L = cb.lib()
    assert L.CUDA_spotrf(uplo, n, ctypes.c_void_p(dA.data_ptr()), n, None, 0,
                         ctypes.c_void_p(info.data_ptr()), handle) == 0
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    F = dA.cpu().numpy().T.astype(np.float64)
    A32 = A.astype(np.float32).astype(np.float64)
    Lref = np.linalg.cholesky(A32)
    tri = np.triu if uplo == 121 else np.tril
    Lg = tri(F) if uplo == 122 else tri(F).T
    assert np.abs(Lg - Lref).max() <= 8 * n * 5.96e-8 * np.sqrt(np.abs(A32).max())
    assert np.array_equal(F - tri(F), A32 - tri(A32))   # other triangle untouched
    if n >= 100:
        B = A.copy()
        B[n - 30, n - 30] = -2.0 * n
        dB = torch.from_numpy(np.asfortranarray(B).T.astype(np.float32).copy()).cuda()
        assert L.CUDA_spotrf(uplo, n, ctypes.c_void_p(dB.data_ptr()), n, None, 0,
                             ctypes.c_void_p(info.data_ptr()), handle) == 0
        torch.cuda.synchronize()
        assert int(info.item()) == n - 29


def test_cuda_generators_match_oracle(cb, orc, handle):
    import torch
    m, n, bigM, m0, n0 = 50, 40, 300, 100, 60
    dA = torch.zeros((n, m), dtype=torch.float64, device="cuda")
    bump = ctypes.c_double(300.0)
    assert cb.lib().CUDA_dplrnt(m, n, ctypes.c_void_p(dA.data_ptr()), m, bigM, m0, n0, 99, handle) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_host(dA, (m, n)), orc.dplrnt(m, n, 99, bigM=bigM, m0=m0, n0=n0))
    full = orc.dplgsy(300.0, 300, 99)
    for (mm0, nn0) in [(100, 60), (60, 100), (80, 80)]:
        assert cb.lib().CUDA_dplgsy(ctypes.byref(bump), m, n, ctypes.c_void_p(dA.data_ptr()), m, bigM, mm0, nn0,
                                    99, handle) == 0
        torch.cuda.synchronize()
        assert np.array_equal(_host(dA, (m, n)), full[mm0:mm0 + m, nn0:nn0 + n])


@pytest.mark.parametrize("m,n", [(70, 33), (4096, 64), (1027, 5), (1, 1), (3, 300)])
def test_cuda_lag2(cb, handle, m, n):
    """Aligned (vector) and unaligned (scalar) columns, ragged row ends."""
    import torch
    rng = np.random.default_rng(1)
    A = rng.standard_normal((m, n))
    dA = _dev(A)
    dS = torch.zeros((n, m), dtype=torch.float32, device="cuda")
    assert cb.lib().CUDA_dlag2s(m, n, ctypes.c_void_p(dA.data_ptr()), m, ctypes.c_void_p(dS.data_ptr()), m,
                                handle) == 0
    torch.cuda.synchronize()
    assert np.array_equal(dS.cpu().numpy().T, A.astype(np.float32))
    assert cb.lib().CHAM_B200_Handle_Overflow(handle) == 0
    dB = torch.zeros_like(dA)
    assert cb.lib().CUDA_slag2d(m, n, ctypes.c_void_p(dS.data_ptr()), m, ctypes.c_void_p(dB.data_ptr()), m,
                                handle) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_host(dB, (m, n)), A.astype(np.float32).astype(np.float64))
    # LAPACK's overflow rule: |a| > FLT_MAX sets the flag, NaN does not
    A[m // 2, n - 1] = np.nan
    dN = _dev(A)
    assert cb.lib().CUDA_dlag2s(m, n, ctypes.c_void_p(dN.data_ptr()), m, ctypes.c_void_p(dS.data_ptr()), m,
                                handle) == 0
    assert cb.lib().CHAM_B200_Handle_Overflow(handle) == 0
    A[m - 1, n // 2] = -1e39
    dO = _dev(A)
    assert cb.lib().CUDA_dlag2s(m, n, ctypes.c_void_p(dO.data_ptr()), m, ctypes.c_void_p(dS.data_ptr()), m,
                                handle) == 0
    assert cb.lib().CHAM_B200_Handle_Overflow(handle) == 1


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB", [(700, 256), (1000, 512)])
def test_fp64_reads_only_uplo_triangle(cb, orc, uplo, N, NB):
    """LAPACK convention: NaN in the unreferenced strict triangle reaches no result."""
    nrhs = 3
    A0 = orc.dplgsy(float(N), N, 71)
    B0 = orc.dplrnt(N, nrhs, 72)
    A = np.asfortranarray(A0.copy())
    if uplo == 121:
        A[np.tril_indices(N, -1)] = np.nan
    else:
        A[np.triu_indices(N, 1)] = np.nan
    cb.set_param(cb.CHAMELEON_TILE_SIZE, NB)
    B = np.asfortranarray(B0.copy())
    assert cb.dposv(uplo, N, nrhs, A, N, B, N) == 0
    assert np.isfinite(B).all()
    assert orc.check_solve(A0, B, B0) < 60


@pytest.mark.parametrize("uplo", [121, 122])
def test_default_stream_writes_are_ordered_before_the_call(cb, uplo):
    """A caller that fills its device matrix on the default stream (here torch
    copies into reused allocations, with no synchronization) and then calls
    dposv_Tile must get the solution of that matrix: the library's stream
    waits for the caller's default-stream work at every entry."""
    import torch
    N, NB, nrhs = 8192, 512, 16
    A0 = torch.zeros((N, N), dtype=torch.float64, device="cuda")
    B0 = torch.zeros((nrhs, N), dtype=torch.float64, device="cuda")
    dA = cb.Desc.create(N, N, NB, mat=A0)
    dB = cb.Desc.create(N, nrhs, NB, mat=B0)
    assert cb.dplgsy_Tile(float(N), 123, dA, 51) == 0
    assert cb.dplrnt_Tile(dB, 5673) == 0
    dA.destroy()
    dB.destroy()
    A = torch.full_like(A0, float("nan"))
    B = torch.full_like(B0, float("nan"))
    for _ in range(3):
        A.fill_(float("nan"))
        B.fill_(float("nan"))
        A.copy_(A0)          # queued on the default stream, not synchronized
        B.copy_(B0)
        dA = cb.Desc.create(N, N, NB, mat=A)
        dB = cb.Desc.create(N, nrhs, NB, mat=B)
        assert cb.dposv_Tile(uplo, dA, dB) == 0
        torch.cuda.synchronize()
        R = B0.T - A0 @ B.T
        r = float(R.abs().sum(0).max() / (A0.abs().sum(0).max() * B.T.abs().sum(0).max() * N * EPS))
        assert r < 60, r
        dA.destroy()
        dB.destroy()


def test_tcuda_tile_forms_match_the_array_forms(cb, orc, handle):
    """TCUDA_d* (gpucublas_ztile.h) take CHAM_tile_t operands, as the runtimes'
    codelets pass them, and give the CUDA_d* results bit for bit; a tile that
    is not full-rank is refused."""
    import torch
    L = cb.lib()
    n, k = 96, 64

    def tile(t, rows, cols, fmt=cb.CHAMELEON_TILE_FULLRANK):
        return cb.CHAM_tile_t(t.data_ptr(), 0, rows, cols, rows, fmt, cb.ChamRealDouble)

    rng = np.random.default_rng(5)
    A = _dev(rng.standard_normal((n, k)))
    B = _dev(rng.standard_normal((n, k)))
    C1 = _dev(rng.standard_normal((n, n)))
    C2 = C1.clone()
    al, be = ctypes.c_double(-1.0), ctypes.c_double(1.0)
    assert L.CUDA_dgemm(111, 112, n, n, k, ctypes.byref(al), ctypes.c_void_p(A.data_ptr()), n,
                        ctypes.c_void_p(B.data_ptr()), n, ctypes.byref(be), ctypes.c_void_p(C1.data_ptr()), n,
                        handle) == 0
    tA, tB, tC = tile(A, n, k), tile(B, n, k), tile(C2, n, n)
    assert L.TCUDA_dgemm(111, 112, n, n, k, ctypes.byref(al), ctypes.byref(tA), ctypes.byref(tB), ctypes.byref(be),
                         ctypes.byref(tC), handle) == 0
    torch.cuda.synchronize()
    assert torch.equal(C1, C2)
    S = orc.dplgsy(float(n), n, 7)
    P1, P2 = _dev(S), _dev(S)
    i1 = torch.zeros(1, dtype=torch.int32, device="cuda")
    i2 = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.CUDA_dpotrf(122, n, ctypes.c_void_p(P1.data_ptr()), n, None, 0, ctypes.c_void_p(i1.data_ptr()),
                         handle) == 0
    tP = tile(P2, n, n)
    assert L.TCUDA_dpotrf(122, n, ctypes.byref(tP), None, 0, ctypes.c_void_p(i2.data_ptr()), handle) == 0
    torch.cuda.synchronize()
    assert torch.equal(P1, P2) and int(i1.item()) == int(i2.item()) == 0
    X1, X2 = _dev(rng.standard_normal((n, k))), None
    X2 = X1.clone()
    one = ctypes.c_double(1.0)
    assert L.CUDA_dtrsm(141, 122, 111, 131, n, k, ctypes.byref(one), ctypes.c_void_p(P1.data_ptr()), n,
                        ctypes.c_void_p(X1.data_ptr()), n, handle) == 0
    tX = tile(X2, n, k)
    assert L.TCUDA_dtrsm(141, 122, 111, 131, n, k, ctypes.byref(one), ctypes.byref(tP), ctypes.byref(tX),
                         handle) == 0
    torch.cuda.synchronize()
    assert torch.equal(X1, X2)
    bad = tile(C2, n, n, cb.CHAMELEON_TILE_DESC)
    assert L.TCUDA_dsyrk(122, 111, n, k, ctypes.byref(al), ctypes.byref(tA), ctypes.byref(be), ctypes.byref(bad),
                         handle) == -103
