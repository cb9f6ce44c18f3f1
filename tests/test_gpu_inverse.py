"""GPU parity of dtrtri / dlauum / dpotri and of the LAPACKE / Fortran LAPACK
entry points, through the C ABI.

The reference computes the SPD inverse as pztrtri then pzlauum
(compute/zpotri.c); its tests (testing/testing_zpotri.c, testing_ztrtri.c,
testing_zlauum.c) check A * A^-1 against the identity.  Here each result is
compared with numpy and, where the reference's own CPU build is present, with
the reference run on the same input.  Tolerances are FP64 backward-error
style: n * eps times the condition-scaled magnitudes.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 1.1102230246251565e-16
UPPER, LOWER = 121, 122
NONUNIT, UNIT = 131, 132


def spd(orc, N, seed=51):
    return orc.dplgsy(float(N), N, seed)


def factor(cb, uplo, A):
    F = np.asfortranarray(A.copy())
    assert cb.dpotrf(uplo, A.shape[0], F, max(A.shape[0], 1)) == 0
    return F


def tri(uplo):
    return np.triu if uplo == UPPER else np.tril


def other(uplo, X):
    """The triangle a call must leave alone (strictly outside uplo)."""
    return np.tril(X, -1) if uplo == UPPER else np.triu(X, 1)


@pytest.mark.parametrize("uplo", [UPPER, LOWER])
@pytest.mark.parametrize("N", [1, 37, 300, 1000, 2500])
def test_dpotri_matches_inverse_and_reference(cb, orc, uplo, N):
    A = spd(orc, N)
    F = factor(cb, uplo, A)
    sentinel = np.full((N, N), 7.25)
    W = np.asfortranarray(tri(uplo)(F) + other(uplo, sentinel))
    assert cb.dpotri(uplo, N, W, max(N, 1)) == 0
    assert np.array_equal(other(uplo, W), other(uplo, sentinel))   # other triangle untouched
    Ainv = tri(uplo)(W) + (np.tril(W, -1).T if uplo == LOWER else np.triu(W, 1).T)
    # testing_zpotri.c check: || I - A A^-1 || / (N eps ||A|| ||A^-1||)
    R = np.eye(N) - A @ Ainv
    res = np.abs(R).sum(0).max() / (N * EPS * np.abs(A).sum(0).max() * np.abs(Ainv).sum(0).max())
    assert res < 60
    ref = np.linalg.inv(A)
    assert np.abs(Ainv - ref).max() <= 64 * N * EPS * np.abs(ref).max()
    if orc.reference_available():
        Fr = np.asfortranarray(tri(uplo)(F))
        Xr, info = orc.ref_dinverse("potri", uplo, Fr, 320)
        assert info == 0
        assert np.abs(tri(uplo)(W) - tri(uplo)(Xr)).max() <= 64 * N * EPS * np.abs(ref).max()


@pytest.mark.parametrize("uplo", [UPPER, LOWER])
@pytest.mark.parametrize("diag", [NONUNIT, UNIT])
@pytest.mark.parametrize("N", [1, 64, 333, 1500])
def test_dtrtri_matches_inverse_and_reference(cb, orc, uplo, diag, N):
    A = spd(orc, N, seed=17)
    T = tri(uplo)(factor(cb, uplo, A))
    sentinel = np.full((N, N), -3.5)
    W = np.asfortranarray(T + other(uplo, sentinel))
    if diag == UNIT:
        np.fill_diagonal(W, 11.0)                         # not referenced, not written
    assert cb.dtrtri(uplo, diag, N, W, max(N, 1)) == 0
    assert np.array_equal(other(uplo, W), other(uplo, sentinel))
    Te = T.copy()
    if diag == UNIT:
        np.fill_diagonal(Te, 1.0)
        assert np.all(np.diag(W) == 11.0)
    X = tri(uplo)(W)
    if diag == UNIT:
        np.fill_diagonal(X, 1.0)
    ref = np.linalg.inv(Te)
    scale = np.abs(ref).max() * max(1.0, np.abs(Te).max() * np.abs(ref).max())
    assert np.abs(X - ref).max() <= 64 * N * EPS * scale
    if orc.reference_available():
        Wr = np.asfortranarray(T + other(uplo, sentinel))
        if diag == UNIT:
            np.fill_diagonal(Wr, 11.0)
        Xr, info = orc.ref_dinverse("trtri", uplo, Wr, 256, diag=diag)
        assert info == 0
        if diag == UNIT:
            assert np.all(np.diag(Xr) == 11.0)
        assert np.abs(tri(uplo)(W) - tri(uplo)(Xr)).max() <= 64 * N * EPS * scale


@pytest.mark.parametrize("uplo", [UPPER, LOWER])
def test_dtrtri_reports_first_zero_pivot_and_leaves_a(cb, orc, uplo):
    N = 200
    T = tri(uplo)(factor(cb, uplo, spd(orc, N)))
    T[57, 57] = 0.0
    T[120, 120] = 0.0
    W = np.asfortranarray(T.copy())
    assert cb.dtrtri(uplo, NONUNIT, N, W, N) == 58           # LAPACK info: 1-based index of the first zero
    assert np.array_equal(W, T)
    # (the reference documents this info for CHAMELEON_dtrtri, compute/ztrtri.c;
    # its OpenMP runtime drops the codelet's iinfo, codelet_ztrtri.c:27-31, so
    # the CPU build is no oracle for it)


@pytest.mark.parametrize("uplo", [UPPER, LOWER])
@pytest.mark.parametrize("N", [1, 100, 777, 2048])
def test_dlauum_matches_product_and_reference(cb, orc, uplo, N):
    rng = np.random.default_rng(N)
    T = tri(uplo)(rng.standard_normal((N, N)))
    sentinel = np.full((N, N), 2.5)
    W = np.asfortranarray(T + other(uplo, sentinel))
    assert cb.dlauum(uplo, N, W, max(N, 1)) == 0
    assert np.array_equal(other(uplo, W), other(uplo, sentinel))
    P = T.T @ T if uplo == LOWER else T @ T.T
    assert np.abs(tri(uplo)(W) - tri(uplo)(P)).max() <= 4 * N * EPS * np.abs(T).max() ** 2 * N ** 0.5
    if orc.reference_available():
        Xr, info = orc.ref_dinverse("lauum", uplo, T, 192)
        assert info == 0
        assert np.abs(tri(uplo)(W) - tri(uplo)(Xr)).max() <= 4 * N * EPS * np.abs(T).max() ** 2 * N ** 0.5


def test_inverse_on_device_arrays_and_ld(cb, orc):
    import torch
    N, lda = 700, 731
    A = spd(orc, N)
    F = factor(cb, LOWER, A)
    host = np.zeros((lda, N), order="F")
    host[:N] = F
    dev = torch.from_numpy(host.T.copy()).cuda()                 # row-major (N, lda) = column-major lda x N
    assert cb.dpotri(LOWER, N, dev, lda) == 0
    W = dev.cpu().numpy().T[:N]
    Ainv = np.tril(W) + np.tril(W, -1).T
    ref = np.linalg.inv(A)
    assert np.abs(Ainv - ref).max() <= 64 * N * EPS * np.abs(ref).max()


@pytest.mark.parametrize("uplo", [UPPER, LOWER])
@pytest.mark.parametrize("N,NB", [(1000, 128), (517, 96)])
def test_inverse_tile_forms(cb, orc, uplo, N, NB):
    A = spd(orc, N)
    F = factor(cb, uplo, A)
    d = cb.Desc.create(N, N, NB)
    d.from_numpy(F)
    assert cb.dpotri_Tile(uplo, d) == 0
    W = d.to_numpy()
    Wl = np.asfortranarray(F.copy())
    assert cb.dpotri(uplo, N, Wl, N) == 0
    assert np.abs(tri(uplo)(W) - tri(uplo)(Wl)).max() <= 8 * N * EPS * np.abs(tri(uplo)(Wl)).max()
    assert np.array_equal(other(uplo, W), other(uplo, F))
    T = tri(uplo)(F)
    d.from_numpy(T)
    assert cb.dtrtri_Tile(uplo, NONUNIT, d) == 0
    X = tri(uplo)(d.to_numpy())
    ref = np.linalg.inv(T)
    assert np.abs(X - ref).max() <= 64 * N * EPS * np.abs(ref).max() * np.abs(T).max() * np.abs(ref).max()
    d.from_numpy(T)
    assert cb.dlauum_Tile(uplo, d) == 0
    P = T.T @ T if uplo == LOWER else T @ T.T
    assert np.abs(tri(uplo)(d.to_numpy()) - tri(uplo)(P)).max() <= 4 * N * EPS * np.abs(P).max()


def test_lapacke_and_fortran_entry_points(cb, orc):
    L = cb.lib()
    COL = 102
    N, nrhs = 600, 7
    A = spd(orc, N)
    B = orc.dplrnt(N, nrhs, 5673)
    Xr = np.linalg.solve(A, B)
    for ch in (b"L", b"l", b"U", b"u"):
        Aw, Bw = np.asfortranarray(A.copy()), np.asfortranarray(B.copy())
        assert L.CHAMELEON_lapacke_dposv(COL, ch, N, nrhs, cb._addr(Aw), N, cb._addr(Bw), N) == 0
        assert np.abs(Bw - Xr).max() < 1e-12
    # layout other than column-major: -1 (lapack_api/src/lapack_zposv.c)
    Aw, Bw = np.asfortranarray(A.copy()), np.asfortranarray(B.copy())
    assert L.CHAMELEON_lapacke_dposv(101, b"L", N, nrhs, cb._addr(Aw), N, cb._addr(Bw), N) == -1
    assert np.array_equal(Bw, B)
    # an illegal uplo reaches CHAMELEON_dposv as an illegal value: argument 1
    assert L.CHAMELEON_lapacke_dposv(COL, b"X", N, nrhs, cb._addr(Aw), N, cb._addr(Bw), N) == -1
    assert L.CHAMELEON_lapacke_dtrtri(COL, b"L", b"Q", N, cb._addr(Aw), N) == -2
    # potrf + potrs == posv; potri after potrf == inv
    Aw, Bw = np.asfortranarray(A.copy()), np.asfortranarray(B.copy())
    assert L.CHAMELEON_lapacke_dpotrf(COL, b"L", N, cb._addr(Aw), N) == 0
    assert L.CHAMELEON_lapacke_dpotrs(COL, b"L", N, nrhs, cb._addr(Aw), N, cb._addr(Bw), N) == 0
    assert np.abs(Bw - Xr).max() < 1e-12
    assert L.CHAMELEON_lapacke_dpotri(COL, b"L", N, cb._addr(Aw), N) == 0
    ref = np.linalg.inv(A)
    assert np.abs(np.tril(Aw) - np.tril(ref)).max() <= 64 * N * EPS * np.abs(ref).max()
    # Fortran: arguments by reference, info out
    c_int = ctypes.c_int
    info = c_int(-99)
    Aw, Bw = np.asfortranarray(A.copy()), np.asfortranarray(B.copy())
    up = ctypes.c_char(b"U")
    L.chameleon_lapack_dposv_(ctypes.byref(up), ctypes.byref(c_int(N)), ctypes.byref(c_int(nrhs)), cb._addr(Aw),
                              ctypes.byref(c_int(N)), cb._addr(Bw), ctypes.byref(c_int(N)), ctypes.byref(info))
    assert info.value == 0
    assert np.abs(Bw - Xr).max() < 1e-12
    T = np.triu(Aw)
    L.chameleon_lapack_dtrtri_(ctypes.byref(up), ctypes.byref(ctypes.c_char(b"N")), ctypes.byref(c_int(N)),
                               cb._addr(Aw), ctypes.byref(c_int(N)), ctypes.byref(info))
    assert info.value == 0
    refT = np.linalg.inv(T)
    assert np.abs(np.triu(Aw) - refT).max() <= 64 * N * EPS * np.abs(refT).max() * np.abs(T).max() * np.abs(refT).max()
    # not positive definite: info = order of the failing minor, as dposv
    Ab = np.asfortranarray(A.copy())
    Ab[300, 300] = -1.0
    Bw = np.asfortranarray(B.copy())
    L.chameleon_lapack_dposv_(ctypes.byref(ctypes.c_char(b"L")), ctypes.byref(c_int(N)), ctypes.byref(c_int(nrhs)),
                              cb._addr(Ab), ctypes.byref(c_int(N)), cb._addr(Bw), ctypes.byref(c_int(N)),
                              ctypes.byref(info))
    assert info.value == 301


@pytest.mark.parametrize("uplo", [UPPER, LOWER])
@pytest.mark.parametrize("N", [1, 130, 1000])
def test_dpotrimm_lapack_and_tile(cb, orc, uplo, N):
    """compute/zpotrimm.c: A (SPD) <- uplo triangle of A^-1, C <- B A^-1."""
    A = spd(orc, N, seed=23)
    B = orc.dplrnt(N, N, 77)
    inv = np.linalg.inv(A)
    sentinel = np.full((N, N), 5.5)
    Aw = np.asfortranarray(tri(uplo)(A) + other(uplo, sentinel))
    Bw = np.asfortranarray(B.copy())
    C = np.zeros((N, N), order="F")
    L = cb.lib()
    assert L.CHAMELEON_dpotrimm(uplo, N, cb._addr(Aw), N, cb._addr(Bw), N, cb._addr(C), N) == 0
    assert np.array_equal(other(uplo, Aw), other(uplo, sentinel))
    scale = np.abs(inv).max()
    assert np.abs(tri(uplo)(Aw) - tri(uplo)(inv)).max() <= 64 * N * EPS * scale
    tolc = 64 * N * EPS * scale * np.abs(B).max() * max(1, N) ** 0.5
    assert np.abs(C - B @ inv).max() <= tolc
    assert np.array_equal(Bw, B)
    if orc.reference_available() and N > 1:
        Ar, Cr, info = orc.ref_dpotrimm(uplo, A, B, 320)
        assert info == 0
        assert np.abs(tri(uplo)(Aw) - tri(uplo)(Ar)).max() <= 64 * N * EPS * scale
        assert np.abs(C - Cr).max() <= tolc
    if N >= 130:
        dA, dB, dC = (cb.Desc.create(N, N, 96) for _ in range(3))
        dA.from_numpy(A)
        dB.from_numpy(B)
        assert L.CHAMELEON_dpotrimm_Tile(uplo, dA.ptr, dB.ptr, dC.ptr) == 0
        assert np.abs(tri(uplo)(dA.to_numpy()) - tri(uplo)(Aw)).max() <= 16 * N * EPS * scale
        assert np.abs(dC.to_numpy() - C).max() <= tolc
    if N > 1:
        # not positive definite: info from the factorization
        Ab = np.asfortranarray(A.copy())
        Ab[N // 2, N // 2] = -1.0
        assert L.CHAMELEON_dpotrimm(uplo, N, cb._addr(Ab), N, cb._addr(Bw), N, cb._addr(C), N) == N // 2 + 1
