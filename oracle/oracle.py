"""Python access to the two CPU checkers (test infrastructure only).

* ``port()``      -- the C restatement oracle/cham_oracle.c, built into
                     oracle/liboracle.so by :func:`build_port`.
* ``reference()`` -- the reference's own CPU library, built from the reference
                     sources by oracle/build_ref.sh into oracle/_ref/libchamref.so.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference arms import this module; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libchamref.so")

UPPER, LOWER, UPPERLOWER = 121, 122, 123
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _ptr(a):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1)
    return a.ctypes.data_as(_dp)


def build_port(force=False):
    src = os.path.join(HERE, "cham_oracle.c")
    if not force and os.path.exists(PORT_SO) and os.path.getmtime(PORT_SO) >= os.path.getmtime(src):
        return PORT_SO
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", src, "-o", PORT_SO + ".tmp", "-lm"])
    os.replace(PORT_SO + ".tmp", PORT_SO)
    return PORT_SO


def reference_source_dir():
    """Where oracle/build_ref.sh reads the reference sources: $CHAMREF_SRC, else
    the recipe's default location."""
    return os.environ.get("CHAMREF_SRC", "/root/reference")


def build_ref(force=False):
    """Build the reference library (needs the reference sources; not on the GPU host)."""
    if not force and os.path.exists(REF_SO):
        return REF_SO
    subprocess.check_call(["bash", os.path.join(HERE, "build_ref.sh")])
    return REF_SO


def build_plugin(force=False):
    """The reference's dposv drivers linked with the B200 runtime plugin
    (oracle/build_plugin.sh; needs the reference sources and libchameleon_b200.so)."""
    out = os.path.join(HERE, "_ref", "libchamb200rt.so")
    src = [os.path.join(HERE, "plugin_harness.c"), os.path.join(HERE, "build_plugin.sh"),
           os.path.join(os.path.dirname(HERE), "chameleon_b200", "runtime", "runtime_b200.c"),
           os.path.join(os.path.dirname(HERE), "chameleon_b200", "libchameleon_b200.so")]
    if not force and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(f) for f in src):
        return out
    subprocess.check_call(["bash", os.path.join(HERE, "build_plugin.sh")])
    return out


_port = None
_ref = None


def port():
    global _port
    if _port is None:
        _port = ctypes.CDLL(build_port())
        L = _port
        L.orc_lcg_skip.restype = ctypes.c_ulonglong
        L.orc_lcg_skip.argtypes = [ctypes.c_ulonglong, ctypes.c_ulonglong]
        L.orc_dplgsy.argtypes = [ctypes.c_double, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_ulonglong]
        L.orc_dplrnt.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_ulonglong]
        L.orc_dpotrf_tiled.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]
        L.orc_dpotrs_tiled.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                       _dp, ctypes.c_int]
        L.orc_check_factorization.restype = ctypes.c_double
        L.orc_check_factorization.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int]
        L.orc_check_solve.restype = ctypes.c_double
        L.orc_check_solve.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                      ctypes.c_int]
    return _port


def reference_available():
    return os.path.exists(REF_SO)


def reference(ncores=0):
    global _ref
    if _ref is None:
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        _ref = ctypes.CDLL(REF_SO)
        L = _ref
        L.chamref_init.argtypes = [ctypes.c_int]
        L.chamref_dplgsy.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_ulonglong]
        L.chamref_dplrnt.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_ulonglong]
        L.chamref_dposv.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                    ctypes.c_int, _dp]
        L.chamref_dpotrf.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp]
        L.chamref_dpotrs.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                     ctypes.c_int]
        L.chamref_dposv_tile_seeded.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_ulonglong, ctypes.c_ulonglong, _dp, _dp, _dp]
        L.chamref_dpotrf_batch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.chamref_dtrsm_batch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.chamref_lapacke_dsposv.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                             ctypes.c_int, _dp, ctypes.c_int, _ip, _dp]
        L.chamref_dgemm_batch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double] + \
            [ctypes.c_int] * 7 + [_dp, _dp, _dp]
        L.chamref_dsyrk_batch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double] + \
            [ctypes.c_int] * 4 + [_dp, _dp]
        L.chamref_dpotrimm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                       ctypes.c_int, _dp, ctypes.c_int]
        L.chamref_dinverse.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                       ctypes.c_int]
        L.chamref_init(ncores if ncores > 0 else (os.cpu_count() or 1))
    return _ref


# ---- convenience wrappers on numpy arrays (column-major) -------------------

def lcg_skip(n, seed):
    return port().orc_lcg_skip(n, seed)


def dplgsy(bump, N, seed, bigM=None, m0=0, n0=0):
    A = np.zeros((N, N), order="F")
    port().orc_dplgsy(bump, N, _ptr(A), max(N, 1), N if bigM is None else bigM, m0, n0, seed)
    return A


def dplrnt(M, N, seed, bigM=None, m0=0, n0=0):
    A = np.zeros((M, N), order="F")
    port().orc_dplrnt(M, N, _ptr(A), max(M, 1), M if bigM is None else bigM, m0, n0, seed)
    return A


def dpotrf_tiled(uplo, A, NB):
    F = np.asfortranarray(A.copy())
    info = port().orc_dpotrf_tiled(uplo, F.shape[0], NB, _ptr(F), max(F.shape[0], 1))
    return F, info


def dpotrs_tiled(uplo, F, B, NB):
    X = np.asfortranarray(B.copy())
    N = F.shape[0]
    port().orc_dpotrs_tiled(uplo, N, X.shape[1], NB, _ptr(F), max(N, 1), _ptr(X), max(N, 1))
    return X


def check_factorization(uplo, A0, F):
    A0 = np.asfortranarray(A0)
    F = np.asfortranarray(F)
    N = A0.shape[0]
    return port().orc_check_factorization(uplo, N, _ptr(A0), max(N, 1), _ptr(F), max(N, 1))


def check_solve(A0, X, B):
    A0, X, B = (np.asfortranarray(a) for a in (A0, X, B))
    N = A0.shape[0]
    return port().orc_check_solve(N, X.shape[1], _ptr(A0), max(N, 1), _ptr(X), max(N, 1), _ptr(B), max(N, 1))


def ref_dposv(uplo, A, B, NB):
    """Reference dposv (LAPACK layout) on copies; returns (F, X, info, seconds)."""
    L = reference()
    F = np.asfortranarray(A.copy())
    X = np.asfortranarray(B.copy())
    t = ctypes.c_double()
    N = F.shape[0]
    info = L.chamref_dposv(uplo, N, X.shape[1], NB, _ptr(F), max(N, 1), _ptr(X), max(N, 1), ctypes.byref(t))
    return F, X, info, t.value


def ref_dplgsy(bump, uplo, N, seed, NB=384):
    L = reference()
    A = np.zeros((N, N), order="F")
    L.chamref_dplgsy(bump, uplo, N, _ptr(A), max(N, 1), NB, seed)
    return A


def ref_dplrnt(M, N, seed, NB=384):
    L = reference()
    A = np.zeros((M, N), order="F")
    L.chamref_dplrnt(M, N, _ptr(A), max(M, 1), NB, seed)
    return A


def ref_dinverse(op, uplo, A, NB, diag=131):
    """Reference CHAMELEON_dpotri / dtrtri / dlauum (op "potri" / "trtri" /
    "lauum"; compute/zpotri.c, ztrtri.c, zlauum.c) on a copy; returns (A', info)."""
    L = reference()
    X = np.asfortranarray(A.copy())
    N = X.shape[0]
    info = L.chamref_dinverse({"potri": 0, "trtri": 1, "lauum": 2}[op], uplo, diag, N, NB, _ptr(X), max(N, 1))
    return X, info


def _stack(X):
    """count x r x c per-tile matrices -> the column-major (count r) x c matrix
    whose tile row i is X[i] (the stacked descriptor the harness builds)."""
    return np.asfortranarray(np.concatenate(list(X), axis=0))


def _unstack(M, cnt):
    r = M.shape[0] // cnt
    return np.stack([M[i * r:(i + 1) * r] for i in range(cnt)])


def ref_dgemm_batch(transA, transB, alpha, A, B, beta, C):
    """Reference CHAMELEON_dgemm_batch_Tile on stacked tiles: A (count, am, an),
    B (count, bm, bn), C (count, m, n) arrays of per-tile matrices; returns C'."""
    L = reference()
    cnt, am, an = A.shape
    _, bm, bn = B.shape
    _, m, n = C.shape
    a, b, c = _stack(A), _stack(B), _stack(C)
    rc = L.chamref_dgemm_batch(transA, transB, alpha, beta, am, an, bm, bn, m, n, cnt, _ptr(a), _ptr(b), _ptr(c))
    assert rc == 0, rc
    return _unstack(c, cnt)


def ref_dsyrk_batch(uplo, trans, alpha, A, beta, C):
    """Reference CHAMELEON_dsyrk_batch_Tile (zherk_batch.c after z->d) on stacked tiles."""
    L = reference()
    cnt, am, an = A.shape
    n = C.shape[1]
    a, c = _stack(A), _stack(C)
    rc = L.chamref_dsyrk_batch(uplo, trans, alpha, beta, am, an, n, cnt, _ptr(a), _ptr(c))
    assert rc == 0, rc
    return _unstack(c, cnt)


def gered(uplo, prec, A, mb):
    """Restatement of chameleon_pzgered (compute/pzgered.c:160-260) with the
    conversion rule of INSERT_TASK_zgered in a CUDA double-precision build
    (runtime/starpu/codelets/codelet_zgered.c): returns (A with the reduced
    tiles rounded, tags[mt, nt] with 0 FP64 / 1 FP32 / 2 FP16)."""
    A = np.array(A, dtype=np.float64, order="F")
    N = A.shape[0]
    mt = (N + mb - 1) // mb
    lower, upper = uplo == 122, uplo == 121
    tiles = []
    for m in range(mt):
        nmin = m if upper else 0
        nmax = min(m + 1, mt) if lower else mt
        for n in range(nmin, nmax):
            sl = np.s_[m * mb:min(N, (m + 1) * mb), n * mb:min(N, (n + 1) * mb)]
            T = A[sl]
            if m == n and (lower or upper):
                T = np.tril(T) if lower else np.triu(T)
            tiles.append((m, n, sl, float(np.sqrt((T * T).sum()))))
    gnorm = float(np.sqrt(sum(t[3] ** 2 for t in tiles)))
    eps = 2.0 ** -53 if prec < 0 else prec
    eps_diag = 2.0 ** -24
    thr = eps * gnorm / mt
    thr_diag = thr if eps < eps_diag else eps_diag * gnorm / mt
    tags = np.zeros((mt, mt), dtype=np.int8)
    for m, n, sl, ln in tiles:
        th = thr_diag if m == n else thr
        if ln < th / 1e-4:
            tags[m, n] = 2
            with np.errstate(over="ignore"):
                A[sl] = A[sl].astype(np.float16).astype(np.float64)
        elif ln < th / eps_diag:
            tags[m, n] = 1
            A[sl] = A[sl].astype(np.float32).astype(np.float64)
    return A, tags


def ref_dpotrimm(uplo, A, B, NB):
    """Reference CHAMELEON_dpotrimm (compute/zpotrimm.c, pzpotrimm.c) on copies:
    returns (A' = uplo triangle of A^-1, C = B A^-1, info)."""
    L = reference()
    Aw = np.asfortranarray(A.copy())
    Bw = np.asfortranarray(B.copy())
    N = Aw.shape[0]
    C = np.zeros((N, N), order="F")
    info = L.chamref_dpotrimm(uplo, N, NB, _ptr(Aw), max(N, 1), _ptr(Bw), max(N, 1), _ptr(C), max(N, 1))
    return Aw, C, info
