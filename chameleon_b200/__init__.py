"""chameleon_b200 -- B200-native tiled Cholesky (dposv) behind Chameleon's API.

The compute lives in the in-tree CUDA library ``libchameleon_b200.so`` (C ABI,
``include/chameleon_b200.h``).  This module is the Python host mirror of the
reference's C interface (include/chameleon.h, include/chameleon/chameleon_z.h
after z->d generation): same entry-point names, argument meaning, enum values
and return codes.  There is no CPU fallback: importing works anywhere, but every
compute call raises ``ChameleonError`` when the CUDA library is not built or no
GPU is present.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchameleon_b200.so")

# include/chameleon/constants.h values
ChamNoTrans, ChamTrans, ChamConjTrans = 111, 112, 113
ChamUpper, ChamLower, ChamUpperLower = 121, 122, 123
ChamNonUnit, ChamUnit = 131, 132
ChamLeft, ChamRight = 141, 142
ChamOneNorm, ChamFrobeniusNorm, ChamInfNorm, ChamMaxNorm = 171, 174, 175, 177
ChamRealFloat, ChamRealDouble = (1 << 2) | 2, (1 << 2) | 3
CHAMELEON_MAT_ALLOC_TILE = ctypes.c_void_p(-1 & 0xFFFFFFFFFFFFFFFF)
CHAMELEON_TILE_SIZE = 2
CHAMELEON_INNER_BLOCK_SIZE = 3
CHAMELEON_B200_PRECISION = 101
CHAMELEON_B200_REFINE_MAXITER = 102
CHAMELEON_B200_WAIT_BUDGET_MS = 103
CHAMELEON_B200_WAIT_BUDGET_US = 104
CHAMELEON_B200_TCGEN05 = 105
CHAMELEON_B200_REC_TILE = 106
CHAMELEON_B200_XINV_SOLVE = 107
CHAMELEON_B200_POTRF_CTA = 108
CHAMELEON_B200_UPD_GROUP_F64 = 109
CHAMELEON_B200_UPD_GROUP_F32 = 110
CHAMELEON_B200_UPD_GROUP_TC = 111
CHAMELEON_B200_FACTOR_NB = 112
CHAMELEON_B200_UPD_TAIL_F64 = 113
PREC_FP64, PREC_FP32, PREC_BF16X3 = 0, 1, 2
CHAMELEON_SUCCESS = 0
CHAMELEON_ERR_NOT_INITIALIZED = -101
CHAMELEON_ERR_ILLEGAL_VALUE = -104
CHAMELEON_ERR_NOT_SUPPORTED = -103
CHAMELEON_ERR_NOT_FOUND = -105
CHAMELEON_ERR_OUT_OF_RESOURCES = -106
CHAMELEON_ERR_UNEXPECTED = -110
CHAMELEON_ERR_DEVICE_TIMEOUT = -120


class ChameleonError(RuntimeError):
    pass


class CHAM_desc_t(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char_p),
        ("get_blkaddr", ctypes.c_void_p),
        ("get_blkldd", ctypes.c_void_p),
        ("tiles", ctypes.c_void_p),
        ("mat", ctypes.c_void_p),
        ("host_mat", ctypes.c_void_p),
        ("A21", ctypes.c_size_t), ("A12", ctypes.c_size_t), ("A22", ctypes.c_size_t),
        ("styp", ctypes.c_int), ("dtyp", ctypes.c_int),
        ("mb", ctypes.c_int), ("nb", ctypes.c_int), ("bsiz", ctypes.c_int),
        ("i", ctypes.c_int), ("j", ctypes.c_int), ("m", ctypes.c_int), ("n", ctypes.c_int),
        ("lm", ctypes.c_int), ("ln", ctypes.c_int),
        ("mt", ctypes.c_int), ("nt", ctypes.c_int), ("lmt", ctypes.c_int), ("lnt", ctypes.c_int),
        ("llm1", ctypes.c_int), ("lln1", ctypes.c_int),
        ("lda", ctypes.c_int), ("alloc_mat", ctypes.c_int), ("id", ctypes.c_int),
        ("schedopt", ctypes.c_void_p),
    ]


class CHAM_tile_t(ctypes.Structure):
    """include/chameleon/struct.h:53-61 (without the trace name)."""
    _fields_ = [("mat", ctypes.c_void_p), ("rank", ctypes.c_int), ("m", ctypes.c_int), ("n", ctypes.c_int),
                ("ld", ctypes.c_int), ("format", ctypes.c_int8), ("flttype", ctypes.c_int)]


CHAMELEON_TILE_FULLRANK, CHAMELEON_TILE_DESC, CHAMELEON_TILE_HMAT = 1, 2, 4


class RefineInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("fallback", ctypes.c_int), ("precision", ctypes.c_int),
                ("backward_error", ctypes.c_double), ("seconds", ctypes.c_double)]


class Task(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int16), ("sub", ctypes.c_int16), ("m", ctypes.c_int16),
                ("n", ctypes.c_int16), ("k", ctypes.c_int16), ("bn", ctypes.c_int16), ("grp", ctypes.c_int32)]


class Request(ctypes.Structure):
    """CHAM_b200_request_t (serving loop)."""
    _fields_ = [("N", ctypes.c_int), ("nrhs", ctypes.c_int), ("uplo", ctypes.c_int),
                ("A", ctypes.c_void_p), ("lda", ctypes.c_int),
                ("B", ctypes.c_void_p), ("ldb", ctypes.c_int),
                ("X", ctypes.c_void_p), ("ldx", ctypes.c_int),
                ("factor_key", ctypes.c_longlong),
                ("status", ctypes.c_int), ("iterations", ctypes.c_int),
                ("t_submit", ctypes.c_double), ("t_start", ctypes.c_double), ("t_done", ctypes.c_double)]


class ServeStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_longlong), ("batches", ctypes.c_longlong),
                ("batched_requests", ctypes.c_longlong), ("max_batch", ctypes.c_longlong),
                ("reused_factors", ctypes.c_longlong), ("kept_factors", ctypes.c_longlong),
                ("bytes_in_use", ctypes.c_double), ("budget_bytes", ctypes.c_double)]


REQ_PENDING = 1 << 30

_D = ctypes.POINTER(CHAM_desc_t)
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_ull = ctypes.c_ulonglong

# name -> (restype, argtypes); every symbol declared in include/chameleon_b200.h
PROTOS = {
    "__chameleon_init": (_i, [_i, _i]),
    "__chameleon_finalize": (_i, []),
    "CHAMELEON_Initialized": (_i, []),
    "CHAMELEON_Set": (_i, [_i, _i]),
    "CHAMELEON_Get": (_i, [_i, ctypes.POINTER(_i)]),
    "CHAMELEON_Enable": (_i, [_i]),
    "CHAMELEON_Disable": (_i, [_i]),
    "CHAMELEON_B200_Strerror": (ctypes.c_char_p, [_i]),
    "CHAMELEON_Desc_Create": (_i, [ctypes.POINTER(_D), _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i]),
    "CHAMELEON_Desc_Destroy": (_i, [ctypes.POINTER(_D)]),
    "CHAMELEON_Desc_Flush": (_i, [_D, _vp]),
    "CHAMELEON_Desc_Acquire": (_i, [_D]),
    "CHAMELEON_Desc_Release": (_i, [_D]),
    "CHAMELEON_Lap2Desc": (_i, [_i, _vp, _i, _D]),
    "CHAMELEON_Desc2Lap": (_i, [_i, _D, _vp, _i]),
    "CHAMELEON_Sequence_Create": (_i, [ctypes.POINTER(_vp)]),
    "CHAMELEON_Sequence_Destroy": (_i, [_vp]),
    "CHAMELEON_Sequence_Wait": (_i, [_vp]),
    "CHAMELEON_dposv": (_i, [_i, _i, _i, _vp, _i, _vp, _i]),
    "CHAMELEON_dposv_Tile": (_i, [_i, _D, _D]),
    "CHAMELEON_dposv_Tile_Async": (_i, [_i, _D, _D, _vp, _vp]),
    "CHAMELEON_dpotrf": (_i, [_i, _i, _vp, _i]),
    "CHAMELEON_dpotrf_Tile": (_i, [_i, _D]),
    "CHAMELEON_dpotrf_Tile_Async": (_i, [_i, _D, _vp, _vp]),
    "CHAMELEON_dpotrs": (_i, [_i, _i, _i, _vp, _i, _vp, _i]),
    "CHAMELEON_dpotrs_Tile": (_i, [_i, _D, _D]),
    "CHAMELEON_dpotrs_Tile_Async": (_i, [_i, _D, _D, _vp, _vp]),
    "CHAMELEON_dpotrf_batch_Tile": (_i, [_i, _D]),
    "CHAMELEON_dtrsm_batch_Tile": (_i, [_i, _i, _i, _i, ctypes.c_double, _D, _D]),
    "CHAM_B200_Dispatch_Cost": (ctypes.c_double, [_i, _i]),
    "CHAM_B200_Dispatch_Bytes": (ctypes.c_double, [_i, _i]),
    "CHAM_B200_Dispatch_Plan": (_i, [_i, _vp, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "CHAMELEON_dgemm_batch_Tile": (_i, [_i, _i, ctypes.c_double, _D, _D, ctypes.c_double, _D]),
    "CHAMELEON_dsyrk_batch_Tile": (_i, [_i, _i, ctypes.c_double, _D, ctypes.c_double, _D]),
    "CHAMELEON_dgered_Tile": (_i, [_i, ctypes.c_double, _D]),
    "CHAMELEON_dgerst_Tile": (_i, [_i, _D]),
    "CHAM_B200_Tile_Precision": (_i, [_D, _i, _i]),
    "CHAMELEON_dtrtri": (_i, [_i, _i, _i, _vp, _i]),
    "CHAMELEON_dlauum": (_i, [_i, _i, _vp, _i]),
    "CHAMELEON_dpotri": (_i, [_i, _i, _vp, _i]),
    "CHAMELEON_dtrtri_Tile": (_i, [_i, _i, _D]),
    "CHAMELEON_dpotrimm": (_i, [_i, _i, _vp, _i, _vp, _i, _vp, _i]),
    "CHAMELEON_dpotrimm_Tile": (_i, [_i, _D, _D, _D]),
    "CHAMELEON_dlauum_Tile": (_i, [_i, _D]),
    "CHAMELEON_dpotri_Tile": (_i, [_i, _D]),
    "CHAMELEON_lapacke_dposv": (_i, [_i, ctypes.c_char, _i, _i, _vp, _i, _vp, _i]),
    "CHAMELEON_lapacke_dpotrf": (_i, [_i, ctypes.c_char, _i, _vp, _i]),
    "CHAMELEON_lapacke_dpotrs": (_i, [_i, ctypes.c_char, _i, _i, _vp, _i, _vp, _i]),
    "CHAMELEON_lapacke_dpotri": (_i, [_i, ctypes.c_char, _i, _vp, _i]),
    "CHAMELEON_lapacke_dlauum": (_i, [_i, ctypes.c_char, _i, _vp, _i]),
    "CHAMELEON_lapacke_dtrtri": (_i, [_i, ctypes.c_char, ctypes.c_char, _i, _vp, _i]),
    "chameleon_lapack_dposv_": (None, [_vp] * 8),
    "chameleon_lapack_dpotrf_": (None, [_vp] * 5),
    "chameleon_lapack_dpotrs_": (None, [_vp] * 8),
    "chameleon_lapack_dpotri_": (None, [_vp] * 5),
    "chameleon_lapack_dlauum_": (None, [_vp] * 5),
    "chameleon_lapack_dtrtri_": (None, [_vp] * 6),
    "CHAMELEON_dplgsy": (_i, [ctypes.c_double, _i, _i, _vp, _i, _ull]),
    "CHAMELEON_dplgsy_Tile": (_i, [ctypes.c_double, _i, _D, _ull]),
    "CHAMELEON_dplrnt": (_i, [_i, _i, _vp, _i, _ull]),
    "CHAMELEON_dplrnt_Tile": (_i, [_D, _ull]),
    "CHAMELEON_dlansy_Tile": (ctypes.c_double, [_i, _i, _D]),
    "CHAMELEON_dlange_Tile": (ctypes.c_double, [_i, _D]),
    "CHAMELEON_dsposv": (_i, [_i, _i, _i, _vp, _i, _vp, _i, _vp, _i, ctypes.POINTER(_i)]),
    "CHAMELEON_dsposv_Tile": (_i, [_i, _D, _D, _D, ctypes.POINTER(_i)]),
    "CHAMELEON_B200_dposv_mixed_Tile": (_i, [_i, _i, _D, _D, _D, ctypes.POINTER(RefineInfo)]),
    "CHAM_B200_Handle_Create": (_i, [ctypes.POINTER(_vp), _vp]),
    "CHAM_B200_Handle_Destroy": (_i, [_vp]),
    "CUDA_dgemm": (_i, [_i, _i, _i, _i, _i, _dp, _vp, _i, _vp, _i, _dp, _vp, _i, _vp]),
    "CUDA_dsyrk": (_i, [_i, _i, _i, _i, _dp, _vp, _i, _dp, _vp, _i, _vp]),
    "CUDA_dtrsm": (_i, [_i, _i, _i, _i, _i, _i, _dp, _vp, _i, _vp, _i, _vp]),
    "CUDA_dpotrf": (_i, [_i, _i, _vp, _i, _vp, _i, _vp, _vp]),
    "CUDA_spotrf": (_i, [_i, _i, _vp, _i, _vp, _i, _vp, _vp]),
    "TCUDA_dgemm": (_i, [_i, _i, _i, _i, _i, _dp, _vp, _vp, _dp, _vp, _vp]),
    "TCUDA_dsyrk": (_i, [_i, _i, _i, _i, _dp, _vp, _dp, _vp, _vp]),
    "TCUDA_dtrsm": (_i, [_i, _i, _i, _i, _i, _i, _dp, _vp, _vp, _vp]),
    "TCUDA_dpotrf": (_i, [_i, _i, _vp, _vp, _i, _vp, _vp]),
    "TCUDA_dplgsy": (_i, [_dp, _i, _i, _vp, _i, _i, _i, _ull, _vp]),
    "TCUDA_dplrnt": (_i, [_i, _i, _vp, _i, _i, _i, _ull, _vp]),
    "TCUDA_dlag2s": (_i, [_i, _i, _vp, _vp, _vp]),
    "TCUDA_slag2d": (_i, [_i, _i, _vp, _vp, _vp]),
    "CUDA_dpotrf_noalloc": (_i, [_i, _i, _vp, _i, _vp, _vp]),
    "CUDA_dplgsy": (_i, [_dp, _i, _i, _vp, _i, _i, _i, _i, _ull, _vp]),
    "CUDA_dplrnt": (_i, [_i, _i, _vp, _i, _i, _i, _i, _ull, _vp]),
    "CUDA_dlag2s": (_i, [_i, _i, _vp, _i, _vp, _i, _vp]),
    "CUDA_slag2d": (_i, [_i, _i, _vp, _i, _vp, _i, _vp]),
    "CHAM_B200_dposv_batch": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "CHAM_B200_sposv_batch": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "CHAM_B200_Serve_Create": (_i, [ctypes.POINTER(_vp), _i, ctypes.c_double, _i]),
    "CHAM_B200_Serve_Submit": (_i, [_vp, ctypes.POINTER(Request)]),
    "CHAM_B200_Serve_Drain": (_i, [_vp]),
    "CHAM_B200_Serve_Stats": (_i, [_vp, ctypes.POINTER(ServeStats)]),
    "CHAM_B200_Serve_Destroy": (_i, [_vp]),
    "CHAM_B200_Serve_Now": (ctypes.c_double, []),
}
# library extras (not in the public header): tracing, schedule inspection, timing
EXTRAS = {
    "CHAM_B200_Handle_Overflow": (_i, [_vp]),
    "CHAM_B200_Trace_Enable": (_i, [_i]),
    "CHAM_B200_Trace_Read": (_i, [_vp, _i]),
    "CHAM_B200_Dag_Create": (_i, [ctypes.POINTER(_vp)]),
    "CHAM_B200_Dag_Destroy": (_i, [_vp]),
    "CHAM_B200_Dag_Clear": (_i, [_vp]),
    "CHAM_B200_Dag_Record": (_i, [_vp, _i, _i, _i, _i, _i]),
    "CHAM_B200_Dag_Size": (_i, [_vp]),
    "CHAM_B200_Dag_Get": (_i, [_vp, _vp, _i]),
    "CHAM_B200_Dag_Schedule": (_i, [_vp, _i, _i, _i, _i, _i, _vp, _i]),
    "CHAM_B200_Dag_Run": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp]),
    "CHAM_B200_Init": (_i, []),
    "CHAM_B200_Schedule_Size": (_i, [_i, _i, _i, _i, _i, _i, _i, _i]),
    "CHAM_B200_Schedule_Build": (_i, [_i, _i, _i, _i, _i, _i, _i, _i, ctypes.POINTER(Task), _i]),
    "CHAM_B200_dposv_timed": (_i, [_i, _i, _i, _vp, _i, _vp, _i, ctypes.POINTER(ctypes.c_float)]),
    "CHAM_B200_Event_Record": (_i, [_i]),
    "CHAM_B200_Event_Elapsed": (ctypes.c_float, [_i, _i]),
    "CHAM_B200_Launch_Count": (ctypes.c_ulonglong, []),
    "CHAM_B200_Device_Sync": (_i, []),
    "CHAM_B200_Mixed_Stats": (_i, [_dp]),
    "CHAM_B200_Test_TC05": (_i, [_vp, _vp, _i, _vp]),
    "CHAM_B200_Mixed_Factor_Only": (_i, [_i, _i, _D, _D, ctypes.POINTER(ctypes.c_float)]),
    "CHAM_B200_Batch_Tuning": (_i, [_i, _dp]),
    "CHAM_B200_Batch_SetShape": (_i, [_i, _i, _i]),
}

_lib = None


def lib():
    """Load the CUDA library; raise if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ChameleonError("libchameleon_b200.so is not built (run `python -m chameleon_b200.build`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in {**PROTOS, **EXTRAS}.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def missing_symbols():
    L = lib()
    return [n for n in PROTOS if not hasattr(L, n)]


def check(rc, what=""):
    if rc != 0:
        msg = lib().CHAMELEON_B200_Strerror(rc).decode()
        raise ChameleonError("%s returned %d (%s)" % (what, rc, msg))
    return rc


_initialized = False


def init(ncpus=0, ngpus=1):
    """CHAMELEON_Init (idempotent here)."""
    global _initialized
    L = lib()
    if L.CHAMELEON_Initialized():
        _initialized = True
        return 0
    rc = L.__chameleon_init(ncpus, ngpus)
    if rc != 0:
        raise ChameleonError("CHAMELEON_Init failed (%d): no usable CUDA device" % rc)
    _initialized = True
    return 0


def finalize():
    global _initialized
    if _initialized:
        lib().__chameleon_finalize()
        _initialized = False


def set_param(param, value):
    return check(lib().CHAMELEON_Set(param, value), "CHAMELEON_Set")


def get_param(param):
    v = ctypes.c_int()
    check(lib().CHAMELEON_Get(param, ctypes.byref(v)), "CHAMELEON_Get")
    return v.value


def _addr(x):
    """Device/host address of a torch tensor or numpy array (column-major storage expected)."""
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(x.ctypes.data)


class Desc:
    """Owning wrapper of a CHAM_desc_t* (CHAMELEON_Desc_Create / Destroy)."""

    def __init__(self, ptr, keep=None):
        self.ptr = ptr
        self._keep = keep

    @classmethod
    def create(cls, m, n, mb, nb=None, dtyp=ChamRealDouble, mat=None):
        nb = mb if nb is None else nb
        init()
        p = _D()
        matp = CHAMELEON_MAT_ALLOC_TILE if mat is None else _addr(mat)
        check(lib().CHAMELEON_Desc_Create(ctypes.byref(p), matp, dtyp, mb, nb, mb * nb, m, n, 0, 0, m, n, 1, 1),
              "CHAMELEON_Desc_Create")
        return cls(p, keep=mat)

    @property
    def d(self):
        return self.ptr.contents

    def destroy(self):
        if self.ptr:
            lib().CHAMELEON_Desc_Destroy(ctypes.byref(self.ptr))
            self.ptr = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def to_numpy(self, uplo=ChamUpperLower):
        d = self.d
        A = np.zeros((d.m, d.n), order="F")
        check(lib().CHAMELEON_Desc2Lap(uplo, self.ptr, _addr(A), max(d.m, 1)), "CHAMELEON_Desc2Lap")
        return A

    def from_numpy(self, A, uplo=ChamUpperLower):
        A = np.asfortranarray(A, dtype=np.float64)
        check(lib().CHAMELEON_Lap2Desc(uplo, _addr(A), max(A.shape[0], 1), self.ptr), "CHAMELEON_Lap2Desc")


# ---- reference-named entry points --------------------------------------------

def dplgsy_Tile(bump, uplo, A, seed):
    return lib().CHAMELEON_dplgsy_Tile(bump, uplo, A.ptr, seed)


def dplrnt_Tile(A, seed):
    return lib().CHAMELEON_dplrnt_Tile(A.ptr, seed)


def dposv_Tile(uplo, A, B):
    return lib().CHAMELEON_dposv_Tile(uplo, A.ptr, B.ptr)


def dpotrf_Tile(uplo, A):
    return lib().CHAMELEON_dpotrf_Tile(uplo, A.ptr)


def dpotrs_Tile(uplo, A, B):
    return lib().CHAMELEON_dpotrs_Tile(uplo, A.ptr, B.ptr)


def dlansy_Tile(norm, uplo, A):
    return lib().CHAMELEON_dlansy_Tile(norm, uplo, A.ptr)


def dposv(uplo, N, NRHS, A, LDA, B, LDB):
    """CHAMELEON_dposv on caller arrays (numpy host arrays or torch CUDA tensors, column-major)."""
    init()
    return lib().CHAMELEON_dposv(uplo, N, NRHS, _addr(A), LDA, _addr(B), LDB)


def dpotrf(uplo, N, A, LDA):
    init()
    return lib().CHAMELEON_dpotrf(uplo, N, _addr(A), LDA)


def dpotrs(uplo, N, NRHS, A, LDA, B, LDB):
    init()
    return lib().CHAMELEON_dpotrs(uplo, N, NRHS, _addr(A), LDA, _addr(B), LDB)


def dtrtri(uplo, diag, N, A, LDA):
    """CHAMELEON_dtrtri (compute/ztrtri.c): the uplo triangle of A <- its inverse."""
    init()
    return lib().CHAMELEON_dtrtri(uplo, diag, N, _addr(A), LDA)


def dlauum(uplo, N, A, LDA):
    """CHAMELEON_dlauum (compute/zlauum.c): the uplo triangle of L^T L / U U^T."""
    init()
    return lib().CHAMELEON_dlauum(uplo, N, _addr(A), LDA)


def dpotri(uplo, N, A, LDA):
    """CHAMELEON_dpotri (compute/zpotri.c): A^-1 from the Cholesky factor in A."""
    init()
    return lib().CHAMELEON_dpotri(uplo, N, _addr(A), LDA)


def dtrtri_Tile(uplo, diag, A):
    init()
    return lib().CHAMELEON_dtrtri_Tile(uplo, diag, A.ptr)


def dlauum_Tile(uplo, A):
    init()
    return lib().CHAMELEON_dlauum_Tile(uplo, A.ptr)


def dpotri_Tile(uplo, A):
    init()
    return lib().CHAMELEON_dpotri_Tile(uplo, A.ptr)


def dplgsy(bump, uplo, N, A, LDA, seed):
    init()
    return lib().CHAMELEON_dplgsy(bump, uplo, N, _addr(A), LDA, seed)


def dplrnt(M, N, A, LDA, seed):
    init()
    return lib().CHAMELEON_dplrnt(M, N, _addr(A), LDA, seed)


def dsposv_Tile(uplo, A, B, X):
    """CHAMELEON_dsposv_Tile: returns (rc, ITER)."""
    it = ctypes.c_int()
    rc = lib().CHAMELEON_dsposv_Tile(uplo, A.ptr, B.ptr, X.ptr, ctypes.byref(it))
    return rc, it.value


def dposv_mixed_Tile(uplo, precision, A, B, X):
    """CHAMELEON_B200_dposv_mixed_Tile: returns (rc, RefineInfo)."""
    info = RefineInfo()
    rc = lib().CHAMELEON_B200_dposv_mixed_Tile(uplo, precision, A.ptr, B.ptr, X.ptr, ctypes.byref(info))
    return rc, info


def dsposv(uplo, N, NRHS, A, LDA, B, LDB, X, LDX):
    init()
    it = ctypes.c_int()
    rc = lib().CHAMELEON_dsposv(uplo, N, NRHS, _addr(A), LDA, _addr(B), LDB, _addr(X), LDX, ctypes.byref(it))
    return rc, it.value


PROF_FP64, PROF_F32_MMA, PROF_F32_TC05 = 0, 1, 2


def schedule(mode, N, NB, nrhs=0, NBB=None, workers=148, prof=PROF_FP64, kgroup=1):
    """The executor's task list for a shape, cost profile and update group
    size (host-only; no GPU needed): rows (kind, sub, m, n, k, bn, grp)."""
    L = lib()
    NBB = NB if NBB is None else NBB
    n = L.CHAM_B200_Schedule_Size(mode, N, NB, nrhs, NBB, workers, prof, kgroup)
    buf = (Task * max(n, 1))()
    got = L.CHAM_B200_Schedule_Build(mode, N, NB, nrhs, NBB, workers, prof, kgroup, buf, n)
    if got != n:
        raise ChameleonError("schedule build returned %d of %d" % (got, n))
    raw = np.frombuffer(buf, dtype=np.int16).reshape(-1, 8)[:n]
    grp = raw[:, 6:8].copy().view(np.int32)
    return np.concatenate([raw[:, :6].astype(np.int32), grp], axis=1)


class Server:
    """Serving loop (CHAM_B200_Serve_*): submit solve requests, read results.

    Arrays are host arrays (numpy or pinned torch CPU tensors), column-major:
    A is N x N (lower triangle read for ChamLower), B and X are N x nrhs.  The
    caller keeps them alive until the request completes (`drain()`).
    """

    def __init__(self, slots=4, hbm_budget_bytes=0.0, small_n=512):
        init()
        h = ctypes.c_void_p()
        check(lib().CHAM_B200_Serve_Create(ctypes.byref(h), slots, float(hbm_budget_bytes), small_n),
              "CHAM_B200_Serve_Create")
        self.h = h
        self._keep = {}

    @staticmethod
    def now():
        return lib().CHAM_B200_Serve_Now()

    def submit(self, A, B, X, nrhs=None, N=None, uplo=ChamLower, factor_key=-1, lda=None, ldb=None, ldx=None):
        """Queue one solve; returns the Request (status == REQ_PENDING until done)."""
        r = Request()
        r.N = N if N is not None else B.shape[0]
        r.nrhs = nrhs if nrhs is not None else (B.shape[1] if B.ndim > 1 else 1)
        r.uplo = uplo
        r.A = _addr(A).value if A is not None else None
        r.lda = lda if lda is not None else r.N
        r.B = _addr(B).value
        r.ldb = ldb if ldb is not None else r.N
        r.X = _addr(X).value
        r.ldx = ldx if ldx is not None else r.N
        r.factor_key = factor_key
        check(lib().CHAM_B200_Serve_Submit(self.h, ctypes.byref(r)), "CHAM_B200_Serve_Submit")
        self._keep[id(r)] = (r, A, B, X)
        return r

    def drain(self):
        check(lib().CHAM_B200_Serve_Drain(self.h), "CHAM_B200_Serve_Drain")
        self._keep.clear()

    def stats(self):
        st = ServeStats()
        check(lib().CHAM_B200_Serve_Stats(self.h, ctypes.byref(st)), "CHAM_B200_Serve_Stats")
        return {k: getattr(st, k) for k, _ in ServeStats._fields_}

    def close(self):
        if self.h:
            lib().CHAM_B200_Serve_Destroy(self.h)
            self.h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
