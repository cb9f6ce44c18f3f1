// inverse.cu -- triangular inverse, triangular product and SPD inverse from
// the Cholesky factor (dtrtri, dlauum, dpotri), and the LAPACKE / Fortran
// LAPACK interfaces of the Cholesky path.
//
// Reference: compute/ztrtri.c, zlauum.c, zpotri.c (zpotri = pztrtri then
// pzlauum, compute/zpotri.c), lapack_api/src/lapack_z{posv,potrf,potrs,potri,
// trtri,lauum}.c.  On the B200 each one is whole-matrix GPU work on the tile
// kernels of the tile ABI:
//   dtrtri: X = op(T)^-1 as the solution of T X = I (CUDA_dtrsm: blocked
//           substitution with inverted 64 x 64 diagonal blocks, FP64 DMMA),
//           then the referenced triangle of X into A;
//   dlauum: A <- L^T L (lower) / U U^T (upper) as one FP64 GEMM of the
//           triangular factor (zero-filled copy) with its transpose;
//   dpotri: dtrtri then dlauum, as LAPACK and the reference.
// LAPACK's contract is kept: only the `uplo` triangle of A is read and
// written; dtrtri returns info = i when A(i,i) is exactly zero (A untouched),
// with diag = Unit the diagonal is neither read nor written.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "core.cuh"
#include "internal.h"

struct cham_b200_handle_s;   // tile_abi.cu

namespace chb {

// dst <- the `uplo` triangle of src (N x N, column-major), zero elsewhere
// (zero_other) or left untouched; the diagonal is skipped when skip_diag.
__global__ void tri_copy_kernel(const double *src, int64_t lds, double *dst, int64_t ldd, int N, int upper,
                                int zero_other, int skip_diag) {
    const int64_t total = (int64_t)N * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % N), j = (int)(idx / N);
        const bool in = upper ? i <= j : i >= j;
        if (i == j && skip_diag) continue;
        if (in) dst[i + j * ldd] = src[i + j * lds];
        else if (zero_other) dst[i + j * ldd] = 0.0;
    }
}

__global__ void identity_kernel(double *X, int64_t ld, int N) {
    const int64_t total = (int64_t)N * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % N), j = (int)(idx / N);
        X[i + j * ld] = (i == j) ? 1.0 : 0.0;
    }
}

// *first = min over i of (i + 1) with A(i,i) == 0 (INT_MAX: none).
__global__ void zero_diag_kernel(const double *A, int64_t lda, int N, int *first) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        if (A[i + (int64_t)i * lda] == 0.0) atomicMin(first, i + 1);
}

namespace {
int grid_for(int64_t total) { return (int)std::min<int64_t>(std::max<int64_t>((total + 255) / 256, 1), 148 * 16); }

// A handle of the tile ABI on the library stream (kept).
cublasHandle_t lib_handle() {
    static cublasHandle_t h = nullptr;
    if (!h && CHAM_B200_Handle_Create(&h, ctx().stream) != 0) h = nullptr;
    return h;
}

double *g_w1 = nullptr, *g_w2 = nullptr, *g_w3 = nullptr, *g_w4 = nullptr;
size_t g_w1_bytes = 0, g_w2_bytes = 0, g_w3_bytes = 0, g_w4_bytes = 0;
int *g_flag = nullptr;

double *work(double **buf, size_t *cap, size_t bytes) {
    if (bytes > *cap) {
        cudaStreamSynchronize(ctx().stream);
        dev_free(*buf);
        *cap = 0;
        if (!(*buf = (double *)dev_alloc(bytes))) return nullptr;
        *cap = bytes;
    }
    return *buf;
}
}  // namespace

// The three operations on a device column-major A (ld lda), on the library
// stream; synchronous.  Return LAPACK's info (> 0) or a CHAMELEON_ERR_* code.
int trtri_dev(cham_uplo_t uplo, cham_diag_t diag, int N, double *A, int lda) {
    cudaStream_t s = ctx().stream;
    cublasHandle_t h = lib_handle();
    if (!h) return CHAMELEON_ERR_UNEXPECTED;
    if (!g_flag && !(g_flag = (int *)dev_alloc(sizeof(int)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    if (diag == ChamNonUnit) {
        const int none = INT_MAX;
        int first = INT_MAX;
        CHB_CUDA(cudaMemcpyAsync(g_flag, &none, sizeof(int), cudaMemcpyHostToDevice, s));
        zero_diag_kernel<<<grid_for(N), 256, 0, s>>>(A, lda, N, g_flag);
        CHB_LAUNCHED(1);
        CHB_CUDA(cudaMemcpyAsync(&first, g_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
        CHB_CUDA(cudaStreamSynchronize(s));
        if (first != INT_MAX) return first;   // singular: A is not modified
    }
    double *X = work(&g_w1, &g_w1_bytes, (size_t)N * N * sizeof(double));
    if (!X) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    identity_kernel<<<grid_for((int64_t)N * N), 256, 0, s>>>(X, N, N);
    CHB_LAUNCHED(1);
    const double one = 1.0;
    if (int rc = CUDA_dtrsm(ChamLeft, uplo, ChamNoTrans, diag, N, N, &one, A, lda, X, N, h)) return rc;
    tri_copy_kernel<<<grid_for((int64_t)N * N), 256, 0, s>>>(X, N, A, lda, N, uplo == ChamUpper, 0,
                                                             diag == ChamUnit);
    CHB_LAUNCHED(1);
    CHB_CUDA(cudaGetLastError());
    CHB_CUDA(cudaStreamSynchronize(s));
    return 0;
}

int lauum_dev(cham_uplo_t uplo, int N, double *A, int lda) {
    cudaStream_t s = ctx().stream;
    cublasHandle_t h = lib_handle();
    if (!h) return CHAMELEON_ERR_UNEXPECTED;
    double *T = work(&g_w1, &g_w1_bytes, (size_t)N * N * sizeof(double));
    double *C = work(&g_w2, &g_w2_bytes, (size_t)N * N * sizeof(double));
    if (!T || !C) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    tri_copy_kernel<<<grid_for((int64_t)N * N), 256, 0, s>>>(A, lda, T, N, N, uplo == ChamUpper, 1, 0);
    CHB_LAUNCHED(1);
    const double one = 1.0, zero = 0.0;
    // lower: L^T L; upper: U U^T
    const cham_trans_t ta = (uplo == ChamLower) ? ChamTrans : ChamNoTrans;
    const cham_trans_t tb = (uplo == ChamLower) ? ChamNoTrans : ChamTrans;
    if (int rc = CUDA_dgemm(ta, tb, N, N, N, &one, T, N, T, N, &zero, C, N, h)) return rc;
    tri_copy_kernel<<<grid_for((int64_t)N * N), 256, 0, s>>>(C, N, A, lda, N, uplo == ChamUpper, 0, 0);
    CHB_LAUNCHED(1);
    CHB_CUDA(cudaGetLastError());
    CHB_CUDA(cudaStreamSynchronize(s));
    return 0;
}

int potri_dev(cham_uplo_t uplo, int N, double *A, int lda) {
    if (int rc = trtri_dev(uplo, ChamNonUnit, N, A, lda)) return rc;
    return lauum_dev(uplo, N, A, lda);
}

// S (N x N, ld N) <- the symmetric matrix whose uplo triangle is in A.
__global__ void sym_full_kernel(const double *A, int64_t lda, double *S, int N, int upper) {
    const int64_t total = (int64_t)N * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % N), j = (int)(idx / N);
        const bool in = upper ? i <= j : i >= j;
        S[i + (int64_t)j * N] = in ? A[i + (int64_t)j * lda] : A[j + (int64_t)i * lda];
    }
}

// compute/pzpotrimm.c: A <- A^-1 (uplo triangle; A is the SPD matrix on
// entry: potrf, trtri, lauum), then C = B A^-1 (the symm of its last loop
// nest, alpha = 1, beta = 0).  Device arrays.
int potrimm_dev(cham_uplo_t uplo, int N, double *A, int lda, const double *B, int ldb, double *C, int ldc) {
    int rc = CHAMELEON_dpotrf(uplo, N, A, lda);
    if (rc) return rc;
    if ((rc = potri_dev(uplo, N, A, lda))) return rc;
    cudaStream_t s = ctx().stream;
    cublasHandle_t h = lib_handle();
    if (!h) return CHAMELEON_ERR_UNEXPECTED;
    double *S = work(&g_w1, &g_w1_bytes, (size_t)N * N * sizeof(double));
    if (!S) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    sym_full_kernel<<<grid_for((int64_t)N * N), 256, 0, s>>>(A, lda, S, N, uplo == ChamUpper);
    CHB_LAUNCHED(1);
    const double one = 1.0, zero = 0.0;
    if ((rc = CUDA_dgemm(ChamNoTrans, ChamNoTrans, N, N, N, &one, B, ldb, S, N, &zero, C, ldc, h))) return rc;
    CHB_CUDA(cudaGetLastError());
    CHB_CUDA(cudaStreamSynchronize(s));
    return 0;
}

// LAPACK layout: A on the host or the device.
enum InvOp { OP_TRTRI, OP_LAUUM, OP_POTRI };
int inverse_lapack(InvOp op, cham_uplo_t uplo, cham_diag_t diag, int N, double *A, int LDA) {
    cudaStream_t s = ctx().stream;
    cudaPointerAttributes at;
    bool dev = false;
    if (cudaPointerGetAttributes(&at, A) == cudaSuccess)
        dev = at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
    else
        cudaGetLastError();
    double *dA = A;
    int lda = LDA;
    if (!dev) {
        if (!(dA = stage_in(0, A, LDA, N, N, s))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        lda = N;
    }
    int rc = (op == OP_TRTRI) ? trtri_dev(uplo, diag, N, dA, lda)
                              : (op == OP_LAUUM) ? lauum_dev(uplo, N, dA, lda) : potri_dev(uplo, N, dA, lda);
    if (!dev && rc >= 0) {
        if (int r2 = stage_out(A, LDA, dA, N, N, s)) return r2;
        CHB_CUDA(cudaStreamSynchronize(s));
    }
    return rc;
}

// Tile layout: the descriptor's tiles <-> a dense device copy.
__global__ void tiles_dense_kernel(double *base, const int64_t *off, const int *ld, int mt, int mb, int nb, int N,
                                   double *D, int to_dense) {
    const int64_t total = (int64_t)N * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % N), j = (int)(idx / N);
        const int m = i / mb, n = j / nb;
        double *t = base + off[m + (int64_t)mt * n] + (i - m * mb) + (int64_t)(j - n * nb) * ld[m];
        if (to_dense) D[i + (int64_t)j * N] = *t;
        else *t = D[i + (int64_t)j * N];
    }
}

int inverse_tile(InvOp op, cham_uplo_t uplo, cham_diag_t diag, CHAM_desc_t *A) {
    if (!A || A->dtyp != ChamRealDouble || A->m != A->n || A->mb != A->nb) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const int N = A->n;
    if (N == 0) return 0;
    if (int rc = desc_upload(A)) return rc;
    cudaStream_t s = ctx().stream;
    double *D = staging(1, (size_t)N * N * sizeof(double));
    if (!D) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    const DescDev &dv = priv(A)->dev;
    tiles_dense_kernel<<<grid_for((int64_t)N * N), 256, 0, s>>>((double *)A->mat, dv.off, dv.ld, A->mt, A->mb, A->nb,
                                                                N, D, 1);
    CHB_LAUNCHED(1);
    int rc = (op == OP_TRTRI) ? trtri_dev(uplo, diag, N, D, N)
                              : (op == OP_LAUUM) ? lauum_dev(uplo, N, D, N) : potri_dev(uplo, N, D, N);
    if (rc == 0) {
        tiles_dense_kernel<<<grid_for((int64_t)N * N), 256, 0, s>>>((double *)A->mat, dv.off, dv.ld, A->mt, A->mb,
                                                                    A->nb, N, D, 0);
        CHB_LAUNCHED(1);
        CHB_CUDA(cudaStreamSynchronize(s));
        if (int r2 = desc_sync_to_host(A)) return r2;
    }
    return rc;
}

}  // namespace chb

using namespace chb;

extern "C" {

// compute/ztrtri.c:ztrtri (LAPACK layout)
int CHAMELEON_dtrtri(cham_uplo_t uplo, cham_diag_t diag, int N, double *A, int LDA) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (diag != ChamUnit && diag != ChamNonUnit) return -2;
    if (N < 0) return -3;
    if (LDA < std::max(1, N)) return -5;
    if (N == 0) return 0;
    return inverse_lapack(OP_TRTRI, uplo, diag, N, A, LDA);
}
int CHAMELEON_dlauum(cham_uplo_t uplo, int N, double *A, int LDA) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (N < 0) return -2;
    if (LDA < std::max(1, N)) return -4;
    if (N == 0) return 0;
    return inverse_lapack(OP_LAUUM, uplo, ChamNonUnit, N, A, LDA);
}
int CHAMELEON_dpotri(cham_uplo_t uplo, int N, double *A, int LDA) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (N < 0) return -2;
    if (LDA < std::max(1, N)) return -4;
    if (N == 0) return 0;
    return inverse_lapack(OP_POTRI, uplo, ChamNonUnit, N, A, LDA);
}
// compute/zpotrimm.c:72 (LAPACK layout): A, B, C host or device arrays.
int CHAMELEON_dpotrimm(cham_uplo_t uplo, int N, double *A, int LDA, double *B, int LDB, double *C, int LDC) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (N < 0) return -2;
    if (LDA < std::max(1, N)) return -4;
    if (LDB < std::max(1, N)) return -6;
    if (LDC < std::max(1, N)) return -8;
    if (N == 0) return 0;
    cudaStream_t s = ctx().stream;
    auto on_dev = [](const void *p) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
    };
    const bool da = on_dev(A), db = on_dev(B), dc = on_dev(C);
    double *dA = A, *dB = B, *dC = C;
    int lda = LDA, ldb = LDB, ldc = LDC;
    if (!da) {
        if (!(dA = stage_in(0, A, LDA, N, N, s))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        lda = N;
    }
    if (!db) {
        if (!(dB = work(&g_w3, &g_w3_bytes, (size_t)N * N * sizeof(double)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        CHB_CUDA(cudaMemcpy2DAsync(dB, (size_t)N * sizeof(double), B, (size_t)LDB * sizeof(double),
                                   (size_t)N * sizeof(double), N, cudaMemcpyHostToDevice, s));
        ldb = N;
    }
    if (!dc) {
        if (!(dC = work(&g_w4, &g_w4_bytes, (size_t)N * N * sizeof(double)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        ldc = N;
    }
    rc = potrimm_dev(uplo, N, dA, lda, dB, ldb, dC, ldc);
    if (rc >= 0) {
        if (!da)
            if (int r2 = stage_out(A, LDA, dA, N, N, s)) return r2;
        if (!dc && rc == 0)
            CHB_CUDA(cudaMemcpy2DAsync(C, (size_t)LDC * sizeof(double), dC, (size_t)N * sizeof(double),
                                       (size_t)N * sizeof(double), N, cudaMemcpyDeviceToHost, s));
        CHB_CUDA(cudaStreamSynchronize(s));
    }
    return rc;
}

// compute/zpotrimm.c:202 (tile layout): square descriptors of one order.
int CHAMELEON_dpotrimm_Tile(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B, CHAM_desc_t *C) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    for (CHAM_desc_t *d : {A, B, C})
        if (!d || d->dtyp != ChamRealDouble || d->m != d->n || d->mb != d->nb) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (B->n != A->n || C->n != A->n) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const int N = A->n;
    if (N == 0) return 0;
    cudaStream_t s = ctx().stream;
    double *DA = staging(1, (size_t)N * N * sizeof(double));
    double *DB = work(&g_w3, &g_w3_bytes, (size_t)N * N * sizeof(double));
    double *DC = work(&g_w4, &g_w4_bytes, (size_t)N * N * sizeof(double));
    if (!DA || !DB || !DC) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    for (CHAM_desc_t *d : {A, B, C})
        if ((rc = desc_upload(d))) return rc;
    auto conv = [&](CHAM_desc_t *d, double *D, int to_dense) {
        const DescDev &dv = priv(d)->dev;
        tiles_dense_kernel<<<grid_for((int64_t)N * N), 256, 0, s>>>((double *)d->mat, dv.off, dv.ld, d->mt, d->mb,
                                                                    d->nb, N, D, to_dense);
        CHB_LAUNCHED(1);
    };
    conv(A, DA, 1);
    conv(B, DB, 1);
    rc = potrimm_dev(uplo, N, DA, N, DB, N, DC, N);
    if (rc == 0) {
        conv(A, DA, 0);
        conv(C, DC, 0);
        CHB_CUDA(cudaStreamSynchronize(s));
        if (int r2 = desc_sync_to_host(A)) return r2;
        if (int r2 = desc_sync_to_host(C)) return r2;
    }
    return rc;
}

int CHAMELEON_dtrtri_Tile(cham_uplo_t uplo, cham_diag_t diag, CHAM_desc_t *A) {
    int rc = ensure_init();
    if (rc) return rc;
    if ((uplo != ChamUpper && uplo != ChamLower) || (diag != ChamUnit && diag != ChamNonUnit))
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    return inverse_tile(OP_TRTRI, uplo, diag, A);
}
int CHAMELEON_dlauum_Tile(cham_uplo_t uplo, CHAM_desc_t *A) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    return inverse_tile(OP_LAUUM, uplo, ChamNonUnit, A);
}
int CHAMELEON_dpotri_Tile(cham_uplo_t uplo, CHAM_desc_t *A) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    return inverse_tile(OP_POTRI, uplo, ChamNonUnit, A);
}

// ---- LAPACKE interface (lapack_api/src/lapack_z*.c after z->d) -------------
// The character arguments convert as lapack_api/src/lapack_api_common.c does:
// an illegal one prints the message and becomes CHAMELEON_ERR_ILLEGAL_VALUE,
// which the routine behind it then rejects with its own argument index.
static int lapacke_uplo(char c) {
    if (c == 'U' || c == 'u') return ChamUpper;
    if (c == 'L' || c == 'l') return ChamLower;
    fprintf(stderr, "CHAMELEON ERROR: %s(): %s\n", "chameleon_blastocblas_uplo",
            "illegal value of BLAS uplo parameter");
    return CHAMELEON_ERR_ILLEGAL_VALUE;
}
static int lapacke_diag(char c) {
    if (c == 'U' || c == 'u') return ChamUnit;
    if (c == 'N' || c == 'n') return ChamNonUnit;
    fprintf(stderr, "CHAMELEON ERROR: %s(): %s\n", "chameleon_blastocblas_diag",
            "illegal value of BLAS diag parameter");
    return CHAMELEON_ERR_ILLEGAL_VALUE;
}
#define CHB_LAPACKE_PROLOGUE(name)                                                                   \
    if (matrix_layout != CHAMELEON_LAPACK_COL_MAJOR) {                                               \
        fprintf(stderr, "CHAMELEON ERROR: %s(): %s\n", name, "illegal value of matrix_layout");      \
        return -1;                                                                                   \
    }                                                                                                \
    const int ul = lapacke_uplo(uplo);

int CHAMELEON_lapacke_dposv(int matrix_layout, char uplo, int N, int NRHS, double *A, int lda, double *B, int ldb) {
    CHB_LAPACKE_PROLOGUE("CHAMELEON_lapacke_dposv");
    return CHAMELEON_dposv((cham_uplo_t)ul, N, NRHS, A, lda, B, ldb);
}
int CHAMELEON_lapacke_dpotrf(int matrix_layout, char uplo, int N, double *A, int lda) {
    CHB_LAPACKE_PROLOGUE("CHAMELEON_lapacke_dpotrf");
    return CHAMELEON_dpotrf((cham_uplo_t)ul, N, A, lda);
}
int CHAMELEON_lapacke_dpotrs(int matrix_layout, char uplo, int N, int NRHS, const double *A, int lda, double *B,
                             int ldb) {
    CHB_LAPACKE_PROLOGUE("CHAMELEON_lapacke_dpotrs");
    return CHAMELEON_dpotrs((cham_uplo_t)ul, N, NRHS, const_cast<double *>(A), lda, B, ldb);
}
int CHAMELEON_lapacke_dpotri(int matrix_layout, char uplo, int N, double *A, int lda) {
    CHB_LAPACKE_PROLOGUE("CHAMELEON_lapacke_dpotri");
    return CHAMELEON_dpotri((cham_uplo_t)ul, N, A, lda);
}
int CHAMELEON_lapacke_dlauum(int matrix_layout, char uplo, int N, double *A, int lda) {
    CHB_LAPACKE_PROLOGUE("CHAMELEON_lapacke_dlauum");
    return CHAMELEON_dlauum((cham_uplo_t)ul, N, A, lda);
}
int CHAMELEON_lapacke_dtrtri(int matrix_layout, char uplo, char diag, int N, double *A, int lda) {
    CHB_LAPACKE_PROLOGUE("CHAMELEON_lapacke_dtrtri");
    const int dg = lapacke_diag(diag);
    return CHAMELEON_dtrtri((cham_uplo_t)ul, (cham_diag_t)dg, N, A, lda);
}

// ---- Fortran LAPACK interface (gfortran names: lower case, trailing _) ----
void chameleon_lapack_dposv_(const char *uplo, const int *n, const int *nrhs, double *a, const int *lda, double *b,
                             const int *ldb, int *info) {
    *info = CHAMELEON_lapacke_dposv(CHAMELEON_LAPACK_COL_MAJOR, *uplo, *n, *nrhs, a, *lda, b, *ldb);
}
void chameleon_lapack_dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info) {
    *info = CHAMELEON_lapacke_dpotrf(CHAMELEON_LAPACK_COL_MAJOR, *uplo, *n, a, *lda);
}
void chameleon_lapack_dpotrs_(const char *uplo, const int *n, const int *nrhs, const double *a, const int *lda,
                              double *b, const int *ldb, int *info) {
    *info = CHAMELEON_lapacke_dpotrs(CHAMELEON_LAPACK_COL_MAJOR, *uplo, *n, *nrhs, a, *lda, b, *ldb);
}
void chameleon_lapack_dpotri_(const char *uplo, const int *n, double *a, const int *lda, int *info) {
    *info = CHAMELEON_lapacke_dpotri(CHAMELEON_LAPACK_COL_MAJOR, *uplo, *n, a, *lda);
}
void chameleon_lapack_dlauum_(const char *uplo, const int *n, double *a, const int *lda, int *info) {
    *info = CHAMELEON_lapacke_dlauum(CHAMELEON_LAPACK_COL_MAJOR, *uplo, *n, a, *lda);
}
void chameleon_lapack_dtrtri_(const char *uplo, const char *diag, const int *n, double *a, const int *lda, int *info) {
    *info = CHAMELEON_lapacke_dtrtri(CHAMELEON_LAPACK_COL_MAJOR, *uplo, *diag, *n, a, *lda);
}

}  // extern "C"
