// tile_abi.cu -- the gpucublas tile-kernel C ABI (gpucublas/include/gpucublas/
// gpucublas_z.h:36-61, gpucublas_zc.h:22-23 after generation), on this
// library's own sm_100a kernels.  The reference forwards each call to cuBLAS /
// cuSOLVER (gpucublas/compute/cuda_zgemm.c:24-45, cuda_zsyrk.c:24-43,
// cuda_ztrsm.c:24-44, cuda_zpotrf.c:23-50); here every call is one launch of a
// kernel built from core.cuh on the handle's stream.  Scalars are host
// pointers (cuBLAS host pointer mode, as the reference uses them).
#include <cuda_runtime.h>
#include <stdlib.h>

#include <algorithm>

#include "core.cuh"
#include "potrf_smem.cuh"
#include "rec.cuh"
#include "gen.cuh"
#include "internal.h"

struct cham_b200_handle_s {
    cudaStream_t stream;
    double *ws;          // scratch: inverted diagonal blocks (grown on demand)
    size_t ws_bytes;
    int *flag;           // dlag2s overflow flag (device)
};

namespace chb {

static int handle_ws(cham_b200_handle_s *h, size_t bytes) {
    if (bytes <= h->ws_bytes) return 0;
    if (h->ws) cudaFree(h->ws);
    h->ws = nullptr;
    h->ws_bytes = 0;
    CHB_CUDA(cudaMalloc(&h->ws, bytes));
    h->ws_bytes = bytes;
    return 0;
}

// C = alpha * sum_k A(i,k) B(j,k) + beta * C over one 128 x 128 block.
__global__ void __launch_bounds__(NT_CTA, 1) gemm_kernel(View A, View B, View C, int M, int N, int K, double alpha,
                                                         double beta, int tri /*0 full, 1 lower, 2 upper*/) {
    extern __shared__ __align__(128) double smem[];
    const int bi = blockIdx.x, bj = blockIdx.y;
    if (tri == 1 && bj > bi) return;
    if (tri == 2 && bi > bj) return;
    const int i0 = bi * 128, j0 = bj * 128;
    const int rows = min(128, M - i0), cols = min(128, N - j0);
    Acc<Cfg128<double>> acc;
    acc.zero();
    cta_gemm(acc, A.sub(i0, 0), B.sub(j0, 0), rows, cols, K, smem);
    const View Cb = C.sub(i0, j0);
    const bool diag = (tri != 0) && bi == bj;
    acc.for_each([&](int r, int c, double v) {
        if (r >= rows || c >= cols) return;
        if (diag && ((tri == 1 && r < c) || (tri == 2 && r > c))) return;
        double *p = Cb.at(r, c);
        *p = (beta == 0.0) ? alpha * v : alpha * v + beta * *p;
    });
}

__global__ void scale_kernel(View X, int M, int N, double alpha) {
    const int64_t total = (int64_t)M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        double *p = X.at(i, j);
        *p = (alpha == 0.0) ? 0.0 : alpha * *p;
    }
}

// Invert the IB x IB diagonal blocks of lower-triangular L (n x n) into invd.
__global__ void __launch_bounds__(NT_CTA, 1) inv_diag_kernel(View L, int n, double *invd, int unit) {
    extern __shared__ __align__(128) double smem[];
    double *sD = smem;
    double *sInv = smem + IB * LDD;
    const int jb = blockIdx.x * IB;
    const int nbk = min(IB, n - jb);
    for (int idx = threadIdx.x; idx < nbk * nbk; idx += NT_CTA) {
        const int r = idx % nbk, c = idx / nbk;
        sD[r + c * LDD] = (r >= c) ? *L.at(jb + r, jb + c) : 0.0;
    }
    __syncthreads();
    blk_inv(sD, sInv, nbk, unit != 0);
    store_inv(invd + (int64_t)blockIdx.x * IB * IB, sInv);
}

// X <- op(L)^{-1} X on column strips of IB.
__global__ void __launch_bounds__(NT_CTA, 1) trsm_kernel(View L, int n, const double *invd, View X, int w,
                                                         int trans) {
    extern __shared__ __align__(128) double smem[];
    const int c0 = blockIdx.x * IB;
    trsm_left<double, SPLIT_BF16X3>(X.sub(0, c0), min(IB, w - c0), L, n, invd, trans != 0, smem);
}

__global__ void __launch_bounds__(NT_CTA, 1) potrf_kernel(View T, int n, double *invd, int *info) {
    extern __shared__ __align__(128) double smem[];
    const int r = rec::tile_potrf_blk<double, SPLIT_BF16X3>(T, n, invd, smem);
    if (threadIdx.x == 0 && info) *info = r;
}

// FP32 tile Cholesky: the shared-memory kernel of the executor's diagonal
// tiles for n <= 256, the blocked one (BF16x3 GEMMs) above.
constexpr size_t SPOTRF_SMEM_BYTES =
    psm::SMEM_BYTES > tile_smem_bytes<float>() ? psm::SMEM_BYTES : tile_smem_bytes<float>();
__global__ void __launch_bounds__(NT_CTA, 1) spotrf_kernel(ViewF T, int n, float *invd, int *info) {
    extern __shared__ __align__(128) float fsm[];
    const int r = (n <= psm::MAXN) ? psm::potrf(T, n, invd, fsm)
                                   : rec::tile_potrf_blk<float, SPLIT_BF16X3>(T, n, invd, fsm);
    if (threadIdx.x == 0 && info) *info = r;
}

__global__ void plgsy_tile_kernel(double *A, int lda, int M, int N, double bump, int bigM, int m0, int n0,
                                  unsigned long long seed) {
    const int64_t total = (int64_t)M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        const long long gi = (long long)i + m0, gj = (long long)j + n0;
        unsigned long long pos;
        if (gi >= gj) pos = (unsigned long long)gi + (unsigned long long)gj * (unsigned long long)bigM;
        else pos = (unsigned long long)gj + (unsigned long long)gi * (unsigned long long)bigM;
        double v = lcg_value(lcg_skip(pos, seed));
        if (gi == gj) v = __dadd_rn(v, bump);
        A[i + (int64_t)j * lda] = v;
    }
}

__global__ void plrnt_tile_kernel(double *A, int lda, int M, int N, int bigM, int m0, int n0,
                                  unsigned long long seed) {
    const int64_t total = (int64_t)M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        const unsigned long long pos =
            (unsigned long long)(i + m0) + (unsigned long long)(j + n0) * (unsigned long long)bigM;
        A[i + (int64_t)j * lda] = lcg_value(lcg_skip(pos, seed));
    }
}

// dlag2s: FP64 -> FP32 with LAPACK's overflow rule (|a| > FLT_MAX sets the
// flag; NaN does not); the reference's GPU kernel (gpucublas/compute/
// cuda_zlag2c.cu:38-106) tests `ind > m` where `ind >= m` is meant and never
// reports its flag; here rows are bounded by `m` and the flag is kept in the
// handle.  Both casts run column-blocked (blockIdx.y strides the columns, so
// no division per element) with 4 rows per thread: two 16-byte FP64 accesses
// and one 16-byte FP32 access where the column pointers allow it.
constexpr double kFltMax = 3.4028234663852886e38;

__device__ __forceinline__ bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

__global__ void dlag2s_kernel(const double *A, int lda, float *SA, int ldsa, int M, int N, int *flag) {
    bool ovf = false;
    for (int j = blockIdx.y; j < N; j += gridDim.y) {
        const double *a = A + (int64_t)j * lda;
        float *sa = SA + (int64_t)j * ldsa;
        const bool vec = aligned16(a) && aligned16(sa);
        for (int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4; i0 < M; i0 += gridDim.x * blockDim.x * 4) {
            if (vec && i0 + 3 < M) {
                const double2 x = *reinterpret_cast<const double2 *>(a + i0);
                const double2 y = *reinterpret_cast<const double2 *>(a + i0 + 2);
                ovf |= fabs(x.x) > kFltMax || fabs(x.y) > kFltMax || fabs(y.x) > kFltMax || fabs(y.y) > kFltMax;
                *reinterpret_cast<float4 *>(sa + i0) =
                    make_float4(__double2float_rn(x.x), __double2float_rn(x.y), __double2float_rn(y.x),
                                __double2float_rn(y.y));
            } else {
                for (int i = i0; i < min(i0 + 4, M); ++i) {
                    const double v = a[i];
                    ovf |= fabs(v) > kFltMax;
                    sa[i] = __double2float_rn(v);
                }
            }
        }
    }
    if (ovf) *flag = 1;
}

__global__ void slag2d_kernel(const float *SA, int ldsa, double *A, int lda, int M, int N) {
    for (int j = blockIdx.y; j < N; j += gridDim.y) {
        const float *sa = SA + (int64_t)j * ldsa;
        double *a = A + (int64_t)j * lda;
        const bool vec = aligned16(a) && aligned16(sa);
        for (int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4; i0 < M; i0 += gridDim.x * blockDim.x * 4) {
            if (vec && i0 + 3 < M) {
                const float4 x = *reinterpret_cast<const float4 *>(sa + i0);
                *reinterpret_cast<double2 *>(a + i0) = make_double2(x.x, x.y);
                *reinterpret_cast<double2 *>(a + i0 + 2) = make_double2(x.z, x.w);
            } else {
                for (int i = i0; i < min(i0 + 4, M); ++i) a[i] = (double)sa[i];
            }
        }
    }
}

// Column-blocked grid of the casts: x covers the rows (1024 per block), y the
// columns, about 16 blocks of 256 threads per SM in all.
static dim3 cast_grid(int m, int n) {
    const int gx = std::max(1, std::min((m + 1023) / 1024, 148 * 16));
    const int gy = std::max(1, std::min({n, 65535, std::max(1, 148 * 16 / gx)}));
    return dim3(gx, gy);
}

static int ew_grid(int64_t total) {
    const int64_t b = (total + 255) / 256;
    return (int)std::min<int64_t>(std::max<int64_t>(b, 1), 148 * 32);
}

static bool smem_attr_done = false;
static int set_smem_attrs() {
    if (smem_attr_done) return 0;
    CHB_CUDA(cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg128<double>::SMEM_BYTES));
    CHB_CUDA(cudaFuncSetAttribute(trsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg64<double>::SMEM_BYTES));
    CHB_CUDA(cudaFuncSetAttribute(potrf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)TILE_KERNEL_SMEM_BYTES));
    CHB_CUDA(cudaFuncSetAttribute(spotrf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)SPOTRF_SMEM_BYTES));
    CHB_CUDA(cudaFuncSetAttribute(inv_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * IB * LDD * sizeof(double))));
    smem_attr_done = true;
    return 0;
}

}  // namespace chb

using namespace chb;

extern "C" {

int CHAM_B200_Handle_Create(cublasHandle_t *handle, void *cuda_stream) {
    if (!handle) return CHAMELEON_ERR_ILLEGAL_VALUE;
    cham_b200_handle_s *h = (cham_b200_handle_s *)calloc(1, sizeof(cham_b200_handle_s));
    h->stream = (cudaStream_t)cuda_stream;
    if (cudaMalloc(&h->flag, sizeof(int)) != cudaSuccess) {
        free(h);
        return CHAMELEON_ERR_OUT_OF_RESOURCES;
    }
    cudaMemset(h->flag, 0, sizeof(int));
    *handle = h;
    return 0;
}

int CHAM_B200_Handle_Destroy(cublasHandle_t h) {
    if (!h) return CHAMELEON_ERR_UNALLOCATED;
    cudaStreamSynchronize(h->stream);
    if (h->ws) cudaFree(h->ws);
    if (h->flag) cudaFree(h->flag);
    free(h);
    return 0;
}

// Reads (and clears) the dlag2s overflow flag of the handle; synchronizes its stream.
int CHAM_B200_Handle_Overflow(cublasHandle_t h) {
    int v = 0;
    cudaMemcpyAsync(&v, h->flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream);
    cudaStreamSynchronize(h->stream);
    return v;
}

int CUDA_dgemm(cham_trans_t transa, cham_trans_t transb, int m, int n, int k, const double *alpha,
               const double *A, int lda, const double *B, int ldb, const double *beta, double *C, int ldc,
               cublasHandle_t handle) {
    if (!handle || !alpha || !beta) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (transa < ChamNoTrans || transa > ChamConjTrans) return -1;
    if (transb < ChamNoTrans || transb > ChamConjTrans) return -2;
    if (m < 0) return -3;
    if (n < 0) return -4;
    if (k < 0) return -5;
    if (m == 0 || n == 0) return 0;
    if (int rc = set_smem_attrs()) return rc;
    const View Av = (transa == ChamNoTrans) ? View{const_cast<double *>(A), 1, lda} : View{const_cast<double *>(A), lda, 1};
    const View Bv = (transb == ChamNoTrans) ? View{const_cast<double *>(B), ldb, 1} : View{const_cast<double *>(B), 1, ldb};
    const View Cv{C, 1, ldc};
    if (k == 0 || *alpha == 0.0) {
        scale_kernel<<<ew_grid((int64_t)m * n), 256, 0, handle->stream>>>(Cv, m, n, *beta);
    } else {
        dim3 grid((m + 127) / 128, (n + 127) / 128);
        gemm_kernel<<<grid, NT_CTA, Cfg128<double>::SMEM_BYTES, handle->stream>>>(Av, Bv, Cv, m, n, k, *alpha, *beta, 0);
    }
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}

int CUDA_dsyrk(cham_uplo_t uplo, cham_trans_t trans, int n, int k, const double *alpha, const double *A, int lda,
               const double *beta, double *C, int ldc, cublasHandle_t handle) {
    if (!handle || !alpha || !beta) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (trans < ChamNoTrans || trans > ChamConjTrans) return -2;
    if (n < 0) return -3;
    if (k < 0) return -4;
    if (n == 0) return 0;
    if (int rc = set_smem_attrs()) return rc;
    const View Av = (trans == ChamNoTrans) ? View{const_cast<double *>(A), 1, lda} : View{const_cast<double *>(A), lda, 1};
    dim3 grid((n + 127) / 128, (n + 127) / 128);
    const View Cv{C, 1, ldc};
    gemm_kernel<<<grid, NT_CTA, Cfg128<double>::SMEM_BYTES, handle->stream>>>(Av, Av, Cv, n, n, k, (k == 0) ? 0.0 : *alpha,
                                                                     *beta, uplo == ChamLower ? 1 : 2);
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}

int CUDA_dtrsm(cham_side_t side, cham_uplo_t uplo, cham_trans_t transa, cham_diag_t diag, int m, int n,
               const double *alpha, const double *A, int lda, double *B, int ldb, cublasHandle_t handle) {
    if (!handle || !alpha) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (side != ChamLeft && side != ChamRight) return -1;
    if (uplo != ChamUpper && uplo != ChamLower) return -2;
    if (transa < ChamNoTrans || transa > ChamConjTrans) return -3;
    if (diag != ChamNonUnit && diag != ChamUnit) return -4;
    if (m < 0) return -5;
    if (n < 0) return -6;
    if (m == 0 || n == 0) return 0;
    if (int rc = set_smem_attrs()) return rc;
    const bool tr = (transa != ChamNoTrans), up = (uplo == ChamUpper);
    const View L = up ? View{const_cast<double *>(A), lda, 1} : View{const_cast<double *>(A), 1, lda};
    const bool left = (side == ChamLeft);
    const bool trans_eff = left ? (tr != up) : (!tr != up);
    const View X = left ? View{B, 1, ldb} : View{B, ldb, 1};
    const int ns = left ? m : n, w = left ? n : m;
    const int nblk = (ns + IB - 1) / IB;
    if (int rc = handle_ws(handle, (size_t)nblk * IB * IB * sizeof(double))) return rc;
    if (*alpha != 1.0) scale_kernel<<<ew_grid((int64_t)ns * w), 256, 0, handle->stream>>>(X, ns, w, *alpha);
    inv_diag_kernel<<<nblk, NT_CTA, 2 * IB * LDD * sizeof(double), handle->stream>>>(L, ns, handle->ws,
                                                                                     diag == ChamUnit);
    trsm_kernel<<<(w + IB - 1) / IB, NT_CTA, Cfg64<double>::SMEM_BYTES, handle->stream>>>(L, ns, handle->ws, X, w,
                                                                                 trans_eff);
    CHB_LAUNCHED(3);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}

int CUDA_dpotrf(cham_uplo_t uplo, int n, double *A, int lda, double *WORK, int lwork, int *d_info,
                cusolverDnHandle_t handle) {
    (void)WORK;
    (void)lwork;
    if (!handle) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (n < 0) return -2;
    if (lda < std::max(1, n)) return -4;
    if (n == 0) {
        if (d_info) cudaMemsetAsync(d_info, 0, sizeof(int), handle->stream);
        return 0;
    }
    if (int rc = set_smem_attrs()) return rc;
    const int nblk = (n + IB - 1) / IB;
    if (int rc = handle_ws(handle, (size_t)nblk * IB * IB * sizeof(double))) return rc;
    const View T = (uplo == ChamLower) ? View{A, 1, lda} : View{A, lda, 1};
    potrf_kernel<<<1, NT_CTA, TILE_KERNEL_SMEM_BYTES, handle->stream>>>(T, n, handle->ws, d_info);
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}

int CUDA_spotrf(cham_uplo_t uplo, int n, float *A, int lda, float *WORK, int lwork, int *d_info,
                cusolverDnHandle_t handle) {
    (void)WORK;
    (void)lwork;
    if (!handle) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (n < 0) return -2;
    if (lda < std::max(1, n)) return -4;
    if (n == 0) {
        if (d_info) cudaMemsetAsync(d_info, 0, sizeof(int), handle->stream);
        return 0;
    }
    if (int rc = set_smem_attrs()) return rc;
    const int nblk = (n + IB - 1) / IB;
    if (int rc = handle_ws(handle, (size_t)nblk * IB * IB * sizeof(float))) return rc;
    const ViewF T = (uplo == ChamLower) ? ViewF{A, 1, lda} : ViewF{A, lda, 1};
    spotrf_kernel<<<1, NT_CTA, SPOTRF_SMEM_BYTES, handle->stream>>>(T, n, reinterpret_cast<float *>(handle->ws),
                                                                    d_info);
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}

int CUDA_dplgsy(const double *bump, int m, int n, double *A, int lda, int bigM, int m0, int n0,
                unsigned long long int seed, cublasHandle_t handle) {
    if (!handle || !bump) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (m <= 0 || n <= 0) return 0;
    plgsy_tile_kernel<<<ew_grid((int64_t)m * n), 256, 0, handle->stream>>>(A, lda, m, n, *bump, bigM, m0, n0, seed);
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}

int CUDA_dplrnt(int m, int n, double *A, int lda, int bigM, int m0, int n0, unsigned long long int seed,
                cublasHandle_t handle) {
    if (!handle) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (m <= 0 || n <= 0) return 0;
    plrnt_tile_kernel<<<ew_grid((int64_t)m * n), 256, 0, handle->stream>>>(A, lda, m, n, bigM, m0, n0, seed);
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}

int CUDA_dlag2s(int m, int n, const double *A, int lda, float *SA, int ldsa, cublasHandle_t handle) {
    if (!handle) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (m < 0) return -1;
    if (n < 0) return -2;
    if (lda < std::max(1, m)) return -4;
    if (ldsa < std::max(1, m)) return -6;
    if (m == 0 || n == 0) return 0;
    dlag2s_kernel<<<cast_grid(m, n), 256, 0, handle->stream>>>(A, lda, SA, ldsa, m, n, handle->flag);
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}

int CUDA_slag2d(int m, int n, const float *SA, int ldsa, double *A, int lda, cublasHandle_t handle) {
    if (!handle) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (m < 0) return -1;
    if (n < 0) return -2;
    if (ldsa < std::max(1, m)) return -4;
    if (lda < std::max(1, m)) return -6;
    if (m == 0 || n == 0) return 0;
    slag2d_kernel<<<cast_grid(m, n), 256, 0, handle->stream>>>(SA, ldsa, A, lda, m, n);
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}


// ---- tile forms (gpucublas_ztile.h): tile -> address + leading dimension ----
static bool full_rank(const CHAM_tile_t *t) { return t && t->mat && (t->format & CHAMELEON_TILE_FULLRANK); }

int TCUDA_dgemm(cham_trans_t transA, cham_trans_t transB, int m, int n, int k, const double *alpha,
                const CHAM_tile_t *A, const CHAM_tile_t *B, const double *beta, CHAM_tile_t *C,
                cublasHandle_t handle) {
    if (!full_rank(A) || !full_rank(B) || !full_rank(C)) return CHAMELEON_ERR_NOT_SUPPORTED;
    return CUDA_dgemm(transA, transB, m, n, k, alpha, (const double *)A->mat, A->ld, (const double *)B->mat, B->ld,
                      beta, (double *)C->mat, C->ld, handle);
}
int TCUDA_dsyrk(cham_uplo_t uplo, cham_trans_t trans, int n, int k, const double *alpha, const CHAM_tile_t *A,
                const double *beta, CHAM_tile_t *C, cublasHandle_t handle) {
    if (!full_rank(A) || !full_rank(C)) return CHAMELEON_ERR_NOT_SUPPORTED;
    return CUDA_dsyrk(uplo, trans, n, k, alpha, (const double *)A->mat, A->ld, beta, (double *)C->mat, C->ld, handle);
}
int TCUDA_dtrsm(cham_side_t side, cham_uplo_t uplo, cham_trans_t transA, cham_diag_t diag, int m, int n,
                const double *alpha, const CHAM_tile_t *A, CHAM_tile_t *B, cublasHandle_t handle) {
    if (!full_rank(A) || !full_rank(B)) return CHAMELEON_ERR_NOT_SUPPORTED;
    return CUDA_dtrsm(side, uplo, transA, diag, m, n, alpha, (const double *)A->mat, A->ld, (double *)B->mat, B->ld,
                      handle);
}
int TCUDA_dpotrf(cham_uplo_t uplo, int n, CHAM_tile_t *A, double *WORK, int lwork, int *d_info,
                 cusolverDnHandle_t handle) {
    if (!full_rank(A)) return CHAMELEON_ERR_NOT_SUPPORTED;
    return CUDA_dpotrf(uplo, n, (double *)A->mat, A->ld, WORK, lwork, d_info, handle);
}
int TCUDA_dplgsy(const double *bump, int m, int n, CHAM_tile_t *A, int bigM, int m0, int n0,
                 unsigned long long int seed, cublasHandle_t handle) {
    if (!full_rank(A)) return CHAMELEON_ERR_NOT_SUPPORTED;
    return CUDA_dplgsy(bump, m, n, (double *)A->mat, A->ld, bigM, m0, n0, seed, handle);
}
int TCUDA_dplrnt(int m, int n, CHAM_tile_t *A, int bigM, int m0, int n0, unsigned long long int seed,
                 cublasHandle_t handle) {
    if (!full_rank(A)) return CHAMELEON_ERR_NOT_SUPPORTED;
    return CUDA_dplrnt(m, n, (double *)A->mat, A->ld, bigM, m0, n0, seed, handle);
}
int TCUDA_dlag2s(int m, int n, const CHAM_tile_t *A, CHAM_tile_t *B, cublasHandle_t handle) {
    if (!full_rank(A) || !full_rank(B)) return CHAMELEON_ERR_NOT_SUPPORTED;
    return CUDA_dlag2s(m, n, (const double *)A->mat, A->ld, (float *)B->mat, B->ld, handle);
}
int TCUDA_slag2d(int m, int n, const CHAM_tile_t *A, CHAM_tile_t *B, cublasHandle_t handle) {
    if (!full_rank(A) || !full_rank(B)) return CHAMELEON_ERR_NOT_SUPPORTED;
    return CUDA_slag2d(m, n, (const float *)A->mat, A->ld, (double *)B->mat, B->ld, handle);
}

}  // extern "C"
