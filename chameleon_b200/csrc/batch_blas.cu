// batch_blas.cu -- batched tile GEMM and SYRK: one independent product per tile.
//
// Reference: CHAMELEON_zgemm_batch_Tile (compute/zgemm_batch.c:154-230) and
// CHAMELEON_zherk_batch_Tile (compute/zherk_batch.c:176-215; zherk -> dsyrk
// in real arithmetic) map one TCORE/CUDA call per tile (m, n) through
// chameleon_pmap:
//   gemm: C(m,n) <- alpha op(A(m,n)) op(B(m,n)) + beta C(m,n), the tile's
//         sizes from C's tile (m, n) and K = A's tile columns (NoTrans) or
//         rows (Trans) at that position;
//   syrk: C(m,n) <- alpha op(A(m,n)) op(A(m,n))^T + beta C(m,n) on the uplo
//         triangle of the tile, N = C's tile columns, K likewise from A.
// Here all tiles go to ONE persistent launch: every 128 x 128 block of every
// C tile (for SYRK, only the blocks that meet the uplo triangle) is an item;
// CTAs take items in turn and run the FP64 tensor-core block product (the
// executor's cta_gemm, DMMA) with an alpha/beta epilogue that reads C only
// when beta != 0 (BLAS: C need not be set when beta is zero).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "core.cuh"
#include "internal.h"

namespace chb {

struct BlasItem {
    int64_t a_off, b_off, c_off;
    int lda, ldb, ldc;
    int rows, cols, k;   // of this 128 x 128 block of C (rows, cols <= 128)
    int r0, c0;          // block origin inside its C tile
};

// trans bits: 1 = op(A) transposed, 2 = op(B) transposed.  syrk: B is A,
// op(B) = op(A)^T, so the B view is op(A) too; uplo: 1 lower, 2 upper, 0 full.
__global__ void __launch_bounds__(NT_CTA, 1)
    blas_batch_kernel(const BlasItem *items, int count, const double *A, const double *B, double *C, int trans,
                      int syrk, int uplo, double alpha, double beta) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double *smem = reinterpret_cast<double *>(smem_raw);
    using Cfg = Cfg128<double, SPLIT_BF16X3>;
    for (int i = blockIdx.x; i < count; i += gridDim.x) {
        const BlasItem it = items[i];
        const double *a = A + it.a_off;
        // op(A)(i, k) and the B operand as (j, k) = op(B)(k, j)
        ViewT<double> Va = (trans & 1) ? ViewT<double>{const_cast<double *>(a), it.lda, 1}
                                       : ViewT<double>{const_cast<double *>(a), 1, it.lda};
        ViewT<double> Vb;
        if (syrk) {
            Vb = Va;
        } else {
            const double *b = B + it.b_off;
            Vb = (trans & 2) ? ViewT<double>{const_cast<double *>(b), 1, it.ldb}
                             : ViewT<double>{const_cast<double *>(b), it.ldb, 1};
        }
        Acc<Cfg> acc;
        acc.zero();
        cta_gemm(acc, Va.sub(it.r0, 0), Vb.sub(it.c0, 0), it.rows, it.cols, it.k, smem);
        const ViewT<double> Cv{C + it.c_off + it.r0 + (int64_t)it.c0 * it.ldc, 1, it.ldc};
        acc.for_each([&](int r, int c, double v) {
            if (r >= it.rows || c >= it.cols) return;
            const int gr = it.r0 + r, gc = it.c0 + c;
            if ((uplo == 1 && gr < gc) || (uplo == 2 && gr > gc)) return;
            double *p = Cv.at(r, c);
            *p = (beta == 0.0) ? alpha * v : alpha * v + beta * *p;
        });
        cta_sync();
    }
}

namespace {

bool g_blas_attr = false;

int launch_blas_batch(const std::vector<BlasItem> &items, const double *A, const double *B, double *C, int trans,
                      int syrk, int uplo, double alpha, double beta) {
    if (items.empty()) return 0;
    if (!g_blas_attr) {
        CHB_CUDA(cudaFuncSetAttribute(blas_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)Cfg128<double, SPLIT_BF16X3>::SMEM_BYTES));
        g_blas_attr = true;
    }
    cudaStream_t s = ctx().stream;
    if (int rc = bws_reserve(g_bws, items.size() * sizeof(BlasItem), 0, 0)) return rc;
    CHB_CUDA(cudaMemcpyAsync(g_bws.items, items.data(), items.size() * sizeof(BlasItem), cudaMemcpyHostToDevice, s));
    const int grid = (int)std::min<size_t>(items.size(), (size_t)ctx().num_sms);
    blas_batch_kernel<<<grid, NT_CTA, Cfg128<double, SPLIT_BF16X3>::SMEM_BYTES, s>>>(
        (const BlasItem *)g_bws.items, (int)items.size(), A, B, C, trans, syrk, uplo, alpha, beta);
    CHB_LAUNCHED(1);
    CHB_CUDA(cudaGetLastError());
    CHB_CUDA(cudaStreamSynchronize(s));
    return 0;
}

// The 128 x 128 blocks of a rows x cols C tile (uplo: only the blocks that
// meet that triangle of the tile).
void add_blocks(std::vector<BlasItem> &out, BlasItem base, int rows, int cols, int uplo) {
    for (int c0 = 0; c0 < cols; c0 += SUBB)
        for (int r0 = 0; r0 < rows; r0 += SUBB) {
            const int br = std::min(SUBB, rows - r0), bc = std::min(SUBB, cols - c0);
            if (uplo == 1 && r0 + br - 1 < c0) continue;   // entirely above the diagonal
            if (uplo == 2 && r0 > c0 + bc - 1) continue;   // entirely below
            BlasItem it = base;
            it.r0 = r0;
            it.c0 = c0;
            it.rows = br;
            it.cols = bc;
            out.push_back(it);
        }
}

bool is_trans(cham_trans_t t) { return t == ChamTrans || t == ChamConjTrans; }

}  // namespace
}  // namespace chb

using namespace chb;

extern "C" {

int CHAMELEON_dgemm_batch_Tile(cham_trans_t transA, cham_trans_t transB, double alpha, CHAM_desc_t *A,
                               CHAM_desc_t *B, double beta, CHAM_desc_t *C) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || !B || !C || A->dtyp != ChamRealDouble || B->dtyp != ChamRealDouble || C->dtyp != ChamRealDouble)
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (transA < ChamNoTrans || transA > ChamConjTrans || transB < ChamNoTrans || transB > ChamConjTrans)
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (A->mt < C->mt || A->nt < C->nt || B->mt < C->mt || B->nt < C->nt) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const bool ta = is_trans(transA), tb = is_trans(transB);
    std::vector<BlasItem> items;
    for (int n = 0; n < C->nt; ++n)
        for (int m = 0; m < C->mt; ++m) {
            const int rows = desc_tile_rows(C, m), cols = desc_tile_cols(C, n);
            const int k = ta ? desc_tile_rows(A, m) : desc_tile_cols(A, n);
            // the operands must cover op(A): rows x k, op(B): k x cols
            const int am = ta ? k : rows, an = ta ? rows : k;
            const int bm = tb ? cols : k, bn = tb ? k : cols;
            if (desc_tile_rows(A, m) < am || desc_tile_cols(A, n) < an || desc_tile_rows(B, m) < bm ||
                desc_tile_cols(B, n) < bn)
                return CHAMELEON_ERR_ILLEGAL_VALUE;
            BlasItem base{desc_tile_off(A, m, n), desc_tile_off(B, m, n), desc_tile_off(C, m, n),
                          desc_tile_ld(A, m), desc_tile_ld(B, m), desc_tile_ld(C, m), 0, 0, k, 0, 0};
            add_blocks(items, base, rows, cols, 0);
        }
    if ((rc = launch_blas_batch(items, (const double *)A->mat, (const double *)B->mat, (double *)C->mat,
                                (ta ? 1 : 0) | (tb ? 2 : 0), 0, 0, alpha, beta)))
        return rc;
    return desc_sync_to_host(C);
}

int CHAMELEON_dsyrk_batch_Tile(cham_uplo_t uplo, cham_trans_t trans, double alpha, CHAM_desc_t *A, double beta,
                               CHAM_desc_t *C) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || !C || A->dtyp != ChamRealDouble || C->dtyp != ChamRealDouble) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (uplo != ChamUpper && uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (trans < ChamNoTrans || trans > ChamConjTrans) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (A->mt < C->mt || A->nt < C->nt) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const bool t = is_trans(trans);
    std::vector<BlasItem> items;
    for (int n = 0; n < C->nt; ++n)
        for (int m = 0; m < C->mt; ++m) {
            const int nn = desc_tile_cols(C, n);
            if (desc_tile_rows(C, m) < nn) return CHAMELEON_ERR_ILLEGAL_VALUE;
            const int k = t ? desc_tile_rows(A, m) : desc_tile_cols(A, n);
            if ((t ? desc_tile_cols(A, n) : desc_tile_rows(A, m)) < nn) return CHAMELEON_ERR_ILLEGAL_VALUE;
            BlasItem base{desc_tile_off(A, m, n), 0, desc_tile_off(C, m, n), desc_tile_ld(A, m), 0,
                          desc_tile_ld(C, m), 0, 0, k, 0, 0};
            add_blocks(items, base, nn, nn, uplo == ChamLower ? 1 : 2);
        }
    if ((rc = launch_blas_batch(items, (const double *)A->mat, nullptr, (double *)C->mat, t ? 1 : 0, 1,
                                uplo == ChamLower ? 1 : 2, alpha, beta)))
        return rc;
    return desc_sync_to_host(C);
}

}  // extern "C"
