// batch.cu -- batched Cholesky on independent matrices.
//
// Reference: CHAMELEON_dpotrf_batch_Tile / CHAMELEON_dtrsm_batch_Tile
// (compute/zpotrf_batch.c:28-118, compute/ztrsm_batch.c:37-213) map one CPU task
// per tile through chameleon_pmap (compute/pmap.c:25-93); potrf has no GPU
// path there (`.cudafunc = NULL`, zpotrf_batch.c:58-64).  Here each batch is
// ONE persistent launch: a CTA takes the next matrix from an atomic cursor
// (largest first, so the long tail is scheduled early), factors / solves it
// entirely on the SM with the tile routines of core.cuh, and keeps its
// inverted diagonal blocks in a per-CTA scratch slot.
//
// CHAM_B200_dposv_batch adds the uneven-size case (no reference equivalent:
// the reference batch API is uniform-size): matrix i is n_i x n_i with
// nrhs_i right-hand sides, factor + forward + backward solve in the same task.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "core.cuh"
#include "rec.cuh"
#include "internal.h"

namespace chb {


__global__ void __launch_bounds__(NT_CTA, 1) dposv_batch_kernel(const BatchItem *items, int count, double *A,
                                                                double *B, int upper, int *info, int *cursor,
                                                                double *scratch, int nib) {
    extern __shared__ __align__(128) double smem[];
    __shared__ int s_i;
    double *invd = scratch + (int64_t)blockIdx.x * nib * IB * IB;
    while (true) {
        if (threadIdx.x == 0) s_i = atomicAdd(cursor, 1);
        __syncthreads();
        const int i = s_i;
        __syncthreads();
        if (i >= count) break;
        const BatchItem it = items[i];
        const View T = upper ? View{A + it.a_off, it.lda, 1} : View{A + it.a_off, 1, it.lda};
        const int r = rec::tile_potrf_blk<double, SPLIT_BF16X3>(T, it.n, invd, smem);
        if (threadIdx.x == 0 && info) info[it.info_idx] = r;
        if (r == 0 && it.nrhs > 0) {
            const View X{B + it.b_off, 1, it.ldb};
            for (int c0 = 0; c0 < it.nrhs; c0 += IB) {
                const int w = min(IB, it.nrhs - c0);
                trsm_left<double, SPLIT_BF16X3>(X.sub(0, c0), w, T, it.n, invd, false, smem);
                trsm_left<double, SPLIT_BF16X3>(X.sub(0, c0), w, T, it.n, invd, true, smem);
            }
        }
        cta_sync_global();
    }
}

// Batched triangular solve: B_i <- alpha op(A_i)^{-1} B_i (Left) or
// alpha B_i op(A_i)^{-1} (Right), in the reduced form "left solve with a lower
// view L and an effective transposition" (see CUDA_dtrsm).
struct TrsmItem {
    int64_t a_off, b_off;
    int na, w, lda, ldb;
};

__global__ void __launch_bounds__(NT_CTA, 1) trsm_batch_kernel(const TrsmItem *items, int count, double *A,
                                                               double *B, int upper, int right, int trans_eff,
                                                               int unit, double alpha, int *cursor,
                                                               double *scratch, int nib) {
    extern __shared__ __align__(128) double smem[];
    __shared__ int s_i;
    double *invd = scratch + (int64_t)blockIdx.x * nib * IB * IB;
    double *sD = smem + Cfg12864<double>::SMEM_ELEMS;
    double *sInv = sD + IB * LDD;
    while (true) {
        if (threadIdx.x == 0) s_i = atomicAdd(cursor, 1);
        __syncthreads();
        const int i = s_i;
        __syncthreads();
        if (i >= count) break;
        const TrsmItem it = items[i];
        const View L = upper ? View{A + it.a_off, it.lda, 1} : View{A + it.a_off, 1, it.lda};
        const View X = right ? View{B + it.b_off, it.ldb, 1} : View{B + it.b_off, 1, it.ldb};
        if (alpha != 1.0) {
            for (int idx = threadIdx.x; idx < it.na * it.w; idx += NT_CTA) {
                double *p = X.at(idx % it.na, idx / it.na);
                *p = (alpha == 0.0) ? 0.0 : alpha * *p;
            }
        }
        for (int jb = 0; jb < it.na; jb += IB) {
            const int nbk = min(IB, it.na - jb);
            for (int idx = threadIdx.x; idx < nbk * nbk; idx += NT_CTA) {
                const int r = idx % nbk, c = idx / nbk;
                sD[r + c * LDD] = (r >= c) ? *L.at(jb + r, jb + c) : 0.0;
            }
            __syncthreads();
            blk_inv(sD, sInv, nbk, unit != 0);
            store_inv(invd + (int64_t)(jb / IB) * IB * IB, sInv);
            __syncthreads();
        }
        cta_sync_global();
        for (int c0 = 0; c0 < it.w; c0 += IB)
            trsm_left<double, SPLIT_BF16X3>(X.sub(0, c0), min(IB, it.w - c0), L, it.na, invd, trans_eff != 0, smem);
        cta_sync_global();
    }
}

BatchWs g_bws;

// Grow-only, stream-ordered (no device-wide synchronization when growing).
int bws_reserve(BatchWs &ws, size_t item_bytes, size_t scratch_bytes, size_t ninfo) {
    if (!ws.cursor && !(ws.cursor = (int *)dev_alloc(sizeof(int)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    if (item_bytes > ws.items_bytes) {
        dev_free(ws.items);
        ws.items_bytes = 0;
        if (!(ws.items = dev_alloc(item_bytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        ws.items_bytes = item_bytes;
    }
    if (scratch_bytes > ws.scratch_bytes) {
        dev_free(ws.scratch);
        ws.scratch_bytes = 0;
        if (!(ws.scratch = (double *)dev_alloc(scratch_bytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        ws.scratch_bytes = scratch_bytes;
    }
    if (ninfo > ws.info_n) {
        dev_free(ws.info);
        ws.info_n = 0;
        if (!(ws.info = (int *)dev_alloc(ninfo * sizeof(int)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        ws.info_n = ninfo;
    }
    return 0;
}

namespace {
bool g_attr = false;
int set_attrs() {
    if (g_attr) return 0;
    CHB_CUDA(cudaFuncSetAttribute(dposv_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)TILE_KERNEL_SMEM_BYTES));
    CHB_CUDA(cudaFuncSetAttribute(trsm_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)TILE_KERNEL_SMEM_BYTES));
    g_attr = true;
    return 0;
}
}  // namespace

// Launch the factor(+solve) batch over host-described items (sorted here,
// largest first).  `info` is a device array indexed by item.info_idx (or null).
int launch_posv_batch(std::vector<BatchItem> &items, double *A, double *B, int upper, int *info, cudaStream_t s,
                      BatchWs &ws) {
    if (items.empty()) return 0;
    if (int rc = set_attrs()) return rc;
    std::stable_sort(items.begin(), items.end(),
                     [](const BatchItem &a, const BatchItem &b) { return a.n > b.n; });
    const int nmax = items.front().n;
    const int nib = std::max(1, (nmax + IB - 1) / IB);
    const int grid = std::min<int>(ctx().num_sms, (int)items.size());
    if (int rc = bws_reserve(ws, items.size() * sizeof(BatchItem), (size_t)grid * nib * IB * IB * sizeof(double), 1))
        return rc;
    CHB_CUDA(cudaMemcpyAsync(ws.items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, s));
    CHB_CUDA(cudaMemsetAsync(ws.cursor, 0, sizeof(int), s));
    CHB_LAUNCHED(1);
    dposv_batch_kernel<<<grid, NT_CTA, TILE_KERNEL_SMEM_BYTES, s>>>((const BatchItem *)ws.items, (int)items.size(),
                                                                    A, B, upper, info, ws.cursor, ws.scratch,
                                                                    nib);
    CHB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace chb

using namespace chb;

extern "C" {

// compute/zpotrf_batch.c:89 -- every tile (m,n) of A is an independent
// tempnn x tempnn matrix factored in place.  As in the reference, a failed
// factorization is reported on stderr and the call still returns success.
int CHAMELEON_dpotrf_batch_Tile(cham_uplo_t uplo, CHAM_desc_t *A) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || A->dtyp != ChamRealDouble) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (uplo != ChamUpper && uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    std::vector<BatchItem> items;
    for (int n = 0; n < A->nt; ++n)
        for (int m = 0; m < A->mt; ++m) {
            BatchItem it{};
            it.a_off = desc_tile_off(A, m, n);
            it.n = desc_tile_cols(A, n);
            if (desc_tile_rows(A, m) < it.n) it.n = desc_tile_rows(A, m);
            it.lda = desc_tile_ld(A, m);
            it.info_idx = (int)items.size();
            items.push_back(it);
        }
    cudaStream_t s = ctx().stream;
    if ((rc = bws_reserve(g_bws, 0, 0, items.size()))) return rc;
    int *dinfo = g_bws.info;
    if ((rc = launch_posv_batch(items, (double *)A->mat, nullptr, uplo == ChamUpper, dinfo, s, g_bws))) return rc;
    std::vector<int> hinfo(items.size());
    CHB_CUDA(cudaMemcpyAsync(hinfo.data(), dinfo, hinfo.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaStreamSynchronize(s));
    for (size_t i = 0; i < hinfo.size(); ++i)
        if (hinfo[i]) {
            char msg[128];
            snprintf(msg, sizeof msg, "Failed to correctly factorize the tile %zu (info = %d)", i, hinfo[i]);
            warning("CHAMELEON_dpotrf_batch_Tile", msg);
        }
    return desc_sync_to_host(A);
}

// compute/ztrsm_batch.c:180 -- tile (m,n) of B solved with tile (m,n) of A.
int CHAMELEON_dtrsm_batch_Tile(cham_side_t side, cham_uplo_t uplo, cham_trans_t trans, cham_diag_t diag,
                               double alpha, CHAM_desc_t *A, CHAM_desc_t *B) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || !B || A->dtyp != ChamRealDouble || B->dtyp != ChamRealDouble) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (side != ChamLeft && side != ChamRight) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (uplo != ChamUpper && uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (B->mt > A->mt || B->nt > A->nt) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if ((rc = set_attrs())) return rc;
    const bool left = side == ChamLeft, up = uplo == ChamUpper, tr = trans != ChamNoTrans;
    const int trans_eff = left ? (tr != up) : (!tr != up);
    std::vector<TrsmItem> items;
    int nmax = 1;
    for (int n = 0; n < B->nt; ++n)
        for (int m = 0; m < B->mt; ++m) {
            TrsmItem it{};
            const int bm = desc_tile_rows(B, m), bn = desc_tile_cols(B, n);
            it.a_off = desc_tile_off(A, m, n);
            it.lda = desc_tile_ld(A, m);
            it.b_off = desc_tile_off(B, m, n);
            it.ldb = desc_tile_ld(B, m);
            it.na = left ? bm : bn;
            it.w = left ? bn : bm;
            nmax = std::max(nmax, it.na);
            items.push_back(it);
        }
    const int nib = (nmax + IB - 1) / IB;
    const int grid = std::min<int>(ctx().num_sms, (int)items.size());
    cudaStream_t s = ctx().stream;
    if ((rc = bws_reserve(g_bws, items.size() * sizeof(TrsmItem), (size_t)grid * nib * IB * IB * sizeof(double), 1)))
        return rc;
    CHB_CUDA(cudaMemcpyAsync(g_bws.items, items.data(), items.size() * sizeof(TrsmItem), cudaMemcpyHostToDevice, s));
    CHB_CUDA(cudaMemsetAsync(g_bws.cursor, 0, sizeof(int), s));
    CHB_LAUNCHED(1);
    trsm_batch_kernel<<<grid, NT_CTA, TILE_KERNEL_SMEM_BYTES, s>>>((const TrsmItem *)g_bws.items, (int)items.size(),
                                                                   (double *)A->mat, (double *)B->mat, up, !left,
                                                                   trans_eff, diag == ChamUnit, alpha, g_bws.cursor,
                                                                   g_bws.scratch, nib);
    CHB_CUDA(cudaGetLastError());
    CHB_CUDA(cudaStreamSynchronize(s));
    return desc_sync_to_host(B);
}

// Uneven batch: factor + solve `count` independent SPD systems in one launch.
// n, nrhs, a_off, b_off, info: device arrays; offsets in elements.
int CHAM_B200_dposv_batch(cham_uplo_t uplo, int count, const int *n, const int *nrhs, double *A,
                          const int64_t *a_off, double *B, const int64_t *b_off, int *info, void *cuda_stream) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (count < 0) return -2;
    if (count == 0) return 0;
    cudaStream_t s = cuda_stream ? (cudaStream_t)cuda_stream : ctx().stream;
    std::vector<int> hn(count), hr(count);
    std::vector<int64_t> ha(count), hb(count);
    CHB_CUDA(cudaMemcpyAsync(hn.data(), n, count * sizeof(int), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaMemcpyAsync(hr.data(), nrhs, count * sizeof(int), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaMemcpyAsync(ha.data(), a_off, count * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaMemcpyAsync(hb.data(), b_off, count * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaStreamSynchronize(s));
    std::vector<BatchItem> items(count);
    for (int i = 0; i < count; ++i) {
        if (hn[i] < 0 || hr[i] < 0) return -3;
        items[i] = BatchItem{ha[i], hb[i], hn[i], hr[i], std::max(1, hn[i]), std::max(1, hn[i]), i, 0};
    }
    items.erase(std::remove_if(items.begin(), items.end(), [](const BatchItem &b) { return b.n == 0; }),
                items.end());
    if (info) CHB_CUDA(cudaMemsetAsync(info, 0, count * sizeof(int), s));
    if ((rc = launch_posv_batch(items, A, B, uplo == ChamUpper, info, s, g_bws))) return rc;
    CHB_CUDA(cudaStreamSynchronize(s));
    return 0;
}

}  // extern "C"
