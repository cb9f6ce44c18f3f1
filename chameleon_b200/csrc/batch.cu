// batch.cu -- batched Cholesky on independent matrices.
//
// Reference: CHAMELEON_dpotrf_batch_Tile / CHAMELEON_dtrsm_batch_Tile
// (compute/zpotrf_batch.c:28-118, compute/ztrsm_batch.c:37-213) map one CPU task
// per tile through chameleon_pmap (compute/pmap.c:25-93); potrf has no GPU
// path there (`.cudafunc = NULL`, zpotrf_batch.c:58-64).  Here a batch is
// sorted largest first and split into size ranges (n <= 64, 65..128,
// 129..256, 257+); each range runs as ONE persistent launch in which a CTA
// takes the next system from an atomic cursor, in one of these shapes:
//
//   * generic: the tile routines (64-wide leaf Cholesky, panel GEMMs on the
//     tensor cores, inverted diagonal blocks in a per-CTA scratch slot), one
//     177 KB CTA per SM;
//   * lean generic: the same routines with 64-row panels and the leaf blocks
//     aliased onto the GEMM staging area (74 KB for FP64), 2 or 3 CTAs per SM,
//     so that the latency-bound leaf of one system overlaps the work of the
//     systems beside it;
//   * small (n <= 64): the whole system in shared memory -- leaf Cholesky +
//     inverse, then X = L^-T L^-1 B by two small products over the live
//     right-hand-side columns -- at 1..3 CTAs per SM.
//
// The shape of each range is picked once per device and element type by
// timing the admissible shapes on synthetic systems of that range; adjacent
// ranges with the same shape merge into one launch.  A small-kernel range
// runs on a side stream, so its CTAs fill SMs as the larger ranges drain.
// CHAM_B200_dposv_batch / sposv_batch (uneven sizes, no reference equivalent:
// the reference batch API is uniform-size) capture the whole sequence in a
// CUDA graph per batch signature and replay it when the same batch comes again.
#include <cuda_runtime.h>

#include <algorithm>
#include <list>
#include <numeric>
#include <vector>

#include "core.cuh"
#include "rec.cuh"
#include "internal.h"

namespace chb {

// Generic bin: factor (+ forward and backward solve) of one system per task.
// LEAN: 64-row panels and the leaf blocks aliased onto the GEMM staging area
// (rec::lean_smem_elems), MINB CTAs per SM, so that the latency-bound leaf of
// one system overlaps the GEMMs and leaves of the systems beside it.
template <class T, bool LEAN = false, int MINB = 1>
__global__ void __launch_bounds__(NT_CTA, MINB) posv_batch_kernel(const BatchItem *items, int count, T *A, T *B,
                                                                  int upper, int *info, int *cursor, T *scratch,
                                                                  int nib) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T *smem = reinterpret_cast<T *>(smem_raw);
    __shared__ int s_i;
    T *invd = scratch + (int64_t)blockIdx.x * nib * IB * IB;
    while (true) {
        if (threadIdx.x == 0) s_i = atomicAdd(cursor, 1);
        __syncthreads();
        const int i = s_i;
        __syncthreads();
        if (i >= count) break;
        const BatchItem it = items[i];
        const ViewT<T> Lv = upper ? ViewT<T>{A + it.a_off, it.lda, 1} : ViewT<T>{A + it.a_off, 1, it.lda};
        const int r = LEAN ? rec::tile_potrf_blk<T, SPLIT_BF16X3, 64, true>(Lv, it.n, invd, smem)
                           : rec::tile_potrf_blk<T, SPLIT_BF16X3>(Lv, it.n, invd, smem);
        if (threadIdx.x == 0 && info) info[it.info_idx] = r;
        if (r == 0 && it.nrhs > 0) {
            const ViewT<T> X{B + it.b_off, 1, it.ldb};
            for (int c0 = 0; c0 < it.nrhs; c0 += IB) {
                const int w = min(IB, it.nrhs - c0);
                // a narrow last block (few right-hand sides, the common case)
                // runs on the narrow tile instead of padding it to 64 columns
                if (w <= Cfg64N<T>::BN) {
                    trsm_left<T, SPLIT_BF16X3, Cfg64N<T>>(X.sub(0, c0), w, Lv, it.n, invd, false, smem);
                    trsm_left<T, SPLIT_BF16X3, Cfg64N<T>>(X.sub(0, c0), w, Lv, it.n, invd, true, smem);
                } else {
                    trsm_left<T, SPLIT_BF16X3>(X.sub(0, c0), w, Lv, it.n, invd, false, smem);
                    trsm_left<T, SPLIT_BF16X3>(X.sub(0, c0), w, Lv, it.n, invd, true, smem);
                }
            }
        }
        cta_sync_global();
    }
}

template <class T>
constexpr size_t lean_smem_bytes() {
    return sizeof(T) * rec::lean_smem_elems<T, SPLIT_BF16X3>() + 64;
}

// Small bin (n <= 64): system in shared memory.  sD holds the identity-padded
// block, then L, then the right-hand sides being solved; sX the inverse.
template <class T>
constexpr size_t small_smem_bytes() {
    return 2 * 64 * rec::LDS * sizeof(T);
}
template <class T, int MINB>
__global__ void __launch_bounds__(NT_CTA, MINB)
    posv_small_kernel(const BatchItem *items, int count, T *A, T *B, int upper, int *info, int *cursor) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T *sD = reinterpret_cast<T *>(smem_raw);
    T *sX = sD + 64 * rec::LDS;
    constexpr int LDS = rec::LDS;
    __shared__ int s_i;
    const int tid = threadIdx.x;
    while (true) {
        if (tid == 0) s_i = atomicAdd(cursor, 1);
        __syncthreads();
        const int i = s_i;
        __syncthreads();
        if (i >= count) break;
        const BatchItem it = items[i];
        const int n = it.n;
        const ViewT<T> Lv = upper ? ViewT<T>{A + it.a_off, it.lda, 1} : ViewT<T>{A + it.a_off, 1, it.lda};
        rec::leaf64_load(Lv, n, sD);
        const int r = rec::leaf64_core<T, true>(sD);
        if (tid == 0 && info) info[it.info_idx] = r;
        if (r != 0) continue;   // uniform across the CTA
        for (int idx = tid; idx < n * n; idx += NT_CTA) {
            const int rr = idx % n, cc = idx / n;
            if (rr >= cc) *Lv.at(rr, cc) = sD[rr + cc * LDS];
        }
        for (int c0 = 0; c0 < it.nrhs; c0 += 64) {
            const int w = min(64, it.nrhs - c0);
            T *Bc = B + it.b_off + (int64_t)c0 * it.ldb;
            __syncthreads();   // sD is free once L has been written back
            for (int idx = tid; idx < 64 * 64; idx += NT_CTA) {
                const int rr = idx & 63, cc = idx >> 6;
                sD[rr + cc * LDS] = (rr < n && cc < w) ? Bc[rr + (int64_t)cc * it.ldb] : T(0);
            }
            __syncthreads();
            // thread (rr = tid & 63, cc = tid / 64 + 4 q) owns output (rr, cc);
            // only the w live columns are computed (cc is uniform per warp)
            T y[16];
            // Y = X B (X lower, zero above the diagonal, identity beyond n)
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int idx = tid + NT_CTA * q, rr = idx & 63, cc = idx >> 6;
                T acc = T(0);
                if (cc < w) {
#pragma unroll 8
                    for (int k = 0; k < 64; ++k) acc += sX[rr + k * LDS] * sD[k + cc * LDS];
                }
                y[q] = acc;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int idx = tid + NT_CTA * q;
                if ((idx >> 6) < w) sD[(idx & 63) + (idx >> 6) * LDS] = y[q];
            }
            __syncthreads();
            // X_out = X^T Y
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int idx = tid + NT_CTA * q, rr = idx & 63, cc = idx >> 6;
                if (cc < w) {
                    T acc = T(0);
#pragma unroll 8
                    for (int k = 0; k < 64; ++k) acc += sX[k + rr * LDS] * sD[k + cc * LDS];
                    if (rr < n) Bc[rr + (int64_t)cc * it.ldb] = acc;
                }
            }
        }
        __syncthreads();
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
    if (!ws.cursor && !(ws.cursor = (int *)dev_alloc(8 * sizeof(int)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
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
    CHB_CUDA(cudaFuncSetAttribute(posv_batch_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tile_smem_bytes<double>()));
    CHB_CUDA(cudaFuncSetAttribute(posv_batch_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)tile_smem_bytes<float>()));
    CHB_CUDA(cudaFuncSetAttribute(posv_batch_kernel<double, true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)lean_smem_bytes<double>()));
    CHB_CUDA(cudaFuncSetAttribute(posv_batch_kernel<double, true, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)lean_smem_bytes<double>()));
    CHB_CUDA(cudaFuncSetAttribute(posv_batch_kernel<float, true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)lean_smem_bytes<float>()));
    CHB_CUDA(cudaFuncSetAttribute(posv_batch_kernel<float, true, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)lean_smem_bytes<float>()));
#define CHB_SMALL_ATTR(T, K)                                                                          \
    CHB_CUDA(cudaFuncSetAttribute(posv_small_kernel<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)small_smem_bytes<T>()))
    CHB_SMALL_ATTR(double, 1);
    CHB_SMALL_ATTR(double, 2);
    CHB_SMALL_ATTR(double, 3);
    CHB_SMALL_ATTR(float, 1);
    CHB_SMALL_ATTR(float, 2);
    CHB_SMALL_ATTR(float, 3);
#undef CHB_SMALL_ATTR
    CHB_CUDA(cudaFuncSetAttribute(trsm_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)TILE_KERNEL_SMEM_BYTES));
    g_attr = true;
    return 0;
}

// Size ranges of a batch and the kernel shapes that can run them.  Range 0 is
// n <= 64 (whole system in shared memory possible), ranges 1..3 are 65..128,
// 129..256 and 257+.  Shapes: 0 = generic kernel, one 177 KB CTA per SM;
// 1..3 = small-system kernel at 1..3 CTAs per SM (range 0 only); 4 / 5 = lean
// generic kernel at 2 / 3 CTAs per SM.  The shape of each range is chosen once
// per device and element type, the first time a batch has systems in that
// range, by timing every admissible shape on synthetic systems of the range
// (autotune_range); adjacent ranges that pick the same shape run as one bin
// (one persistent launch), so the bin boundaries follow from the tuning.
constexpr int NRANGE = 4;
constexpr int NSHAPE = 6;
constexpr int RANGE_LO[NRANGE] = {1, 65, 129, 257};
constexpr int RANGE_HI[NRANGE] = {64, 128, 256, 1 << 30};
constexpr int TUNE_HI[NRANGE] = {64, 128, 256, 512};   // synthetic sizes of the top range

int range_of(int n) {
    int r = 0;
    while (r < NRANGE - 1 && n > RANGE_HI[r]) ++r;
    return r;
}

struct BinTune {
    int mode[NRANGE] = {-1, -1, -1, -1};
    float ms[NRANGE][NSHAPE];
    BinTune() {
        for (auto &r : ms)
            for (float &v : r) v = -1.f;
    }
};
BinTune g_tune[2];   // [0] double, [1] float
std::mutex g_tune_mu;

template <class T>
constexpr int tidx() {
    return sizeof(T) == 8 ? 0 : 1;
}

// CTAs per SM of a shape, and whether the device runs it at that occupancy.
int shape_ctas(int shape) { return shape == 0 ? 1 : shape <= 3 ? shape : shape - 2; }

template <class T>
bool shape_fits(int shape) {
    int occ = 0;
    switch (shape) {
    case 0: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, posv_batch_kernel<T, false, 1>, NT_CTA, tile_smem_bytes<T>()); break;
    case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, posv_small_kernel<T, 1>, NT_CTA, small_smem_bytes<T>()); break;
    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, posv_small_kernel<T, 2>, NT_CTA, small_smem_bytes<T>()); break;
    case 3: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, posv_small_kernel<T, 3>, NT_CTA, small_smem_bytes<T>()); break;
    case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, posv_batch_kernel<T, true, 2>, NT_CTA, lean_smem_bytes<T>()); break;
    case 5: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, posv_batch_kernel<T, true, 3>, NT_CTA, lean_smem_bytes<T>()); break;
    default: return false;
    }
    cudaGetLastError();
    return occ >= shape_ctas(shape);
}

// One persistent launch of `shape` over items [0, cnt) of d_items (largest
// first); nmax = the largest order among them.  Stream operations only.
template <class T>
int launch_shape(int shape, const BatchItem *d_items, int cnt, int nmax, T *A, T *B, int upper, int *info,
                 int *cursor, cudaStream_t st, BatchWs &ws) {
    if (cnt <= 0) return 0;
    const int sms = ctx().num_sms;
    const int grid = std::min(sms * shape_ctas(shape), cnt);
    const int nib = std::max(1, (std::max(nmax, 64) + IB - 1) / IB);
    T *scr = (T *)ws.scratch;
    switch (shape) {
    case 0: posv_batch_kernel<T, false, 1><<<grid, NT_CTA, tile_smem_bytes<T>(), st>>>(d_items, cnt, A, B, upper, info, cursor, scr, nib); break;
    case 1: posv_small_kernel<T, 1><<<grid, NT_CTA, small_smem_bytes<T>(), st>>>(d_items, cnt, A, B, upper, info, cursor); break;
    case 2: posv_small_kernel<T, 2><<<grid, NT_CTA, small_smem_bytes<T>(), st>>>(d_items, cnt, A, B, upper, info, cursor); break;
    case 3: posv_small_kernel<T, 3><<<grid, NT_CTA, small_smem_bytes<T>(), st>>>(d_items, cnt, A, B, upper, info, cursor); break;
    case 4: posv_batch_kernel<T, true, 2><<<grid, NT_CTA, lean_smem_bytes<T>(), st>>>(d_items, cnt, A, B, upper, info, cursor, scr, nib); break;
    case 5: posv_batch_kernel<T, true, 3><<<grid, NT_CTA, lean_smem_bytes<T>(), st>>>(d_items, cnt, A, B, upper, info, cursor, scr, nib); break;
    default: return CHAMELEON_ERR_ILLEGAL_VALUE;
    }
    CHB_LAUNCHED(1);
    CHB_CUDA(cudaGetLastError());
    return 0;
}

// Scratch the generic shapes need: one slot of inverted diagonal blocks per
// CTA, for up to 3 CTAs per SM.
template <class T>
size_t scratch_bytes(int nmax) {
    const int nib = std::max(1, (std::max(nmax, 64) + IB - 1) / IB);
    return (size_t)3 * ctx().num_sms * nib * IB * IB * sizeof(T);
}

// Synthetic symmetric diagonally dominant systems for the autotuner.
template <class T>
__global__ void tune_fill_kernel(const BatchItem *items, int count, T *A, T *B) {
    const int i = blockIdx.x;
    if (i >= count) return;
    const BatchItem it = items[i];
    for (int idx = threadIdx.x; idx < it.n * it.n; idx += blockDim.x) {
        const int r = idx % it.n, c = idx / it.n;
        const unsigned lo = min(r, c), hi = max(r, c);
        const unsigned h = (lo * 2654435761u) ^ (hi * 40503u) ^ ((unsigned)i * 97u);
        A[it.a_off + idx] = (r == c) ? T(it.n) : T((h & 1023) / 1024.0 - 0.5);
    }
    for (int idx = threadIdx.x; idx < it.n * it.nrhs; idx += blockDim.x) B[it.b_off + idx] = T(1);
}

// Time every admissible shape of range r on 6 systems per SM with orders
// uniform over the range (4 right-hand sides) and keep the fastest.
template <class T>
int autotune_range(int r, cudaStream_t s, BatchWs &ws) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    BinTune &tu = g_tune[tidx<T>()];
    if (tu.mode[r] >= 0) return 0;
    const int cnt = 6 * ctx().num_sms, k = 4;
    const int lo = RANGE_LO[r] < 16 ? 16 : RANGE_LO[r], hi = TUNE_HI[r];
    std::vector<BatchItem> items(cnt);
    int64_t oa = 0, ob = 0;
    uint32_t st = 12345u + 977u * r;
    for (int i = 0; i < cnt; ++i) {
        st = st * 1664525u + 1013904223u;
        const int n = lo + (int)((st >> 8) % (uint32_t)(hi - lo + 1));
        items[i] = BatchItem{oa, ob, n, k, n, n, i, 0};
        oa += (int64_t)n * n;
        ob += (int64_t)n * k;
    }
    std::sort(items.begin(), items.end(), [](const BatchItem &a, const BatchItem &b) { return a.n > b.n; });
    if (int rc = bws_reserve(ws, 0, scratch_bytes<T>(hi), 0)) return rc;
    T *A = (T *)dev_alloc(oa * sizeof(T)), *B = (T *)dev_alloc(ob * sizeof(T));
    BatchItem *d_items = (BatchItem *)dev_alloc(cnt * sizeof(BatchItem));
    int *d_info = (int *)dev_alloc(cnt * sizeof(int));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = (A && B && d_items && d_info) ? 0 : CHAMELEON_ERR_OUT_OF_RESOURCES;
    if (!rc) rc = (cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) ? 0 : CHAMELEON_ERR_UNEXPECTED;
    if (!rc && cudaMemcpyAsync(d_items, items.data(), cnt * sizeof(BatchItem), cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = CHAMELEON_ERR_UNEXPECTED;
    int best = 0;
    float best_ms = 1e30f;
    for (int shape = 0; shape < NSHAPE && !rc; ++shape) {
        if ((r > 0 && shape >= 1 && shape <= 3) || !shape_fits<T>(shape)) continue;
        float t = 0.f;
        for (int rep = 0; rep < 2 && !rc; ++rep) {   // rep 0 warms the kernel up
            tune_fill_kernel<T><<<cnt, 128, 0, s>>>(d_items, cnt, A, B);
            if (cudaMemsetAsync(ws.cursor + 7, 0, sizeof(int), s) != cudaSuccess) rc = CHAMELEON_ERR_UNEXPECTED;
            cudaEventRecord(e0, s);
            if (!rc) rc = launch_shape<T>(shape, d_items, cnt, items[0].n, A, B, 0, d_info, ws.cursor + 7, s, ws);
            cudaEventRecord(e1, s);
            if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = CHAMELEON_ERR_UNEXPECTED;
            if (!rc) cudaEventElapsedTime(&t, e0, e1);
        }
        tu.ms[r][shape] = t;
        if (!rc && t < best_ms) {
            best_ms = t;
            best = shape;
        }
    }
    cudaStreamSynchronize(s);
    dev_free(A);
    dev_free(B);
    dev_free(d_items);
    dev_free(d_info);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc) return rc;
    tu.mode[r] = best;
    return 0;
}

// Items sorted largest first, split into the size ranges: range r is
// [beg[r], beg[r] + cnt[r]), nmax[r] its largest order.
struct Bins {
    int beg[NRANGE] = {0, 0, 0, 0}, cnt[NRANGE] = {0, 0, 0, 0}, nmax[NRANGE] = {0, 0, 0, 0};
    int nmax_all = 0;
};
Bins make_bins(std::vector<BatchItem> &items) {
    std::stable_sort(items.begin(), items.end(), [](const BatchItem &a, const BatchItem &b) { return a.n > b.n; });
    Bins b;
    b.nmax_all = items.empty() ? 0 : items[0].n;
    for (int i = 0; i < (int)items.size(); ++i) {
        const int r = range_of(items[i].n);
        if (b.cnt[r]++ == 0) {
            b.beg[r] = i;
            b.nmax[r] = items[i].n;
        }
    }
    return b;
}

// Launch the bins: the generic-kernel ranges on `s` one after another (from
// the largest orders down; adjacent ranges with the same shape merge into one
// launch), a small-kernel range 0 concurrently on the side stream; `s` waits
// for both.  Stream operations only (capturable).  *nlaunch = kernels launched.
template <class T>
int launch_bins(const BatchItem *d_items, const Bins &b, const int *mode, T *A, T *B, int upper, int *info,
                cudaStream_t s, BatchWs &ws, int *nlaunch) {
    *nlaunch = 0;
    CHB_CUDA(cudaMemsetAsync(ws.cursor, 0, 8 * sizeof(int), s));
    const bool side = b.cnt[0] > 0 && mode[0] >= 1 && mode[0] <= 3;
    if (side) {
        CHB_CUDA(cudaEventRecord(ws.fork, s));
        CHB_CUDA(cudaStreamWaitEvent(ws.side, ws.fork, 0));
        if (int rc = launch_shape<T>(mode[0], d_items + b.beg[0], b.cnt[0], b.nmax[0], A, B, upper, info, ws.cursor + 6,
                                     ws.side, ws))
            return rc;
        ++*nlaunch;
        CHB_CUDA(cudaEventRecord(ws.join, ws.side));
    }
    int seg_shape = -1, seg_beg = 0, seg_cnt = 0, seg_nmax = 0, slot = 0;
    auto flush = [&]() -> int {
        if (seg_cnt == 0) return 0;
        const int rc = launch_shape<T>(seg_shape, d_items + seg_beg, seg_cnt, seg_nmax, A, B, upper, info,
                                       ws.cursor + slot++, s, ws);
        ++*nlaunch;
        seg_cnt = 0;
        return rc;
    };
    for (int r = NRANGE - 1; r >= 0; --r) {
        if (b.cnt[r] == 0 || (r == 0 && side)) continue;
        if (seg_cnt > 0 && mode[r] == seg_shape) {
            seg_cnt += b.cnt[r];
            continue;
        }
        if (int rc = flush()) return rc;
        seg_shape = mode[r];
        seg_beg = b.beg[r];
        seg_cnt = b.cnt[r];
        seg_nmax = b.nmax[r];
    }
    if (int rc = flush()) return rc;
    if (side) CHB_CUDA(cudaStreamWaitEvent(s, ws.join, 0));
    return 0;
}

template <class T>
int prepare(BatchWs &ws, cudaStream_t s, size_t nitems, const Bins &b) {
    if (int rc = set_attrs()) return rc;
    if (!ws.side) {
        CHB_CUDA(cudaStreamCreateWithFlags(&ws.side, cudaStreamNonBlocking));
        CHB_CUDA(cudaEventCreateWithFlags(&ws.fork, cudaEventDisableTiming));
        CHB_CUDA(cudaEventCreateWithFlags(&ws.join, cudaEventDisableTiming));
    }
    for (int r = 0; r < NRANGE; ++r)
        if (b.cnt[r] > 0)
            if (int rc = autotune_range<T>(r, s, ws)) return rc;
    return bws_reserve(ws, nitems * sizeof(BatchItem), scratch_bytes<T>(b.nmax_all), 1);
}
}  // namespace

// Launch the factor(+solve) batch over host-described items (binned and sorted
// here, largest first).  `info` is a device array indexed by item.info_idx (or null).
template <class T>
int launch_posv_batch_t(std::vector<BatchItem> &items, T *A, T *B, int upper, int *info, cudaStream_t s,
                        BatchWs &ws) {
    if (items.empty()) return 0;
    const Bins b = make_bins(items);
    if (int rc = prepare<T>(ws, s, items.size(), b)) return rc;
    CHB_CUDA(cudaMemcpyAsync(ws.items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, s));
    int nl = 0;
    return launch_bins<T>((const BatchItem *)ws.items, b, g_tune[tidx<T>()].mode, A, B, upper, info, s, ws, &nl);
}

int launch_posv_batch(std::vector<BatchItem> &items, double *A, double *B, int upper, int *info, cudaStream_t s,
                      BatchWs &ws) {
    return launch_posv_batch_t<double>(items, A, B, upper, info, s, ws);
}

// CUDA graphs of whole batches, keyed by the batch signature (sizes, offsets,
// pointers, triangle, element type); each owns a device copy of its item list.
namespace {
struct BatchGraph {
    uint64_t key = 0;
    cudaGraphExec_t exec = nullptr;
    BatchItem *d_items = nullptr;
    int nlaunch = 0;   // kernels in the graph
};
std::list<BatchGraph> g_graphs;   // most recent first
std::mutex g_graph_mu;
constexpr size_t MAX_GRAPHS = 8;

uint64_t fnv(uint64_t h, const void *p, size_t n) {
    const unsigned char *c = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
    return h;
}

template <class T>
int posv_batch_graph(std::vector<BatchItem> &items, T *A, T *B, int upper, int *info, int count, cudaStream_t s) {
    BatchWs &ws = g_bws;
    const Bins b = make_bins(items);
    if (int rc = prepare<T>(ws, s, items.size(), b)) return rc;
    const int *mode = g_tune[tidx<T>()].mode;
    uint64_t key = 1469598103934665603ull;
    key = fnv(key, items.data(), items.size() * sizeof(BatchItem));
    const void *ptrs[4] = {A, B, info, ws.scratch};
    const int ints[4] = {upper, count, (int)sizeof(T), (int)items.size()};
    key = fnv(key, ptrs, sizeof ptrs);
    key = fnv(key, ints, sizeof ints);
    key = fnv(key, mode, NRANGE * sizeof(int));
    std::lock_guard<std::mutex> lk(g_graph_mu);
    for (auto it = g_graphs.begin(); it != g_graphs.end(); ++it) {
        if (it->key != key) continue;
        g_graphs.splice(g_graphs.begin(), g_graphs, it);
        CHB_LAUNCHED(g_graphs.front().nlaunch);
        CHB_CUDA(cudaGraphLaunch(g_graphs.front().exec, s));
        return 0;
    }
    BatchGraph g;
    g.key = key;
    if (!(g.d_items = (BatchItem *)dev_alloc(items.size() * sizeof(BatchItem)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    CHB_CUDA(cudaMemcpyAsync(g.d_items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, s));
    cudaGraph_t graph = nullptr;
    CHB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    if (info) cudaMemsetAsync(info, 0, count * sizeof(int), s);
    const int rcl = launch_bins<T>(g.d_items, b, mode, A, B, upper, info, s, ws, &g.nlaunch);
    const cudaError_t ec = cudaStreamEndCapture(s, &graph);
    if (rcl || ec != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        dev_free(g.d_items);
        return rcl ? rcl : CHAMELEON_ERR_UNEXPECTED;
    }
    const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        dev_free(g.d_items);
        return CHAMELEON_ERR_UNEXPECTED;
    }
    CHB_CUDA(cudaGraphLaunch(g.exec, s));
    g_graphs.push_front(g);
    if (g_graphs.size() > MAX_GRAPHS) {
        cudaStreamSynchronize(s);
        cudaGraphExecDestroy(g_graphs.back().exec);
        dev_free(g_graphs.back().d_items);
        g_graphs.pop_back();
    }
    return 0;
}

// Uneven batch entry: read the device-side sizes, then the graph path.
template <class T>
int posv_batch_entry(cham_uplo_t uplo, int count, const int *n, const int *nrhs, T *A, const int64_t *a_off, T *B,
                     const int64_t *b_off, int *info, void *cuda_stream) {
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
    if (items.empty()) {
        if (info) CHB_CUDA(cudaMemsetAsync(info, 0, count * sizeof(int), s));
    } else if ((rc = posv_batch_graph<T>(items, A, B, uplo == ChamUpper, info, count, s))) {
        return rc;
    }
    CHB_CUDA(cudaStreamSynchronize(s));
    return 0;
}
}  // namespace

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

// Uneven batch: factor + solve `count` independent SPD systems.
// n, nrhs, a_off, b_off, info: device arrays; offsets in elements.
int CHAM_B200_dposv_batch(cham_uplo_t uplo, int count, const int *n, const int *nrhs, double *A,
                          const int64_t *a_off, double *B, const int64_t *b_off, int *info, void *cuda_stream) {
    return posv_batch_entry<double>(uplo, count, n, nrhs, A, a_off, B, b_off, info, cuda_stream);
}

// The same for FP32 systems (FP32 arithmetic, tensor-core products as BF16x3).
int CHAM_B200_sposv_batch(cham_uplo_t uplo, int count, const int *n, const int *nrhs, float *A,
                          const int64_t *a_off, float *B, const int64_t *b_off, int *info, void *cuda_stream) {
    return posv_batch_entry<float>(uplo, count, n, nrhs, A, a_off, B, b_off, info, cuda_stream);
}

// Autotuner choice for the small bin (n <= 64) of element type `dtype`
// (ChamRealDouble / ChamRealFloat): out[0] = mode (0: generic kernel, k: small
// kernel at k CTAs per SM), out[1..4] = the timed ms of modes 0..3 (-1: not run).
// Forces the shape of size range r for an element type (shape -1: tune again
// at the next batch).  For tests and experiments; CHAMELEON_ERR_NOT_SUPPORTED
// when the device cannot run the shape, or it does not apply to the range.
int CHAM_B200_Batch_SetShape(int dtype, int range, int shape) {
    if (range < 0 || range >= NRANGE || shape < -1 || shape >= NSHAPE) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (int rc = ensure_init()) return rc;
    if (int rc = set_attrs()) return rc;
    const bool dbl = dtype != ChamRealFloat;
    if (shape >= 0) {
        if (range > 0 && shape >= 1 && shape <= 3) return CHAMELEON_ERR_NOT_SUPPORTED;
        if (!(dbl ? shape_fits<double>(shape) : shape_fits<float>(shape))) return CHAMELEON_ERR_NOT_SUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[dbl ? 0 : 1].mode[range] = shape;
    return 0;
}

// The batch autotuner's choices for an element type: out[r] = the shape of
// size range r (4 ranges: n <= 64, 65..128, 129..256, 257+; -1 = not tuned
// yet), out[4 + 6 r + k] = the milliseconds shape k took on range r's
// synthetic batch (-1: not admissible).  28 doubles.
int CHAM_B200_Batch_Tuning(int dtype, double *out) {
    if (!out) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const BinTune &tu = g_tune[dtype == ChamRealFloat ? 1 : 0];
    for (int r = 0; r < NRANGE; ++r) {
        out[r] = tu.mode[r];
        for (int k = 0; k < NSHAPE; ++k) out[NRANGE + NSHAPE * r + k] = tu.ms[r][k];
    }
    return 0;
}

}  // extern "C"
