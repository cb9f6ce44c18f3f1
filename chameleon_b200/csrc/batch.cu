// batch.cu -- batched Cholesky on independent matrices.
//
// Reference: CHAMELEON_dpotrf_batch_Tile / CHAMELEON_dtrsm_batch_Tile
// (compute/zpotrf_batch.c:28-118, compute/ztrsm_batch.c:37-213) map one CPU task
// per tile through chameleon_pmap (compute/pmap.c:25-93); potrf has no GPU
// path there (`.cudafunc = NULL`, zpotrf_batch.c:58-64).  Here a batch is split
// into two size bins, each ONE persistent launch where a CTA takes the next
// system from an atomic cursor (largest first, so the long tail starts early):
//
//   * n > 64: the tile routines (64-wide leaf Cholesky, panel GEMMs on the
//     tensor cores, inverted diagonal blocks in a per-CTA scratch slot), one
//     256-thread CTA per SM;
//   * n <= 64: the whole system in shared memory -- leaf Cholesky + inverse,
//     then X = L^-T L^-1 B by two small products -- with a footprint that lets
//     several CTAs share an SM.  How the small bin runs (the generic kernel, or
//     the small kernel at 1..3 CTAs per SM) is chosen once per device and
//     element type by timing each option on synthetic systems (autotune_small).
//
// The small bin runs on a side stream, so its CTAs fill SMs as the large bin's
// tail drains.  CHAM_B200_dposv_batch / sposv_batch (uneven sizes, no
// reference equivalent: the reference batch API is uniform-size) capture the
// whole sequence in a CUDA graph per batch signature and replay it when the
// same batch comes again.
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
template <class T>
__global__ void __launch_bounds__(NT_CTA, 1) posv_batch_kernel(const BatchItem *items, int count, T *A, T *B,
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
        const int r = rec::tile_potrf_blk<T, SPLIT_BF16X3>(Lv, it.n, invd, smem);
        if (threadIdx.x == 0 && info) info[it.info_idx] = r;
        if (r == 0 && it.nrhs > 0) {
            const ViewT<T> X{B + it.b_off, 1, it.ldb};
            for (int c0 = 0; c0 < it.nrhs; c0 += IB) {
                const int w = min(IB, it.nrhs - c0);
                trsm_left<T, SPLIT_BF16X3>(X.sub(0, c0), w, Lv, it.n, invd, false, smem);
                trsm_left<T, SPLIT_BF16X3>(X.sub(0, c0), w, Lv, it.n, invd, true, smem);
            }
        }
        cta_sync_global();
    }
}

// Small bin (n <= 64): system in shared memory.  sD holds the identity-padded
// block, then L, then the right-hand sides being solved; sX the inverse.
template <class T>
constexpr size_t small_smem_bytes() {
    return 2 * 64 * rec::LDS * sizeof(T);
}
template <class T>
constexpr int small_min_blocks() {
    return sizeof(T) == 8 ? 2 : 3;
}
template <class T>
__global__ void __launch_bounds__(NT_CTA, small_min_blocks<T>())
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
        const int r = rec::leaf64_core<T, true>(sD, sX);
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
            T y[16];
            // Y = X B (X lower, zero above the diagonal, identity beyond n)
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int idx = tid + NT_CTA * q, rr = idx & 63, cc = idx >> 6;
                T acc = T(0);
#pragma unroll 8
                for (int k = 0; k < 64; ++k) acc += sX[rr + k * LDS] * sD[k + cc * LDS];
                y[q] = acc;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int idx = tid + NT_CTA * q;
                sD[(idx & 63) + (idx >> 6) * LDS] = y[q];
            }
            __syncthreads();
            // X_out = X^T Y
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int idx = tid + NT_CTA * q, rr = idx & 63, cc = idx >> 6;
                T acc = T(0);
#pragma unroll 8
                for (int k = 0; k < 64; ++k) acc += sX[k + rr * LDS] * sD[k + cc * LDS];
                if (rr < n && cc < w) Bc[rr + (int64_t)cc * it.ldb] = acc;
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
    if (!ws.cursor && !(ws.cursor = (int *)dev_alloc(2 * sizeof(int)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
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
    CHB_CUDA(cudaFuncSetAttribute(posv_small_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)small_smem_bytes<double>()));
    CHB_CUDA(cudaFuncSetAttribute(posv_small_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)small_smem_bytes<float>()));
    CHB_CUDA(cudaFuncSetAttribute(trsm_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)TILE_KERNEL_SMEM_BYTES));
    g_attr = true;
    return 0;
}

// How the small bin runs: 0 = generic kernel, k >= 1 = small kernel with k CTAs
// per SM.  Chosen by autotune_small (per element type), times kept for reporting.
struct SmallTune {
    int mode = -1;
    float ms[4] = {-1.f, -1.f, -1.f, -1.f};
};
SmallTune g_tune[2];   // [0] double, [1] float
std::mutex g_tune_mu;

template <class T>
constexpr int tidx() {
    return sizeof(T) == 8 ? 0 : 1;
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

template <class T>
int launch_bins(const BatchItem *d_items, int nlarge, int nsmall, int nmax_large, T *A, T *B, int upper, int *info,
                cudaStream_t s, BatchWs &ws, int mode);

// Time each way of running a small bin on 4096 synthetic systems (n ~ U{16..64},
// 4 right-hand sides) and keep the fastest.  Once per device and element type.
template <class T>
int autotune_small(cudaStream_t s, BatchWs &ws) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    SmallTune &tu = g_tune[tidx<T>()];
    if (tu.mode >= 0) return 0;
    const int cnt = 4096, k = 4;
    std::vector<BatchItem> items(cnt);
    int64_t oa = 0, ob = 0;
    uint32_t st = 12345u;
    for (int i = 0; i < cnt; ++i) {
        st = st * 1664525u + 1013904223u;
        const int n = 16 + (int)((st >> 8) % 49);
        items[i] = BatchItem{oa, ob, n, k, n, n, i, 0};
        oa += (int64_t)n * n;
        ob += (int64_t)n * k;
    }
    std::sort(items.begin(), items.end(), [](const BatchItem &a, const BatchItem &b) { return a.n > b.n; });
    T *A = (T *)dev_alloc(oa * sizeof(T)), *B = (T *)dev_alloc(ob * sizeof(T));
    BatchItem *d_items = (BatchItem *)dev_alloc(cnt * sizeof(BatchItem));
    int *d_info = (int *)dev_alloc(cnt * sizeof(int));
    cudaEvent_t e0, e1;
    int rc = (A && B && d_items && d_info) ? 0 : CHAMELEON_ERR_OUT_OF_RESOURCES;
    if (!rc) rc = (cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) ? 0 : CHAMELEON_ERR_UNEXPECTED;
    if (!rc && cudaMemcpyAsync(d_items, items.data(), cnt * sizeof(BatchItem), cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = CHAMELEON_ERR_UNEXPECTED;
    int occ = 1;
    if (!rc) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, posv_small_kernel<T>, NT_CTA, small_smem_bytes<T>());
    int best = 0;
    float best_ms = 1e30f;
    for (int mode = 0; mode <= std::min(3, occ) && !rc; ++mode) {
        float t = 0.f;
        for (int rep = 0; rep < 2 && !rc; ++rep) {   // rep 0 warms the kernel up
            tune_fill_kernel<T><<<cnt, 128, 0, s>>>(d_items, cnt, A, B);
            cudaEventRecord(e0, s);
            rc = launch_bins<T>(d_items, 0, cnt, 0, A, B, 0, d_info, s, ws, mode);
            cudaEventRecord(e1, s);
            if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = CHAMELEON_ERR_UNEXPECTED;
            if (!rc) cudaEventElapsedTime(&t, e0, e1);
        }
        tu.ms[mode] = t;
        if (!rc && t < best_ms) {
            best_ms = t;
            best = mode;
        }
    }
    cudaStreamSynchronize(s);
    dev_free(A);
    dev_free(B);
    dev_free(d_items);
    dev_free(d_info);
    if (rc) return rc;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tu.mode = best;
    return 0;
}

// Launch the two bins: items [0, nlarge) (n > 64, largest first) on the generic
// kernel on `s`, items [nlarge, nlarge + nsmall) on the side stream per `mode`;
// `s` waits for both.  Only stream operations (capturable).
template <class T>
int launch_bins(const BatchItem *d_items, int nlarge, int nsmall, int nmax_large, T *A, T *B, int upper, int *info,
                cudaStream_t s, BatchWs &ws, int mode) {
    const int sms = ctx().num_sms;
    const int nib = std::max(1, (std::max(nmax_large, 64) + IB - 1) / IB);
    CHB_CUDA(cudaMemsetAsync(ws.cursor, 0, 2 * sizeof(int), s));
    if (nsmall > 0 && mode >= 1) {
        CHB_CUDA(cudaEventRecord(ws.fork, s));
        CHB_CUDA(cudaStreamWaitEvent(ws.side, ws.fork, 0));
        const int grid = std::min(sms * mode, nsmall);
        posv_small_kernel<T><<<grid, NT_CTA, small_smem_bytes<T>(), ws.side>>>(d_items + nlarge, nsmall, A, B,
                                                                                 upper, info, ws.cursor + 1);
        CHB_LAUNCHED(1);
        CHB_CUDA(cudaGetLastError());
        CHB_CUDA(cudaEventRecord(ws.join, ws.side));
    }
    // the generic kernel runs the large bin, and the small bin too when mode == 0
    const int ngen = nlarge + ((mode == 0) ? nsmall : 0);
    if (ngen > 0) {
        const int grid = std::min(sms, ngen);
        posv_batch_kernel<T><<<grid, NT_CTA, tile_smem_bytes<T>(), s>>>(d_items, ngen, A, B, upper, info, ws.cursor,
                                                                      (T *)ws.scratch, nib);
        CHB_LAUNCHED(1);
        CHB_CUDA(cudaGetLastError());
    }
    if (nsmall > 0 && mode >= 1) CHB_CUDA(cudaStreamWaitEvent(s, ws.join, 0));
    return 0;
}

// Host items -> bins (sorted largest first within each bin), device upload of
// the item list to `d_items` (capacity checked by the caller).
void make_bins(std::vector<BatchItem> &items, int *nlarge, int *nsmall, int *nmax_large) {
    std::stable_sort(items.begin(), items.end(), [](const BatchItem &a, const BatchItem &b) { return a.n > b.n; });
    int nl = 0;
    while (nl < (int)items.size() && items[nl].n > 64) ++nl;
    *nlarge = nl;
    *nsmall = (int)items.size() - nl;
    *nmax_large = nl ? items[0].n : 0;
}

template <class T>
int prepare(BatchWs &ws, cudaStream_t s, size_t nitems, int nmax) {
    if (int rc = set_attrs()) return rc;
    if (!ws.side) {
        CHB_CUDA(cudaStreamCreateWithFlags(&ws.side, cudaStreamNonBlocking));
        CHB_CUDA(cudaEventCreateWithFlags(&ws.fork, cudaEventDisableTiming));
        CHB_CUDA(cudaEventCreateWithFlags(&ws.join, cudaEventDisableTiming));
    }
    const int nib = std::max(1, (std::max(nmax, 64) + IB - 1) / IB);
    if (int rc = bws_reserve(ws, nitems * sizeof(BatchItem), (size_t)ctx().num_sms * nib * IB * IB * sizeof(T), 1))
        return rc;
    return autotune_small<T>(s, ws);
}
}  // namespace

// Launch the factor(+solve) batch over host-described items (binned and sorted
// here, largest first).  `info` is a device array indexed by item.info_idx (or null).
template <class T>
int launch_posv_batch_t(std::vector<BatchItem> &items, T *A, T *B, int upper, int *info, cudaStream_t s,
                        BatchWs &ws) {
    if (items.empty()) return 0;
    int nl, ns, nmax;
    make_bins(items, &nl, &ns, &nmax);
    if (int rc = prepare<T>(ws, s, items.size(), nmax)) return rc;
    CHB_CUDA(cudaMemcpyAsync(ws.items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, s));
    return launch_bins<T>((const BatchItem *)ws.items, nl, ns, nmax, A, B, upper, info, s, ws,
                          g_tune[tidx<T>()].mode);
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
    int nl, ns, nmax;
    make_bins(items, &nl, &ns, &nmax);
    if (int rc = prepare<T>(ws, s, items.size(), nmax)) return rc;
    const int mode = g_tune[tidx<T>()].mode;
    uint64_t key = 1469598103934665603ull;
    key = fnv(key, items.data(), items.size() * sizeof(BatchItem));
    const void *ptrs[4] = {A, B, info, ws.scratch};
    const int ints[5] = {upper, count, mode, (int)sizeof(T), (int)items.size()};
    key = fnv(key, ptrs, sizeof ptrs);
    key = fnv(key, ints, sizeof ints);
    std::lock_guard<std::mutex> lk(g_graph_mu);
    for (auto it = g_graphs.begin(); it != g_graphs.end(); ++it) {
        if (it->key != key) continue;
        g_graphs.splice(g_graphs.begin(), g_graphs, it);
        CHB_LAUNCHED(ns > 0 && mode >= 1 ? 2 : 1);
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
    const int rcl = launch_bins<T>(g.d_items, nl, ns, nmax, A, B, upper, info, s, ws, mode);
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
int CHAM_B200_Batch_Tuning(int dtype, double *out) {
    if (!out) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const SmallTune &tu = g_tune[dtype == ChamRealFloat ? 1 : 0];
    out[0] = tu.mode;
    for (int m = 0; m < 4; ++m) out[1 + m] = tu.ms[m];
    return 0;
}

}  // extern "C"
