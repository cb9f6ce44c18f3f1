// executor_kernel.cuh -- device side of the persistent tile-DAG executor.
//
// Dispatch by atomic cursor, bounded waits on per-tile counters, the tile
// operations of core.cuh / rec.cuh / tc05.cuh, release by red.release.  Each
// kernel variant (element type x split products x tcgen05 updates) is
// instantiated in its own translation unit (exec_*.cu) so that the variants
// compile in parallel; executor.cu holds the host side.
#pragma once
#include <cuda_runtime.h>

#include "core.cuh"
#include "internal.h"
#include "rec.cuh"
#include "tc05.cuh"

namespace chb {

// ---------------------------------------------------------------------------
// Device
// ---------------------------------------------------------------------------
template <class T>
struct Dims {
    const ExecParams &p;
    __device__ int tm(int m) const { return (m == p.NT - 1) ? p.N - m * p.NB : p.NB; }
    __device__ int nbi(int m) const { return (tm(m) + SUBB - 1) / SUBB; }
    __device__ int S(int m, int n) const {
        const int a = nbi(m), b = nbi(n);
        return (m == n) ? a * (a + 1) / 2 : a * b;
    }
    __device__ int wB(int bn) const { return (bn == p.NTB - 1) ? p.nrhs - bn * p.NBB : p.NBB; }
    // Logical lower tile (m,n), m >= n.
    __device__ ViewT<T> A(int m, int n) const {
        T *a = static_cast<T *>(p.A);
        if (!p.upper) return ViewT<T>{a + p.a_off[m + p.NT * n], 1, p.a_ld[m]};
        return ViewT<T>{a + p.a_off[n + p.NT * m], p.a_ld[n], 1};
    }
    __device__ ViewT<T> Bt(int m, int bn) const {
        return ViewT<T>{static_cast<T *>(p.B) + p.b_off[m + p.NT * bn], 1, p.b_ld[m]};
    }
    // Tile (m, bn) of the forward results (MODE_XINV), layout of B.
    __device__ ViewT<T> Yt(int m, int bn) const {
        return ViewT<T>{static_cast<T *>(p.Y) + p.b_off[m + p.NT * bn], 1, p.b_ld[m]};
    }
    // Sub-tasks a substitution of tile k is split into (its row blocks, MODE_XINV).
    __device__ int nsolve(int k) const { return (p.mode & MODE_XINV) ? nbi(k) : 1; }
    __device__ T *inv(int k) const {
        return static_cast<T *>(p.invd) + (p.full_inv ? (int64_t)k * p.NB * p.NB : (int64_t)k * p.NIB * IB * IB);
    }
    // Full inverse of diagonal tile k (full_inv mode), lower, ld NB.
    __device__ ViewT<T> X(int k) const { return ViewT<T>{inv(k), 1, p.NB}; }
    // Full inverse of diagonal tile k (MODE_XINV), lower, ld NB.
    __device__ ViewT<T> XI(int k) const {
        return ViewT<T>{static_cast<T *>(p.xinv) + (int64_t)k * p.NB * p.NB, 1, p.NB};
    }
};

// Thread 0 only.  Returns false when the run aborted or the wait ran out.
__device__ inline bool wait_geq(const int *ctr, int target, const ExecParams &p, int task) {
    if (ld_acquire(ctr) >= target) return true;
    const uint64_t t0 = globaltimer();
    unsigned ns = 32;
    while (true) {
        if (ld_acquire(ctr) >= target) return true;
        if (*(volatile int *)&p.st->abort) return false;
        if (globaltimer() - t0 > p.wait_budget_ns) {
            atomicCAS(&p.st->error, 0, CHAMELEON_ERR_DEVICE_TIMEOUT);
            atomicExch(&p.st->stuck_task, task);
            atomicExch(&p.st->abort, 1);
            return false;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
}

template <class T>
__device__ bool task_wait(const Task &t, const ExecParams &p, const Dims<T> &d, int ti) {
    const bool fact = p.mode & MODE_FACT;
    switch (t.kind) {
    case TK_POTRF:
        return wait_geq(&p.updA[t.k + p.NT * t.k], t.k * d.S(t.k, t.k), p, ti);
    case TK_TRSM:
        return wait_geq(&p.panA[t.k + p.NT * t.k], 1, p, ti) &&
               wait_geq(&p.updA[t.m + p.NT * t.k], t.k * d.S(t.m, t.k), p, ti);
    case TK_UPD:
        return wait_geq(&p.panA[t.m + p.NT * t.k], d.nbi(t.m), p, ti) &&
               wait_geq(&p.panA[t.n + p.NT * t.k], d.nbi(t.n), p, ti) &&
               wait_geq(&p.updA[t.m + p.NT * t.n], t.k * d.S(t.m, t.n), p, ti);
    case TK_INV:
        return true;
    case TK_XINV:
        return !fact || wait_geq(&p.panA[t.k + p.NT * t.k], 1, p, ti);
    case TK_FWD_TRSM: {
        bool ok = true;
        if (!(p.mode & MODE_XINV)) ok = wait_geq(&p.panA[t.k + p.NT * t.k], 1, p, ti);
        else if (!(p.mode & MODE_NOINV)) ok = wait_geq(&p.xinvDone[t.k], 1, p, ti);
        return ok && wait_geq(&p.fwdB[t.k + p.NT * t.bn], t.k * d.nbi(t.k), p, ti);
    }
    case TK_FWD_UPD:
        return wait_geq(&p.fwdDone[t.k + p.NT * t.bn], d.nsolve(t.k), p, ti) &&
               (!fact || wait_geq(&p.panA[t.m + p.NT * t.k], d.nbi(t.m), p, ti)) &&
               wait_geq(&p.fwdB[t.m + p.NT * t.bn], t.k * d.nbi(t.m), p, ti);
    case TK_BWD_TRSM:
        return wait_geq(&p.fwdDone[t.k + p.NT * t.bn], d.nsolve(t.k), p, ti) &&
               wait_geq(&p.bwdB[t.k + p.NT * t.bn], (p.NT - 1 - t.k) * d.nbi(t.k), p, ti);
    case TK_BWD_UPD:
        return wait_geq(&p.bwdDone[t.k + p.NT * t.bn], d.nsolve(t.k), p, ti) &&
               wait_geq(&p.bwdB[t.m + p.NT * t.bn], (p.NT - 1 - t.k) * d.nbi(t.m), p, ti);
    }
    return false;
}

// Split chunks (hi/lo BF16, swizzled) of panel tile (m,k), m > k.
__device__ __forceinline__ uint8_t *split_tile(const ExecParams &p, int m, int k) {
    const size_t tile_bytes = (size_t)p.split_nrb * p.split_nkc * 2 * tc05::CHUNK_BYTES;
    return p.split + ((size_t)m * (m - 1) / 2 + k) * tile_bytes;
}

template <class T, int SP, bool TC>
__device__ void run_task(const Task &t, const ExecParams &p, const Dims<T> &d, T *smem, tc05::Smem *tsm,
                         uint8_t *stage) {
    using VT = ViewT<T>;
    switch (t.kind) {
    case TK_POTRF: {
        int info;
        if constexpr (std::is_same<T, float>::value) {
            if (p.full_inv) info = rec::tile_potrf_inv<T, SP>(d.A(t.k, t.k), d.X(t.k), d.tm(t.k), smem);
            else info = rec::tile_potrf_blk<T, SP>(d.A(t.k, t.k), d.tm(t.k), d.inv(t.k), smem);
        } else {
            info = rec::tile_potrf_blk<T, SP>(d.A(t.k, t.k), d.tm(t.k), d.inv(t.k), smem);
        }
        if (info && threadIdx.x == 0) {
            atomicMin(&p.st->info, t.k * p.NB + info);
            atomicExch(&p.st->abort, 1);
        }
        break;
    }
    case TK_INV:
        if constexpr (std::is_same<T, float>::value) {
            if (p.full_inv) {
                rec::tile_trtri<T, SP>(d.A(t.k, t.k), d.X(t.k), d.tm(t.k), smem);
                break;
            }
        }
        rec::tile_inv_blk<T>(d.A(t.k, t.k), d.tm(t.k), d.inv(t.k), smem);
        break;
    case TK_TRSM: {
        const int r0 = t.sub * SUBB;
        const int rows = min(SUBB, d.tm(t.m) - r0);
        bool done = false;
        if constexpr (std::is_same<T, float>::value) {
            if (p.full_inv) {
                rec::apply_inv_right<T, SP>(d.A(t.m, t.k).sub(r0, 0), rows, d.X(t.k), d.tm(t.k), smem);
                done = true;
            }
        }
        if (!done) trsm_rows<T, SP>(d.A(t.m, t.k).sub(r0, 0), rows, d.A(t.k, t.k), d.tm(t.k), d.inv(t.k), smem);
        if constexpr (TC) {
            // emit the split-BF16 chunks of these 128 rows for the tcgen05 updates
            const VT X = d.A(t.m, t.k).sub(r0, 0);
            const int K = d.tm(t.k);
            uint8_t *base = split_tile(p, t.m, t.k) + (size_t)t.sub * p.split_nkc * 2 * tc05::CHUNK_BYTES;
            // one thread per (row, group of 8 columns): 16-byte stores
            for (int idx = threadIdx.x; idx < 16 * K; idx += NT_CTA) {
                const int r = idx % 128, c0 = (idx / 128) * 8;
                float v[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) v[e] = (r < rows) ? (float)*X.at(r, c0 + e) : 0.f;
                tc05::split_store8(base + (size_t)(c0 / tc05::BK) * 2 * tc05::CHUNK_BYTES, r, c0 % tc05::BK, v);
            }
            tc05::fence_proxy_async();   // published by the executor's fence + release at task end
            cta_sync();
        }
        break;
    }
    case TK_UPD: {
        const int bi = t.sub & 0xff, bj = (t.sub >> 8) & 0xff;
        const int rows = min(SUBB, d.tm(t.m) - bi * SUBB), cols = min(SUBB, d.tm(t.n) - bj * SUBB);
        const VT C = d.A(t.m, t.n).sub(bi * SUBB, bj * SUBB);
        const bool diag = (t.m == t.n) && (bi == bj);
        if constexpr (TC) {
            const size_t rbytes = (size_t)p.split_nkc * 2 * tc05::CHUNK_BYTES;
            const uint8_t *a = split_tile(p, t.m, t.k) + bi * rbytes;
            const uint8_t *b = split_tile(p, t.n, t.k) + bj * rbytes;
            // C block into L2 while the MMAs run: one prefetch per 128-byte
            // line (32 rows) of each column
            for (int idx = threadIdx.x; idx < 4 * cols; idx += NT_CTA) {
                const int line = idx & 3, c = idx >> 2;
                if (line * 32 < rows) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(C.at(line * 32, c)));
            }
            // epilogue: each thread reads its 64 old values of C first, then
            // subtracts the accumulator 16 columns at a time
            float old[4][16];
            const bool ok = tc05::gemm_bf16x3(
                tsm, stage, a, b, p.split_nkc,
                [&](int r, int c0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
#pragma unroll
                        for (int i = 0; i < 16; ++i) {
                            const int c = c0 + 16 * q + i;
                            old[q][i] = (r < rows && c < cols && (!diag || r >= c)) ? __ldcg(C.at(r, c)) : 0.f;
                        }
                },
                [&](int r, int c0, const float *v, int q) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const int c = c0 + i;
                        if (r < rows && c < cols && (!diag || r >= c)) *C.at(r, c) = old[q][i] - v[i];
                    }
                });
            if (!ok && threadIdx.x == 0) {
                atomicCAS(&p.st->error, 0, CHAMELEON_ERR_DEVICE_TIMEOUT);
                atomicExch(&p.st->abort, 1);
            }
            break;
        }
        Acc<Cfg128<T, SP>> acc;
        acc.zero();
        cta_gemm(acc, d.A(t.m, t.k).sub(bi * SUBB, 0), d.A(t.n, t.k).sub(bj * SUBB, 0), rows, cols,
                 d.tm(t.k), smem);
        acc.sub_from(C, rows, cols, diag);
        break;
    }
    case TK_XINV:
        if constexpr (std::is_same<T, float>::value) rec::tile_trtri<T, SP>(d.A(t.k, t.k), d.XI(t.k), d.tm(t.k), smem);
        break;
    case TK_FWD_TRSM:
    case TK_BWD_TRSM: {
        const VT X = d.Bt(t.k, t.bn);
        const int w = d.wB(t.bn);
        if constexpr (std::is_same<T, float>::value) {
            if (p.mode & MODE_XINV) {
                // row block t.sub of the tile: forward Y_k = X_k B_k, backward B_k = X_k^T Y_k
                const int r0 = t.sub * SUBB, n = d.tm(t.k);
                const int mr = min(SUBB, n - r0);
                const VT Xk = d.XI(t.k);
                const VT Yk = d.Yt(t.k, t.bn);
                for (int c0 = 0; c0 < w; c0 += 64) {
                    const int wc = min(64, w - c0);
                    Acc<Cfg12864<T, SP>> acc;
                    acc.zero();
                    if (t.kind == TK_FWD_TRSM) {
                        cta_gemm(acc, Xk.sub(r0, 0), X.sub(0, c0).t(), mr, wc, r0 + mr, smem);
                        acc.store_to(Yk.sub(r0, c0), mr, wc);
                    } else {
                        cta_gemm(acc, Xk.sub(r0, r0).t(), Yk.sub(r0, c0).t(), mr, wc, n - r0, smem);
                        acc.store_to(X.sub(r0, c0), mr, wc);
                    }
                }
                break;
            }
            if (p.full_inv) {
                const VT Xk = d.X(t.k);
                if (t.kind == TK_FWD_TRSM) rec::apply_inv_left<T, SP, false>(X, w, Xk, d.tm(t.k), smem);
                else rec::apply_inv_left<T, SP, true>(X, w, Xk, d.tm(t.k), smem);
                break;
            }
        }
        for (int c0 = 0; c0 < w; c0 += IB)
            trsm_left<T, SP>(X.sub(0, c0), min(IB, w - c0), d.A(t.k, t.k), d.tm(t.k), d.inv(t.k),
                      t.kind == TK_BWD_TRSM, smem);
        break;
    }
    case TK_FWD_UPD:
    case TK_BWD_UPD: {
        const int r0 = t.sub * SUBB;
        const int rows = min(SUBB, d.tm(t.m) - r0);
        const int w = d.wB(t.bn);
        // MODE_XINV: forward updates read Y_k into B_m, backward ones read B_k into Y_m
        const bool y = p.mode & MODE_XINV;
        const VT Bm = ((y && t.kind == TK_BWD_UPD) ? d.Yt(t.m, t.bn) : d.Bt(t.m, t.bn)).sub(r0, 0);
        const VT Bk = (y && t.kind == TK_FWD_UPD) ? d.Yt(t.k, t.bn) : d.Bt(t.k, t.bn);
        const VT L = (t.kind == TK_FWD_UPD) ? d.A(t.m, t.k).sub(r0, 0) : d.A(t.k, t.m).t().sub(r0, 0);
        for (int c0 = 0; c0 < w; c0 += 64) {
            const int wc = min(64, w - c0);
            Acc<Cfg12864<T, SP>> acc;
            acc.zero();
            cta_gemm(acc, L, Bk.sub(0, c0).t(), rows, wc, d.tm(t.k), smem);
            acc.sub_from(Bm.sub(0, c0), rows, wc, false);
        }
        break;
    }
    }
}

__device__ inline int *task_counter(const Task &t, const ExecParams &p) {
    switch (t.kind) {
    case TK_POTRF:
    case TK_INV: return &p.panA[t.k + p.NT * t.k];
    case TK_XINV: return &p.xinvDone[t.k];
    case TK_TRSM: return &p.panA[t.m + p.NT * t.k];
    case TK_UPD: return &p.updA[t.m + p.NT * t.n];
    case TK_FWD_TRSM: return &p.fwdDone[t.k + p.NT * t.bn];
    case TK_FWD_UPD: return &p.fwdB[t.m + p.NT * t.bn];
    case TK_BWD_TRSM: return &p.bwdDone[t.k + p.NT * t.bn];
    case TK_BWD_UPD: return &p.bwdB[t.m + p.NT * t.bn];
    }
    return nullptr;
}

template <class T, int SP, bool TC>
__global__ void __launch_bounds__(NT_CTA, 1) cholesky_dag_kernel(ExecParams p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned base: the tcgen05 stages need it; other tasks share it
    uint8_t *stage = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    T *smem = reinterpret_cast<T *>(stage);
    __shared__ int s_task;
    __shared__ int s_ok;
    __shared__ tc05::Smem tsm;
    const Dims<T> d{p};
    if constexpr (TC) tc05::init(&tsm);
    while (true) {
        if (threadIdx.x == 0) {
            int ti = -1;
            if (!*(volatile int *)&p.st->abort) {
                ti = atomicAdd(&p.st->next, 1);
                if (ti >= p.ntasks) ti = -1;
            }
            s_task = ti;
            s_ok = (ti >= 0) ? (int)task_wait(p.tasks[ti], p, d, ti) : 0;
        }
        __syncthreads();
        const int ti = s_task;
        if (ti < 0 || !s_ok) break;
        __threadfence();
        const Task t = p.tasks[ti];
        uint64_t t0 = 0;
        if (p.trace && threadIdx.x == 0) t0 = globaltimer();
        run_task<T, SP, TC>(t, p, d, smem, &tsm, stage);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            red_release_add(task_counter(t, p), 1);
            atomicAdd(&p.st->done, 1);
            if (p.trace) {
                unsigned smid;
                asm volatile("mov.u32 %0, %%smid;\n" : "=r"(smid));
                p.trace[ti] = TraceRec{ti, (int)smid, t0, globaltimer()};
            }
        }
    }
    if constexpr (TC) tc05::finish(&tsm);
}

template <class T, int SP, bool TC>
constexpr size_t dag_smem_bytes() {
    return (TC && (size_t)tc05::SMEM_BYTES > tile_smem_bytes<T, SP>() + 1024) ? (size_t)tc05::SMEM_BYTES
                                                                           : tile_smem_bytes<T, SP>() + 1024;
}

// Launch one persistent executor kernel of a variant (its shared-memory size
// attribute is set on first use).
template <class T, int SP, bool TC>
int launch_dag(const ExecParams &p, int grid, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        CHB_CUDA(cudaFuncSetAttribute(cholesky_dag_kernel<T, SP, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)dag_smem_bytes<T, SP, TC>()));
        attr = true;
    }
    cholesky_dag_kernel<T, SP, TC><<<grid, NT_CTA, dag_smem_bytes<T, SP, TC>(), s>>>(p);
    CHB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace chb
