// executor_kernel.cuh -- device side of the persistent tile-DAG executor.
//
// Dispatch by atomic cursor, bounded waits on per-tile counters, the tile
// operations of core.cuh / rec.cuh / tc05.cuh, release by red.release.  Each
// kernel variant (element type x split products x tcgen05 updates) is
// instantiated in its own translation unit (exec_*.cu) so that the variants
// compile in parallel; executor.cu holds the host side.
#pragma once
#include <climits>
#include <cuda_runtime.h>

#include "core.cuh"
#include "internal.h"
#include "potrf_smem.cuh"
#include "rec.cuh"
#include "tc05.cuh"

namespace chb {

// ---------------------------------------------------------------------------
// Device
// ---------------------------------------------------------------------------
// CTAs of the persistent executor per SM: FP64 runs two (16 warps feed the
// DMMA pipe; every FP64 task fits 112 KB of shared memory), FP32 one.
template <class T, bool TC>
constexpr int dag_ctas_per_sm() {
    return (sizeof(T) == 8 && !TC) ? 2 : 1;
}

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
    // Row blocks of tile m in the substitution updates (SOLB rows with MODE_XINV).
    __device__ int nsb(int m) const {
        const int r = solve_rows(p.mode);
        return (tm(m) + r - 1) / r;
    }
    // Sub-tasks a substitution of tile k is split into (its row blocks, MODE_XINV).
    __device__ int nsolve(int k) const { return (p.mode & MODE_XINV) ? nsb(k) : 1; }
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

// The counters a task waits on and the values they must reach (up to three;
// unused entries have a null counter).  bad: unknown task kind.
struct Deps {
    const int *c[3];
    int v[3];
    bool bad;
};

template <class T>
__device__ Deps task_deps(const Task &t, const ExecParams &p, const Dims<T> &d) {
    const bool fact = p.mode & MODE_FACT;
    Deps r{{nullptr, nullptr, nullptr}, {0, 0, 0}, false};
    auto need = [&](int i, const int *c, int v) {
        r.c[i] = c;
        r.v[i] = v;
    };
    switch (t.kind) {
    case TK_POTRF:
        need(0, &p.updA[t.k + p.NT * t.k], upd_ngroups(t.k, p.kgroup, p.utail) * d.S(t.k, t.k));
        if ((p.mode & MODE_CAST) && t.k == 0) need(1, &p.castDone[0], 1);
        break;
    case TK_TRSM:
        need(0, &p.panA[t.k + p.NT * t.k], 1);
        need(1, &p.updA[t.m + p.NT * t.k], upd_ngroups(t.k, p.kgroup, p.utail) * d.S(t.m, t.k));
        // tile column 0 has no update before its panel solve: wait for its cast
        if ((p.mode & MODE_CAST) && t.k == 0) need(1, &p.castDone[t.m], 1);
        break;
    case TK_CAST:
        // copy q delivers tile column q of the logical lower triangle (for
        // Upper storage: block row q of the stored upper triangle)
        need(0, &p.carrive[t.n], p.cepoch);
        break;
    case TK_UPD: {
        // the group's last panel being solved implies the earlier ones are
        // (each panel solve waits for the previous panels' updates of its tile)
        const int kl = t.k + t.bn - 1;
        need(0, &p.panA[t.m + p.NT * kl], d.nbi(t.m));
        need(1, &p.panA[t.n + p.NT * kl], d.nbi(t.n));
        need(2, &p.updA[t.m + p.NT * t.n], t.grp * d.S(t.m, t.n));
        // the first update of a tile is its first reader: wait for its cast
        if ((p.mode & MODE_CAST) && t.grp == 0) need(2, &p.castDone[t.m + p.NT * t.n], 1);
        break;
    }
    case TK_INV:
        break;
    case TK_XINV:
        if (fact) need(0, &p.panA[t.k + p.NT * t.k], 1);
        break;
    case TK_FWD_TRSM:
        if (!(p.mode & MODE_XINV)) need(0, &p.panA[t.k + p.NT * t.k], 1);
        else if (!(p.mode & MODE_NOINV)) need(0, &p.xinvDone[t.k], 1);
        need(1, &p.fwdB[t.k + p.NT * t.bn], t.k * d.nsb(t.k));
        break;
    case TK_FWD_UPD:
        need(0, &p.fwdDone[t.k + p.NT * t.bn], d.nsolve(t.k));
        if (fact) need(1, &p.panA[t.m + p.NT * t.k], d.nbi(t.m));
        need(2, &p.fwdB[t.m + p.NT * t.bn], t.k * d.nsb(t.m));
        break;
    case TK_BWD_TRSM:
        need(0, &p.fwdDone[t.k + p.NT * t.bn], d.nsolve(t.k));
        need(1, &p.bwdB[t.k + p.NT * t.bn], (p.NT - 1 - t.k) * d.nsb(t.k));
        break;
    case TK_BWD_UPD:
        need(0, &p.bwdDone[t.k + p.NT * t.bn], d.nsolve(t.k));
        need(1, &p.bwdB[t.m + p.NT * t.bn], (p.NT - 1 - t.k) * d.nsb(t.m));
        break;
    default:
        r.bad = true;
    }
    return r;
}

// Thread 0 only.  Each round reads every counter of the task and the abort
// flag together (relaxed loads: one memory round trip, where acquire loads
// would serialize); once all counters have reached their values one acquire
// fence orders the task's reads after the producers' releases, and the
// CTA barrier that follows extends that order to every thread.  Returns false
// when the run aborted or the wait ran out.
__device__ __forceinline__ bool deps_met(const Deps &dp) {
    int v[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = dp.c[i] ? ld_relaxed(dp.c[i]) : INT_MAX;
    return v[0] >= dp.v[0] && v[1] >= dp.v[1] && v[2] >= dp.v[2];
}

__device__ inline bool wait_deps(const Deps &dp, const ExecParams &p, int task) {
    if (dp.bad) return false;
    uint64_t t0 = 0;
    unsigned ns = 32;
    while (true) {
        const int ab = ld_relaxed(&p.st->abort);
        if (deps_met(dp)) {
            fence_acq_rel_gpu();
            return true;
        }
        if (ab) return false;
        const uint64_t now = globaltimer();
        if (t0 == 0) {
            t0 = now;
        } else if (now - t0 > p.wait_budget_ns) {
            atomicCAS(&p.st->error, 0, CHAMELEON_ERR_DEVICE_TIMEOUT);
            atomicExch(&p.st->stuck_task, task);
            atomicExch(&p.st->abort, 1);
            return false;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
}

// Split chunks (hi/lo BF16, swizzled) of panel tile (m,k), m > k.
__device__ __forceinline__ uint8_t *split_tile(const ExecParams &p, int m, int k) {
    const size_t tile_bytes = (size_t)p.split_nrb * p.split_nkc * 2 * tc05::CHUNK_BYTES;
    return p.split + ((size_t)m * (m - 1) / 2 + k) * tile_bytes;
}

// TK_CAST: stored tile (p, q) of the FP64 source -> the same tile of the FP32
// A (its stored orientation), plus the tile's share of the symmetric
// infinity norm: absolute row sums go to colsum[p NB + i], column sums to
// colsum[q NB + j] (on a diagonal tile only the referenced triangle counts,
// its diagonal once).  Warp w takes stored rows w*32 + lane (+256, ...) and
// walks the columns: every load is one coalesced 256-byte row segment, read
// through L2 (the copy engine wrote it during this launch).  s_col: NB doubles.
template <class T>
__device__ void cast_tile(const Task &t, const ExecParams &p, const Dims<T> &d, double *s_col) {
    const int P = p.upper ? t.n : t.m, Q = p.upper ? t.m : t.n;   // stored tile
    const int rows = d.tm(P), cols = d.tm(Q);
    const bool diag = (P == Q);
    const double *src = p.csrc + (int64_t)P * p.NB + (int64_t)Q * p.NB * p.csrc_ld;
    T *dst = static_cast<T *>(p.A) + p.a_off[P + p.NT * Q];
    const int ldd = p.a_ld[P];
    for (int j = threadIdx.x; j < cols; j += NT_CTA) s_col[j] = 0.0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int ovf = 0;
    for (int r0 = warp * 32; r0 < rows; r0 += NT_CTA) {
        const int i = r0 + lane;
        const bool rv = i < rows;
        double rs = 0.0;
#pragma unroll 4
        for (int j = 0; j < cols; ++j) {
            const double v = rv ? __ldcg(src + i + (int64_t)j * p.csrc_ld) : 0.0;
            if (rv) dst[i + (int64_t)j * ldd] = (T)v;
            const bool ref = rv && (!diag || (p.upper ? i <= j : i >= j));
            const double av = ref ? fabs(v) : 0.0;
            ovf |= av > 3.4028234663852886e38;
            if (!diag || i != j) rs += av;
            double cs = av;
#pragma unroll
            for (int o = 16; o; o >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, o);
            if (lane == 0 && cs != 0.0) atomicAdd(&s_col[j], cs);
        }
        if (rv && rs != 0.0) atomicAdd(&p.colsum[(int64_t)P * p.NB + i], rs);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cols; j += NT_CTA)
        if (s_col[j] != 0.0) atomicAdd(&p.colsum[(int64_t)Q * p.NB + j], s_col[j]);
    if (ovf) atomicOr(p.covf, 1);
}

// Look-ahead of the dispatch loop, in shared memory.  A tcgen05 update task
// does the dispatch work of the next task on a thread that is idle while the
// copies and MMAs run: it claims the next cursor position, loads that task's
// descriptor and checks its dependencies once (acquire fence if met), so the
// dispatch round trips overlap the task; thread 0 consumes the result at the
// top of the loop.  When the next task is a tcgen05 update that is ready, the
// finished task's release is handed to that idle thread too (rel), so that
// thread 0 does not stall on the release fence between tasks; the hand-over
// cannot delay a dependency of the next task, which was met without it.
struct Ahead {
    int raw;     // cursor value claimed ahead (INT_MIN: none)
    int have;    // t holds the descriptor of task raw
    int ready;   // its dependencies were met (acquire fence done)
    int *rel;    // counter whose release the next task performs (or null)
    Task t;
};

template <class T, int SP, bool TC>
__device__ void run_task(const Task &t, const ExecParams &p, const Dims<T> &d, T *smem, tc05::Smem *tsm,
                         uint8_t *stage, unsigned *ph, Ahead *ah) {
    using VT = ViewT<T>;
    switch (t.kind) {
    case TK_POTRF: {
        int info;
        if constexpr (std::is_same<T, float>::value) {
            if (p.full_inv) info = rec::tile_potrf_inv<T, SP>(d.A(t.k, t.k), d.X(t.k), d.tm(t.k), smem);
            else if (d.tm(t.k) <= psm::MAXN) info = psm::potrf(d.A(t.k, t.k), d.tm(t.k), d.inv(t.k), smem, ph);
            else info = rec::tile_potrf_blk<T, SP>(d.A(t.k, t.k), d.tm(t.k), d.inv(t.k), smem, ph);
        } else {
            // FP64: the lean form (64-row panels, leaf on the staging area) fits
            // the two-CTAs-per-SM shared memory
            info = rec::tile_potrf_blk<T, SP, 64, true>(d.A(t.k, t.k), d.tm(t.k), d.inv(t.k), smem, ph);
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
            // the split tiles of panels k .. k + bn - 1 of one tile row are
            // consecutive in the split buffer (index m(m-1)/2 + k)
            const size_t rbytes = (size_t)p.split_nkc * 2 * tc05::CHUNK_BYTES;
            const size_t tstride = (size_t)p.split_nrb * rbytes;
            const uint8_t *a = split_tile(p, t.m, t.k) + bi * rbytes;
            const uint8_t *b = split_tile(p, t.n, t.k) + bj * rbytes;
            // warps 4-7 stage the old C block in TMEM while the MMAs run; the
            // epilogue subtracts the accumulator from it
            auto owned = [&](int r, int c) { return r < rows && c < cols && (!diag || r >= c); };
            const bool ok = tc05::gemm_bf16x3_sub(
                tsm, stage, a, b, p.split_nkc, t.bn, tstride,
                [&](int r, int c) { return owned(r, c) ? __ldcg(C.at(r, c)) : 0.f; },
                [&](int r, int c, float v) {
                    if (owned(r, c)) *C.at(r, c) = v;
                },
                [&]() {
                    if (ah->rel) {
                        red_release_add(ah->rel, 1);
                        ah->rel = nullptr;
                    }
                    if (p.npotrf > 0) return;   // the dedicated-POTRF dispatch claims by itself
                    const int raw = atomicAdd(&p.st->next, 1);
                    int ready = 0;
                    if (raw < p.ntasks) {
                        const Task nt = p.tasks[raw];
                        ah->t = nt;
                        const Deps dp = task_deps(nt, p, d);
                        if (!dp.bad && deps_met(dp)) {
                            fence_acq_rel_gpu();
                            ready = 1;
                        }
                    }
                    ah->have = raw < p.ntasks;
                    ah->ready = ready;
                    ah->raw = raw;
                },
                ph);
            if (!ok && threadIdx.x == 0) {
                atomicCAS(&p.st->error, 0, CHAMELEON_ERR_DEVICE_TIMEOUT);
                atomicExch(&p.st->abort, 1);
            }
            break;
        }
        if constexpr (sizeof(T) == 8) {
            // FP64: two 128 x 64 halves (the 111 KB of stages that let two
            // CTAs share an SM); on a diagonal block the second half is the
            // 64 x 64 lower block of rows and columns 64..127
            for (int h = 0; h < 2; ++h) {
                const int c0 = 64 * h, r0 = diag ? c0 : 0;
                if (c0 >= cols || r0 >= rows) break;
                Acc<Cfg12864<T, SP>> acc;
                acc.zero();
                for (int k = t.k; k < t.k + t.bn; ++k)
                    cta_gemm(acc, d.A(t.m, k).sub(bi * SUBB + r0, 0), d.A(t.n, k).sub(bj * SUBB + c0, 0), rows - r0,
                             min(64, cols - c0), d.tm(k), smem);
                acc.sub_from(C.sub(r0, c0), rows - r0, min(64, cols - c0), diag);
            }
        } else {
            Acc<Cfg128<T, SP>> acc;
            acc.zero();
            for (int k = t.k; k < t.k + t.bn; ++k)
                cta_gemm(acc, d.A(t.m, k).sub(bi * SUBB, 0), d.A(t.n, k).sub(bj * SUBB, 0), rows, cols, d.tm(k),
                         smem);
            acc.sub_from(C, rows, cols, diag);
        }
        break;
    }
    case TK_XINV:
        if constexpr (std::is_same<T, float>::value) rec::tile_trtri<T, SP>(d.A(t.k, t.k), d.XI(t.k), d.tm(t.k), smem);
        break;
    case TK_CAST:
        if constexpr (std::is_same<T, float>::value) cast_tile(t, p, d, reinterpret_cast<double *>(smem));
        break;
    case TK_FWD_TRSM:
    case TK_BWD_TRSM: {
        const VT X = d.Bt(t.k, t.bn);
        const int w = d.wB(t.bn);
        if constexpr (std::is_same<T, float>::value) {
            if (p.mode & MODE_XINV) {
                // row block t.sub (SOLB rows) of the tile: forward Y_k = X_k B_k,
                // backward B_k = X_k^T Y_k
                const int r0 = t.sub * SOLB, n = d.tm(t.k);
                const int mr = min(SOLB, n - r0);
                const VT Xk = d.XI(t.k);
                const VT Yk = d.Yt(t.k, t.bn);
                for (int c0 = 0; c0 < w; c0 += 64) {
                    const int wc = min(64, w - c0);
                    Acc<Cfg64<T, SP>> acc;
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
        for (int c0 = 0; c0 < w; c0 += IB) {
            const int wc = min(IB, w - c0);
            if (wc <= Cfg64N<T, SP>::BN)   // few right-hand sides: the narrow tile
                trsm_left<T, SP, Cfg64N<T, SP>>(X.sub(0, c0), wc, d.A(t.k, t.k), d.tm(t.k), d.inv(t.k),
                                                t.kind == TK_BWD_TRSM, smem);
            else
                trsm_left<T, SP>(X.sub(0, c0), wc, d.A(t.k, t.k), d.tm(t.k), d.inv(t.k), t.kind == TK_BWD_TRSM,
                                 smem);
        }
        break;
    }
    case TK_FWD_UPD:
    case TK_BWD_UPD: {
        // MODE_XINV: forward updates read Y_k into B_m, backward ones read B_k
        // into Y_m, in SOLB-row blocks
        const bool y = p.mode & MODE_XINV;
        const int rb = y ? SOLB : SUBB;
        const int r0 = t.sub * rb;
        const int rows = min(rb, d.tm(t.m) - r0);
        const int w = d.wB(t.bn);
        const VT Bm = ((y && t.kind == TK_BWD_UPD) ? d.Yt(t.m, t.bn) : d.Bt(t.m, t.bn)).sub(r0, 0);
        const VT Bk = (y && t.kind == TK_FWD_UPD) ? d.Yt(t.k, t.bn) : d.Bt(t.k, t.bn);
        const VT L = (t.kind == TK_FWD_UPD) ? d.A(t.m, t.k).sub(r0, 0) : d.A(t.k, t.m).t().sub(r0, 0);
        for (int c0 = 0; c0 < w; c0 += 64) {
            const int wc = min(64, w - c0);
            if (y) {
                Acc<Cfg64<T, SP>> acc;
                acc.zero();
                cta_gemm(acc, L, Bk.sub(0, c0).t(), rows, wc, d.tm(t.k), smem);
                acc.sub_from(Bm.sub(0, c0), rows, wc, false);
            } else {
                Acc<Cfg12864<T, SP>> acc;
                acc.zero();
                cta_gemm(acc, L, Bk.sub(0, c0).t(), rows, wc, d.tm(t.k), smem);
                acc.sub_from(Bm.sub(0, c0), rows, wc, false);
            }
        }
        break;
    }
    }
}

__device__ inline int *task_counter(const Task &t, const ExecParams &p) {
    switch (t.kind) {
    case TK_CAST: return &p.castDone[t.m + p.NT * t.n];
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
__global__ void __launch_bounds__(NT_CTA, dag_ctas_per_sm<T, TC>()) cholesky_dag_kernel(ExecParams p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned base: the tcgen05 stages need it; other tasks share it
    // (an offset added to the __shared__ array, not a rounded integer: the
    // pointer stays visibly in shared memory, so every access through it is
    // an ld/st.shared rather than a generic load or store)
    uint8_t *stage = smem_raw + ((1024u - (unsigned)(reinterpret_cast<uintptr_t>(smem_raw) & 1023u)) & 1023u);
    T *smem = reinterpret_cast<T *>(stage);
    __shared__ int s_task;
    __shared__ int s_ok;
    __shared__ tc05::Smem tsm;
    __shared__ unsigned s_ph[3];   // phase cycles of the current task (tracing only)
    const Dims<T> d{p};
    if constexpr (TC) tc05::init(&tsm);
    __shared__ Task s_desc;
    uint64_t tg = 0;
    const bool potrf_cta = p.npotrf > 0 && blockIdx.x == 0;
    int pnext = 0;   // thread 0 of the POTRF CTA: next entry of potrf_idx
    int ndone = 0;   // thread 0: tasks this CTA completed
    __shared__ Ahead ah;   // task claimed ahead by the previous task
    if (threadIdx.x == 0) {
        ah.raw = INT_MIN;
        ah.have = ah.ready = 0;
        ah.rel = nullptr;
    }
    while (true) {
        if (threadIdx.x == 0) {
            int ti;
            if (ah.raw != INT_MIN) {
                ti = (ah.raw < p.ntasks) ? ah.raw : -1;
            } else if (potrf_cta) {
                ti = (pnext < p.npotrf) ? p.potrf_idx[pnext++] : -1;
            } else {
                do {
                    ti = atomicAdd(&p.st->next, 1);
                } while (p.npotrf > 0 && ti < p.ntasks && p.tasks[ti].kind == TK_POTRF);
                if (ti >= p.ntasks) ti = -1;
            }
            if (p.trace) {
                tg = globaltimer();
                s_ph[0] = s_ph[1] = s_ph[2] = 0u;
            }
            bool ok = false;
            if (ti >= 0) {
                const Task t = ah.have ? ah.t : p.tasks[ti];
                s_desc = t;
                ok = ah.ready || wait_deps(task_deps(t, p, d), p, ti);
            }
            ah.raw = INT_MIN;
            ah.have = ah.ready = 0;
            s_task = ti;
            s_ok = ok;
        }
        __syncthreads();
        const int ti = s_task;
        if (ti < 0 || !s_ok) break;
        const Task t = s_desc;
        uint64_t t0 = 0;
        if (p.trace && threadIdx.x == 0) t0 = globaltimer();
        run_task<T, SP, TC>(t, p, d, smem, &tsm, stage, p.trace ? s_ph : nullptr, &ah);
        // Every thread's writes of the task precede thread 0's release through
        // the barrier (the release is cumulative), so no per-thread fence.
        __syncthreads();
        if (threadIdx.x == 0) {
            int *ctr = task_counter(t, p);
            if (TC && ah.ready && ah.t.kind == TK_UPD) ah.rel = ctr;   // released by the next task
            else red_release_add(ctr, 1);
            ++ndone;
            if (p.trace) {
                unsigned smid;
                asm volatile("mov.u32 %0, %%smid;\n" : "=r"(smid));
                p.trace[ti] = TraceRec{ti, (int)smid, t0, globaltimer(), (uint32_t)(t0 - tg),
                                       {s_ph[0], s_ph[1], s_ph[2]}};
            }
        }
    }
    if (threadIdx.x == 0 && ndone) atomicAdd(&p.st->done, ndone);
    if constexpr (TC) tc05::finish(&tsm);
}

template <class T, int SP, bool TC>
constexpr size_t dag_smem_bytes() {
    // FP64: two CTAs per SM, each task within a 128 x 64 DMMA tile's stages
    if (sizeof(T) == 8 && !TC) return Cfg12864<T, SP>::SMEM_BYTES + 1024;
    // one CTA per SM: every variant may use the shared memory its largest task needs
    // (the tcgen05 stages; FP32: the shared-memory diagonal-tile factorization)
    size_t b = tile_smem_bytes<T, SP>() + 1024;
    if (TC && (size_t)tc05::SMEM_BYTES > b) b = tc05::SMEM_BYTES;
    if (std::is_same<T, float>::value && psm::SMEM_BYTES + 1024 > b) b = psm::SMEM_BYTES + 1024;
    return b;
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
