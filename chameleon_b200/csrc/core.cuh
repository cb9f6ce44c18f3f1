// core.cuh -- device building blocks of the B200 tile kernels (FP64 path).
//
// Every tile operation of the Cholesky path (reference: the POTRF / TRSM /
// SYRK / GEMM tile kernels of coreblas and gpucublas, e.g.
// coreblas/compute/core_zpotrf.c:75-81, gpucublas/compute/cuda_zgemm.c:24-45)
// is expressed here with three CTA-wide primitives:
//
//   cta_gemm      acc(i,j) += sum_k A(i,k) * B(j,k)  ("NT" form) on FP64 DMMA
//                 (mma.sync m8n8k4 f64) with operands staged global -> shared
//                 by cp.async, two-stage pipeline, any operand orientation;
//   blk_potrf     Cholesky of a <=64 x 64 block in shared memory, plus the
//                 explicit inverse of its triangular factor;
//   trsm_rows / trsm_left   blocked triangular solves that use the inverted
//                 64 x 64 diagonal blocks so that all bulk work is GEMM-shaped.
//
// Matrices are addressed through View: element (i,j) at p[i*rs + j*cs].  A
// column-major tile with leading dimension ld is {p, 1, ld}; its transpose is
// {p, ld, 1}.  This is how the Upper variants become the Lower algorithm on
// transposed views (Upper tile (n,m) == transpose of Lower tile (m,n)).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace chb {

constexpr int NT_CTA = 256;   // threads per CTA of every tile kernel
constexpr int KC     = 32;    // k-extent of one pipeline stage
constexpr int IB     = 64;    // inner block of POTRF / TRSM (inverted diagonal blocks)
constexpr int PAD_MN = 8;     // shared-memory pad for M/N-contiguous stages
constexpr int LDK    = KC + 4;// shared-memory leading dimension of K-contiguous stages

struct View {
    double *p;
    int64_t rs, cs;
    __device__ __forceinline__ double *at(int i, int j) const { return p + (int64_t)i * rs + (int64_t)j * cs; }
    __device__ __forceinline__ View sub(int i, int j) const { return View{at(i, j), rs, cs}; }
    __device__ __forceinline__ View t() const { return View{p, cs, rs}; }
};

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, int src_bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(int *p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
// Make this CTA's global writes visible at GPU scope (they are re-read through
// L2 by cp.async.cg), then join the CTA.
__device__ __forceinline__ void cta_sync_global() {
    __threadfence();
    __syncthreads();
}
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Stage loader: a (rows x KC) slab of operand V (rows < M, k0 <= k < min(K,
// k0+KC)) into shared memory.  KMAJ = false: layout [k][row] with leading
// dimension ROWS+PAD_MN (V.rs == 1).  KMAJ = true: layout [row][k] with leading
// dimension LDK (V.cs == 1).  Out-of-range elements are zero-filled.  ALIGNED:
// 16-byte cp.async of element pairs (base 16-byte aligned, non-unit stride
// even); otherwise one 8-byte cp.async per element.
// ---------------------------------------------------------------------------
template <int ROWS, bool KMAJ>
__device__ __forceinline__ void load_stage(double *s, const View &V, int M, int K, int k0, bool aligned) {
    const int tid = threadIdx.x;
    if (!KMAJ) {
        constexpr int LD = ROWS + PAD_MN;
        constexpr int PAIRS = ROWS / 2;
        for (int idx = tid; idx < KC * PAIRS; idx += NT_CTA) {
            const int kk = idx / PAIRS, i = 2 * (idx % PAIRS);
            const int gk = k0 + kk;
            const double *src = V.p + i + (int64_t)gk * V.cs;
            double *dst = s + kk * LD + i;
            const bool kin = gk < K;
            if (aligned) {
                const int nb = (kin && i < M) ? ((i + 1 < M) ? 16 : 8) : 0;
                cp_async16(dst, nb ? src : V.p, nb);
            } else {
                const int b0 = (kin && i < M) ? 8 : 0, b1 = (kin && i + 1 < M) ? 8 : 0;
                cp_async8(dst, b0 ? src : V.p, b0);
                cp_async8(dst + 1, b1 ? src + 1 : V.p, b1);
            }
        }
    } else {
        constexpr int KP = KC / 2;
        for (int idx = tid; idx < ROWS * KP; idx += NT_CTA) {
            const int i = idx / KP, kk = 2 * (idx % KP);
            const int gk = k0 + kk;
            const double *src = V.p + (int64_t)i * V.rs + gk;
            double *dst = s + i * LDK + kk;
            const bool iin = i < M;
            if (aligned) {
                const int nb = (iin && gk < K) ? ((gk + 1 < K) ? 16 : 8) : 0;
                cp_async16(dst, nb ? src : V.p, nb);
            } else {
                const int b0 = (iin && gk < K) ? 8 : 0, b1 = (iin && gk + 1 < K) ? 8 : 0;
                cp_async8(dst, b0 ? src : V.p, b0);
                cp_async8(dst + 1, b1 ? src + 1 : V.p, b1);
            }
        }
    }
}

template <int ROWS, bool KMAJ>
__device__ __forceinline__ double frag(const double *s, int row, int kk) {
    if (KMAJ) return s[row * LDK + kk];
    return s[kk * (ROWS + PAD_MN) + row];
}

template <int ROWS, bool KMAJ>
__host__ __device__ constexpr int stage_elems() {
    return KMAJ ? ROWS * LDK : KC * (ROWS + PAD_MN);
}
template <int ROWS>
__host__ __device__ constexpr int stage_elems_max() {
    return ROWS * LDK > KC * (ROWS + PAD_MN) ? ROWS * LDK : KC * (ROWS + PAD_MN);
}

// Tile configuration of cta_gemm: BM x BN outputs, WM x WN warps (8 warps).
template <int BM_, int BN_, int WM_, int WN_>
struct GemmCfg {
    static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_;
    static constexpr int WTM = BM / WM, WTN = BN / WN;
    static constexpr int FM = WTM / 8, FN = WTN / 8;
    static_assert(WM * WN * 32 == NT_CTA, "8 warps");
    static constexpr int SA = stage_elems_max<BM>(), SB = stage_elems_max<BN>();
    static constexpr int SMEM_ELEMS = 2 * (SA + SB);   // two pipeline stages
    static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_ELEMS;
};
using Cfg128 = GemmCfg<128, 128, 2, 4>;  // trailing-update sub-blocks
using Cfg12864 = GemmCfg<128, 64, 4, 2>; // panel rows x one inner block
using Cfg64 = GemmCfg<64, 64, 2, 4>;     // inner block x inner block

template <class C>
struct Acc {
    double v[C::FM][C::FN][2];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int a = 0; a < C::FM; ++a)
#pragma unroll
            for (int b = 0; b < C::FN; ++b) v[a][b][0] = v[a][b][1] = 0.0;
    }
    // f(row, col, value) for every accumulator element owned by this thread.
    template <class F>
    __device__ __forceinline__ void for_each(F &&f) const {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int wm = warp / C::WN, wn = warp % C::WN;
#pragma unroll
        for (int a = 0; a < C::FM; ++a)
#pragma unroll
            for (int b = 0; b < C::FN; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int r = wm * C::WTM + a * 8 + (lane >> 2);
                    const int c = wn * C::WTN + b * 8 + 2 * (lane & 3) + e;
                    f(r, c, v[a][b][e]);
                }
    }
};

template <class C, bool AK, bool BK>
__device__ __forceinline__ void mma_stage(Acc<C> &acc, const double *sA, const double *sB) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp / C::WN, wn = warp % C::WN;
    const int r0 = wm * C::WTM + (lane >> 2), c0 = wn * C::WTN + (lane >> 2), kq = lane & 3;
#pragma unroll
    for (int k4 = 0; k4 < KC; k4 += 4) {
        double a[C::FM], b[C::FN];
#pragma unroll
        for (int i = 0; i < C::FM; ++i) a[i] = frag<C::BM, AK>(sA, r0 + i * 8, k4 + kq);
#pragma unroll
        for (int j = 0; j < C::FN; ++j) b[j] = frag<C::BN, BK>(sB, c0 + j * 8, k4 + kq);
#pragma unroll
        for (int i = 0; i < C::FM; ++i)
#pragma unroll
            for (int j = 0; j < C::FN; ++j) dmma884(acc.v[i][j], a[i], b[j]);
    }
}

template <class C, bool AK, bool BK>
__device__ void cta_gemm_impl(Acc<C> &acc, const View &A, const View &B, int M, int N, int K,
                              double *smem, bool alA, bool alB) {
    double *sA[2] = {smem, smem + C::SA};
    double *sB[2] = {smem + 2 * C::SA, smem + 2 * C::SA + C::SB};
    const int nk = (K + KC - 1) / KC;
    load_stage<C::BM, AK>(sA[0], A, M, K, 0, alA);
    load_stage<C::BN, BK>(sB[0], B, N, K, 0, alB);
    cp_async_commit();
    for (int c = 0; c < nk; ++c) {
        if (c + 1 < nk) {
            load_stage<C::BM, AK>(sA[(c + 1) & 1], A, M, K, (c + 1) * KC, alA);
            load_stage<C::BN, BK>(sB[(c + 1) & 1], B, N, K, (c + 1) * KC, alB);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        mma_stage<C, AK, BK>(acc, sA[c & 1], sB[c & 1]);
        __syncthreads();
    }
}

__device__ __forceinline__ bool view_aligned(const View &V) {
    const int64_t ld = V.rs == 1 ? V.cs : V.rs;
    return ((reinterpret_cast<uintptr_t>(V.p) & 15) == 0) && ((ld & 1) == 0);
}

// acc(i,j) += sum_{k<K} A(i,k) B(j,k), i < M <= BM, j < N <= BN.  All threads
// of the CTA call it; shared memory `smem` holds C::SMEM_BYTES.  Ends with a
// barrier, so `smem` may be reused right after.
template <class C>
__device__ void cta_gemm(Acc<C> &acc, const View &A, const View &B, int M, int N, int K, double *smem) {
    if (K <= 0 || M <= 0 || N <= 0) return;
    const bool ak = (A.rs != 1), bk = (B.rs != 1);
    const bool alA = view_aligned(A), alB = view_aligned(B);
    if (!ak && !bk) cta_gemm_impl<C, false, false>(acc, A, B, M, N, K, smem, alA, alB);
    else if (!ak && bk) cta_gemm_impl<C, false, true>(acc, A, B, M, N, K, smem, alA, alB);
    else if (ak && !bk) cta_gemm_impl<C, true, false>(acc, A, B, M, N, K, smem, alA, alB);
    else cta_gemm_impl<C, true, true>(acc, A, B, M, N, K, smem, alA, alB);
}

// ---------------------------------------------------------------------------
// Inner-block Cholesky + triangular inverse in shared memory.
// sD: n x n (n <= IB) column-major with leading dimension IB+1, lower triangle
// valid.  On return sD holds L (lower) and sInv holds L^{-1} (lower, zero
// upper).  Returns 0 or the 1-based column of the first non-positive pivot
// (LAPACK dpotrf info convention).
// ---------------------------------------------------------------------------
constexpr int LDD = IB + 1;

__device__ inline int blk_chol(double *sD, int n) {
    const int tid = threadIdx.x;
    for (int j = 0; j < n; ++j) {
        const double d = sD[j + j * LDD];
        if (!(d > 0.0)) {      // also catches NaN; uniform across the CTA
            __syncthreads();
            return j + 1;
        }
        const double ljj = sqrt(d);
        const double inv = 1.0 / ljj;
        for (int i = j + 1 + tid; i < n; i += NT_CTA) sD[i + j * LDD] *= inv;
        __syncthreads();
        if (tid == 0) sD[j + j * LDD] = ljj;
        const int w = n - j - 1;
        for (int idx = tid; idx < w * w; idx += NT_CTA) {
            const int i = j + 1 + idx % w, c = j + 1 + idx / w;
            if (c <= i) sD[i + c * LDD] -= sD[i + j * LDD] * sD[c + j * LDD];
        }
        __syncthreads();
    }
    return 0;
}

// sInv = L^{-1} for L = lower triangle of sD (n x n): row sweep, row i from
// rows < i; 4 threads per column split the dot product (shuffle combine).
__device__ inline void blk_inv(const double *sD, double *sInv, int n, bool unit = false) {
    const int tid = threadIdx.x;
    for (int idx = tid; idx < IB * IB; idx += NT_CTA) sInv[idx] = 0.0;
    __syncthreads();
    const int c = tid >> 2, part = tid & 3;   // 64 columns x 4 parts
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        if (c < i) {
            for (int k = c + part; k < i; k += 4) s += sD[i + k * LDD] * sInv[k + c * IB];
        }
        s += __shfl_down_sync(0xffffffffu, s, 2, 4);
        s += __shfl_down_sync(0xffffffffu, s, 1, 4);
        if (part == 0 && c <= i) {
            const double rhs = (c == i) ? 1.0 : 0.0;
            sInv[i + c * IB] = unit ? (rhs - s) : (rhs - s) / sD[i + i * LDD];
        }
        __syncthreads();
    }
}

__device__ inline int blk_potrf_inv(double *sD, double *sInv, int n) {
    const int info = blk_chol(sD, n);
    if (info) return info;
    blk_inv(sD, sInv, n);
    return 0;
}

// Copy an IB x IB lower inverse from shared (ld IB) to global (ld IB).
__device__ __forceinline__ void store_inv(double *g, const double *sInv) {
    for (int idx = threadIdx.x; idx < IB * IB; idx += NT_CTA) g[idx] = sInv[idx];
}

// ---------------------------------------------------------------------------
// Row-block right solve:  X <- X * L^{-T}  for X = rows x n (rows <= 128),
// L lower n x n with inverted diagonal blocks invd[b] (IB x IB, ld IB,
// column-major) -- i.e. the panel TRSM Right/Lower/Trans/NonUnit of
// coreblas/compute/core_ztrsm.c as used by compute/pzpotrf.c:100-105.
// Left-looking over inner blocks; all work in cta_gemm.
// ---------------------------------------------------------------------------
__device__ inline void trsm_rows(const View &X, int rows, const View &L, int n, const double *invd,
                          double *smem) {
    for (int jb = 0; jb < n; jb += IB) {
        const int nbk = min(IB, n - jb);
        Acc<Cfg12864> acc;
        if (jb > 0) {
            acc.zero();
            cta_gemm(acc, X, L.sub(jb, 0), rows, nbk, jb, smem);
            const View Xj = X.sub(0, jb);
            acc.for_each([&](int r, int c, double v) {
                if (r < rows && c < nbk) *Xj.at(r, c) -= v;
            });
            cta_sync_global();
        }
        acc.zero();
        const View Inv{const_cast<double *>(invd) + (int64_t)(jb / IB) * IB * IB, 1, IB};
        cta_gemm(acc, X.sub(0, jb), Inv, rows, nbk, nbk, smem);
        const View Xj = X.sub(0, jb);
        acc.for_each([&](int r, int c, double v) {
            if (r < rows && c < nbk) *Xj.at(r, c) = v;
        });
        cta_sync_global();
    }
}

// ---------------------------------------------------------------------------
// Left solve on a column strip:  X <- op(L)^{-1} X,  X = n x w (w <= 64),
// op = N (forward) or T (backward); inverted diagonal blocks as above.
// The solves of compute/pztrsm.c:58-200 (Left, Lower, {NoTrans, Trans}) on
// one diagonal tile.
// ---------------------------------------------------------------------------
__device__ inline void trsm_left(const View &X, int w, const View &L, int n, const double *invd,
                          bool trans, double *smem) {
    const int nblk = (n + IB - 1) / IB;
    for (int s = 0; s < nblk; ++s) {
        const int b = trans ? (nblk - 1 - s) : s;
        const int jb = b * IB, nbk = min(IB, n - jb);
        Acc<Cfg64> acc;
        if (!trans && jb > 0) {
            acc.zero();
            // acc(i,c) = sum_k L(jb+i, k) X(k, c), k < jb
            cta_gemm(acc, L.sub(jb, 0), X.t(), nbk, w, jb, smem);
        } else if (trans && jb + nbk < n) {
            acc.zero();
            // acc(i,c) = sum_k L(jb+nbk+k, jb+i) X(jb+nbk+k, c)
            cta_gemm(acc, L.sub(jb + nbk, jb).t(), X.sub(jb + nbk, 0).t(), nbk, w, n - jb - nbk, smem);
        } else {
            acc.zero();
        }
        const bool had = (!trans && jb > 0) || (trans && jb + nbk < n);
        const View Xj = X.sub(jb, 0);
        if (had) {
            acc.for_each([&](int r, int c, double v) {
                if (r < nbk && c < w) *Xj.at(r, c) -= v;
            });
            cta_sync_global();
        }
        acc.zero();
        View Inv{const_cast<double *>(invd) + (int64_t)b * IB * IB, 1, IB};
        if (trans) Inv = Inv.t();
        // acc(i,c) = sum_k op(Inv)(i,k) Xj(k,c)
        cta_gemm(acc, Inv, Xj.t(), nbk, w, nbk, smem);
        acc.for_each([&](int r, int c, double v) {
            if (r < nbk && c < w) *Xj.at(r, c) = v;
        });
        cta_sync_global();
    }
}

// ---------------------------------------------------------------------------
// Diagonal-tile Cholesky (lower, on view T, n x n): left-looking over inner
// blocks of IB; writes L into T's lower triangle (upper untouched, as LAPACK
// dpotrf), the inverted diagonal blocks into invd.  Returns LAPACK info.
// Follows the semantics of CORE_dpotrf (coreblas/compute/core_zpotrf.c:75-81).
// smem: >= max(Cfg12864/Cfg64) + 2*IB*LDD doubles.
// ---------------------------------------------------------------------------
__device__ inline int tile_potrf(const View &T, int n, double *invd, double *smem) {
    double *sD = smem + Cfg12864::SMEM_ELEMS;
    double *sInv = sD + IB * LDD;
    for (int jb = 0; jb < n; jb += IB) {
        const int nbk = min(IB, n - jb);
        Acc<Cfg64> acc;
        acc.zero();
        if (jb > 0) cta_gemm(acc, T.sub(jb, 0), T.sub(jb, 0), nbk, nbk, jb, smem);
        for (int idx = threadIdx.x; idx < nbk * nbk; idx += NT_CTA) {
            const int r = idx % nbk, c = idx / nbk;
            if (r >= c) sD[r + c * LDD] = *T.at(jb + r, jb + c);
        }
        __syncthreads();
        acc.for_each([&](int r, int c, double v) {
            if (r < nbk && c < nbk && r >= c) sD[r + c * LDD] -= v;
        });
        __syncthreads();
        const int info = blk_potrf_inv(sD, sInv, nbk);
        if (info) return jb + info;
        for (int idx = threadIdx.x; idx < nbk * nbk; idx += NT_CTA) {
            const int r = idx % nbk, c = idx / nbk;
            if (r >= c) *T.at(jb + r, jb + c) = sD[r + c * LDD];
        }
        store_inv(invd + (int64_t)(jb / IB) * IB * IB, sInv);
        cta_sync_global();
        // panel below the inner diagonal block
        for (int r0 = jb + nbk; r0 < n; r0 += 128) {
            const int mr = min(128, n - r0);
            Acc<Cfg12864> pa;
            if (jb > 0) {
                pa.zero();
                cta_gemm(pa, T.sub(r0, 0), T.sub(jb, 0), mr, nbk, jb, smem);
                const View P = T.sub(r0, jb);
                pa.for_each([&](int r, int c, double v) {
                    if (r < mr && c < nbk) *P.at(r, c) -= v;
                });
                cta_sync_global();
            }
            pa.zero();
            const View Inv{invd + (int64_t)(jb / IB) * IB * IB, 1, IB};
            cta_gemm(pa, T.sub(r0, jb), Inv, mr, nbk, nbk, smem);
            const View P = T.sub(r0, jb);
            pa.for_each([&](int r, int c, double v) {
                if (r < mr && c < nbk) *P.at(r, c) = v;
            });
            cta_sync_global();
        }
    }
    return 0;
}

constexpr size_t TILE_KERNEL_SMEM_ELEMS() {
    return (Cfg128::SMEM_ELEMS > (Cfg12864::SMEM_ELEMS + 2 * IB * LDD)
                ? Cfg128::SMEM_ELEMS
                : (Cfg12864::SMEM_ELEMS + 2 * IB * LDD));
}
constexpr size_t TILE_KERNEL_SMEM_BYTES = sizeof(double) * TILE_KERNEL_SMEM_ELEMS() + 64;

}  // namespace chb
