// core.cuh -- device building blocks of the B200 tile kernels.
//
// Every tile operation of the Cholesky path (reference: the POTRF / TRSM /
// SYRK / GEMM tile kernels of coreblas and gpucublas, e.g.
// coreblas/compute/core_zpotrf.c:75-81, gpucublas/compute/cuda_zgemm.c:24-45)
// is expressed with three CTA-wide primitives, generic over the element type:
//
//   cta_gemm      acc(i,j) += sum_k A(i,k) * B(j,k)  ("NT" form), operands
//                 staged global -> shared by cp.async (two-stage pipeline, any
//                 operand orientation), multiplied on the tensor cores:
//                   double: FP64 DMMA (mma.sync m8n8k4 f64);
//                   float : split products on mma.sync with FP32 accumulation,
//                           BF16x3 (x = hi + lo in bf16, hi*hi + hi*lo + lo*hi,
//                           m16n8k16) or TF32x3 (same split in tf32, m16n8k8);
//   blk_inv       the explicit inverse of a <= 64 x 64 triangular block in
//                 shared memory;
//   trsm_rows / trsm_left   blocked triangular solves that apply the inverted
//                 64 x 64 diagonal blocks, so that all bulk work is GEMM-shaped.
//
// Matrices are addressed through ViewT: element (i,j) at p[i*rs + j*cs].  A
// column-major tile with leading dimension ld is {p, 1, ld}; its transpose is
// {p, ld, 1}.  This is how the Upper variants become the Lower algorithm on
// transposed views (Upper tile (n,m) == transpose of Lower tile (m,n)).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace chb {

constexpr int NT_CTA = 256;   // threads per CTA of every tile kernel
constexpr int KC     = 32;    // k-extent of one pipeline stage
constexpr int IB     = 64;    // inner block of POTRF / TRSM (inverted diagonal blocks)
constexpr int LDD    = IB + 1;// leading dimension of the inner block in shared memory

enum SplitKind : int { SPLIT_BF16X3 = 0, SPLIT_TF32X3 = 1 };

template <class T>
struct ViewT {
    T *p;
    int64_t rs, cs;
    __device__ __forceinline__ T *at(int i, int j) const { return p + (int64_t)i * rs + (int64_t)j * cs; }
    __device__ __forceinline__ ViewT sub(int i, int j) const { return ViewT{at(i, j), rs, cs}; }
    __device__ __forceinline__ ViewT t() const { return ViewT{p, cs, rs}; }
};
using View = ViewT<double>;
using ViewF = ViewT<float>;

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
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, int src_bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}
__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ void mma_tf32_1688(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// (x0, x1) -> packed bf16x2 hi part and the packed bf16x2 of the remainders.
__device__ __forceinline__ void split_bf16(float x0, float x1, uint32_t &hi, uint32_t &lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - __low2float(h), x1 - __high2float(h));
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}
__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;\n" ::: "memory"); }
__device__ __forceinline__ void red_release_add(int *p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
// Make this CTA's global writes visible at GPU scope (they are re-read through
// L2 by cp.async.cg), then join the CTA.
__device__ __forceinline__ void cta_sync_global() {
    __threadfence();
    __syncthreads();
}
// Join the CTA after global writes that only this CTA reads back: bar.sync
// orders every participating thread's earlier memory accesses before the
// others' later ones (cp.async reads included), with no GPU-scope fence, which
// is slow while the memory system is loaded.  Visibility to other CTAs is
// established once per task by the executor (fence + release).
__device__ __forceinline__ void cta_sync() { __syncthreads(); }
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Shared-memory stage geometry per element type.  A stage holds a (ROWS x KC)
// slab of one operand.  MN-contiguous operands (V.rs == 1) are stored [k][row]
// with leading dimension ROWS + PAD; K-contiguous ones (V.cs == 1) [row][k]
// with leading dimension LDK.  The pads make the fragment reads conflict-free.
// ---------------------------------------------------------------------------
template <class T>
struct Geom;
// Fragment reads of an MN-contiguous stage: lanes (g, t) of one 16-lane phase
// read rows g (0..3) of k rows t (0..3); a leading dimension of 4 mod 16
// doubles (8 mod 32 floats) puts the four k rows on disjoint banks.
template <>
struct Geom<double> {
    static constexpr int VEC = 2, PAD = 4, LDK = KC + 4;
};
template <>
struct Geom<float> {
    static constexpr int VEC = 4, PAD = 4, LDK = KC + 8;
};

template <class T, int ROWS, bool KMAJ>
__host__ __device__ constexpr int stage_ld() {
    return KMAJ ? Geom<T>::LDK : ROWS + Geom<T>::PAD;
}
template <class T, int ROWS>
__host__ __device__ constexpr int stage_elems_max() {
    return ROWS * Geom<T>::LDK > KC * (ROWS + Geom<T>::PAD) ? ROWS * Geom<T>::LDK : KC * (ROWS + Geom<T>::PAD);
}

// Stage loader: rows < M, k0 <= k < min(K, k0+KC); out-of-range elements are
// zero-filled.  ALIGNED: 16-byte cp.async of VEC elements (base 16-byte
// aligned, non-unit stride a multiple of VEC); otherwise one cp.async per element.
template <class T, int ROWS, bool KMAJ>
__device__ __forceinline__ void load_stage(T *s, const ViewT<T> &V, int M, int K, int k0, bool aligned) {
    constexpr int VEC = Geom<T>::VEC;
    constexpr int LD = stage_ld<T, ROWS, KMAJ>();
    const int tid = threadIdx.x;
    if (!KMAJ) {
        constexpr int CH = ROWS / VEC;
        for (int idx = tid; idx < KC * CH; idx += NT_CTA) {
            const int kk = idx / CH, i = VEC * (idx % CH);
            const int gk = k0 + kk;
            const T *src = V.p + i + (int64_t)gk * V.cs;
            T *dst = s + kk * LD + i;
            const bool kin = gk < K;
            if (aligned) {
                const int nv = kin ? max(0, min(VEC, M - i)) : 0;
                cp_async16(dst, nv ? src : V.p, nv * (int)sizeof(T));
            } else {
#pragma unroll
                for (int e = 0; e < VEC; ++e) {
                    const bool in = kin && i + e < M;
                    if (sizeof(T) == 8) cp_async8(dst + e, in ? src + e : V.p, in ? 8 : 0);
                    else cp_async4(dst + e, in ? src + e : V.p, in ? 4 : 0);
                }
            }
        }
    } else {
        constexpr int CH = KC / VEC;
        for (int idx = tid; idx < ROWS * CH; idx += NT_CTA) {
            const int i = idx / CH, kk = VEC * (idx % CH);
            const int gk = k0 + kk;
            const T *src = V.p + (int64_t)i * V.rs + gk;
            T *dst = s + i * LD + kk;
            const bool iin = i < M;
            if (aligned) {
                const int nv = iin ? max(0, min(VEC, K - gk)) : 0;
                cp_async16(dst, nv ? src : V.p, nv * (int)sizeof(T));
            } else {
#pragma unroll
                for (int e = 0; e < VEC; ++e) {
                    const bool in = iin && gk + e < K;
                    if (sizeof(T) == 8) cp_async8(dst + e, in ? src + e : V.p, in ? 8 : 0);
                    else cp_async4(dst + e, in ? src + e : V.p, in ? 4 : 0);
                }
            }
        }
    }
}

template <class T, int ROWS, bool KMAJ>
__device__ __forceinline__ T frag(const T *s, int row, int kk) {
    if (KMAJ) return s[row * Geom<T>::LDK + kk];
    return s[kk * (ROWS + Geom<T>::PAD) + row];
}

// Tile configuration of cta_gemm: BM x BN outputs, WM x WN warps (8 warps).
template <class T_, int BM_, int BN_, int WM_, int WN_, int SP_ = SPLIT_BF16X3, int ST_ = 2>
struct GemmCfg {
    using T = T_;
    static constexpr bool F64 = std::is_same<T_, double>::value;
    static constexpr int SP = SP_;
    static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_;
    static constexpr int WTM = BM / WM, WTN = BN / WN;
    static constexpr int MT = F64 ? 8 : 16;          // rows of one MMA tile
    static constexpr int FM = WTM / MT, FN = WTN / 8;
    static constexpr int NACC = F64 ? 2 : 4;         // accumulators per MMA tile and thread
    static_assert(WM * WN * 32 == NT_CTA, "8 warps");
    static_assert(FM >= 1 && FN >= 1, "warp tile too small");
    static constexpr int SA = stage_elems_max<T_, BM>(), SB = stage_elems_max<T_, BN>();
    // cp.async pipeline depth (2 in the executor kernel: deeper pipelines
    // measured slower there, and FP64 tiles would not fit more; standalone
    // long-K kernels such as the residual use 3)
    static constexpr int ST = ST_;
    static constexpr int SMEM_ELEMS = ST * (SA + SB);
    static constexpr size_t SMEM_BYTES = sizeof(T_) * SMEM_ELEMS;
};
template <class T, int SP = SPLIT_BF16X3>
using Cfg128 = GemmCfg<T, 128, 128, 2, 4, SP>;   // trailing-update sub-blocks
template <class T, int SP = SPLIT_BF16X3>
using Cfg12864 = GemmCfg<T, 128, 64, 4, 2, SP>;  // panel rows x one inner block
template <class T, int SP = SPLIT_BF16X3>
using Cfg64 = GemmCfg<T, 64, 64, 2, 4, SP>;      // inner block x inner block
// inner block x a narrow right-hand-side block: 8 columns (one DMMA n8 tile per
// warp) for double, 16 for float (one m16n8 tile per warp)
template <class T, int SP = SPLIT_BF16X3>
using Cfg64N = typename std::conditional<std::is_same<T, double>::value, GemmCfg<T, 64, 8, 8, 1, SP>,
                                         GemmCfg<T, 64, 16, 4, 2, SP>>::type;

template <class C_>
struct Acc {
    using C = C_;
    using T = typename C_::T;
    T v[C::FM][C::FN][C::NACC];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int a = 0; a < C::FM; ++a)
#pragma unroll
            for (int b = 0; b < C::FN; ++b)
#pragma unroll
                for (int e = 0; e < C::NACC; ++e) v[a][b][e] = T(0);
    }
    // C(r, c) -= acc for r < rows, c < cols (and r >= c when lower_only): per
    // MMA row tile, all loads are issued before any store, so they overlap
    // instead of serializing behind possible aliasing.
    __device__ __forceinline__ void sub_from(const ViewT<T> &C, int rows, int cols, bool lower_only) const {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int wm = warp / C_::WN, wn = warp % C_::WN;
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int a = 0; a < C_::FM; ++a) {
            T old[C_::FN][C_::NACC];
            bool ok[C_::FN][C_::NACC];
#pragma unroll
            for (int b = 0; b < C_::FN; ++b)
#pragma unroll
                for (int e = 0; e < C_::NACC; ++e) {
                    const int r = wm * C_::WTM + a * C_::MT + g + ((e >= 2) ? 8 : 0);
                    const int c = wn * C_::WTN + b * 8 + 2 * t + (e & 1);
                    ok[b][e] = r < rows && c < cols && (!lower_only || r >= c);
                    old[b][e] = ok[b][e] ? __ldcg(C.at(r, c)) : T(0);
                }
#pragma unroll
            for (int b = 0; b < C_::FN; ++b)
#pragma unroll
                for (int e = 0; e < C_::NACC; ++e) {
                    const int r = wm * C_::WTM + a * C_::MT + g + ((e >= 2) ? 8 : 0);
                    const int c = wn * C_::WTN + b * 8 + 2 * t + (e & 1);
                    if (ok[b][e]) *C.at(r, c) = old[b][e] - v[a][b][e];
                }
        }
    }
    // C(r, c) = acc for r < rows, c < cols.
    __device__ __forceinline__ void store_to(const ViewT<T> &C, int rows, int cols) const {
        for_each([&](int r, int c, T x) {
            if (r < rows && c < cols) *C.at(r, c) = x;
        });
    }
    // f(a, b, e, row, col, value): for_each with the register coordinates.
    template <class F>
    __device__ __forceinline__ void for_each_idx(F &&f) const {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int wm = warp / C::WN, wn = warp % C::WN;
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int a = 0; a < C::FM; ++a)
#pragma unroll
            for (int b = 0; b < C::FN; ++b)
#pragma unroll
                for (int e = 0; e < C::NACC; ++e) {
                    const int r = wm * C::WTM + a * C::MT + g + ((e >= 2) ? 8 : 0);
                    const int c = wn * C::WTN + b * 8 + 2 * t + (e & 1);
                    f(a, b, e, r, c, v[a][b][e]);
                }
    }
    // f(row, col, value) for every accumulator element owned by this thread.
    template <class F>
    __device__ __forceinline__ void for_each(F &&f) const {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int wm = warp / C::WN, wn = warp % C::WN;
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int a = 0; a < C::FM; ++a)
#pragma unroll
            for (int b = 0; b < C::FN; ++b)
#pragma unroll
                for (int e = 0; e < C::NACC; ++e) {
                    const int r = wm * C::WTM + a * C::MT + g + ((e >= 2) ? 8 : 0);
                    const int c = wn * C::WTN + b * 8 + 2 * t + (e & 1);
                    f(r, c, v[a][b][e]);
                }
    }
};

template <class C, bool AK, bool BK>
__device__ __forceinline__ void mma_stage(Acc<C> &acc, const typename C::T *sA, const typename C::T *sB) {
    using T = typename C::T;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp / C::WN, wn = warp % C::WN;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = wm * C::WTM + g, c0 = wn * C::WTN + g;
    if constexpr (C::F64) {
#pragma unroll
        for (int k4 = 0; k4 < KC; k4 += 4) {
            double a[C::FM], b[C::FN];
#pragma unroll
            for (int i = 0; i < C::FM; ++i) a[i] = frag<T, C::BM, AK>(sA, r0 + i * 8, k4 + t);
#pragma unroll
            for (int j = 0; j < C::FN; ++j) b[j] = frag<T, C::BN, BK>(sB, c0 + j * 8, k4 + t);
#pragma unroll
            for (int i = 0; i < C::FM; ++i)
#pragma unroll
                for (int j = 0; j < C::FN; ++j) dmma884(acc.v[i][j], a[i], b[j]);
        }
    } else if constexpr (C::SP == SPLIT_BF16X3) {
#pragma unroll
        for (int k16 = 0; k16 < KC; k16 += 16) {
            uint32_t ah[C::FM][4], al[C::FM][4], bh[C::FN][2], bl[C::FN][2];
            const int ka = k16 + 2 * t;
#pragma unroll
            for (int i = 0; i < C::FM; ++i) {
                const int r = r0 + i * 16;
                split_bf16(frag<T, C::BM, AK>(sA, r, ka), frag<T, C::BM, AK>(sA, r, ka + 1), ah[i][0], al[i][0]);
                split_bf16(frag<T, C::BM, AK>(sA, r + 8, ka), frag<T, C::BM, AK>(sA, r + 8, ka + 1), ah[i][1],
                           al[i][1]);
                split_bf16(frag<T, C::BM, AK>(sA, r, ka + 8), frag<T, C::BM, AK>(sA, r, ka + 9), ah[i][2], al[i][2]);
                split_bf16(frag<T, C::BM, AK>(sA, r + 8, ka + 8), frag<T, C::BM, AK>(sA, r + 8, ka + 9), ah[i][3],
                           al[i][3]);
            }
#pragma unroll
            for (int j = 0; j < C::FN; ++j) {
                const int n = c0 + j * 8;
                split_bf16(frag<T, C::BN, BK>(sB, n, ka), frag<T, C::BN, BK>(sB, n, ka + 1), bh[j][0], bl[j][0]);
                split_bf16(frag<T, C::BN, BK>(sB, n, ka + 8), frag<T, C::BN, BK>(sB, n, ka + 9), bh[j][1], bl[j][1]);
            }
#pragma unroll
            for (int i = 0; i < C::FM; ++i)
#pragma unroll
                for (int j = 0; j < C::FN; ++j) {
                    mma_bf16_16816(acc.v[i][j], al[i], bh[j]);
                    mma_bf16_16816(acc.v[i][j], ah[i], bl[j]);
                    mma_bf16_16816(acc.v[i][j], ah[i], bh[j]);
                }
        }
    } else {
#pragma unroll
        for (int k8 = 0; k8 < KC; k8 += 8) {
            uint32_t ah[C::FM][4], al[C::FM][4], bh[C::FN][2], bl[C::FN][2];
#pragma unroll
            for (int i = 0; i < C::FM; ++i) {
                const int r = r0 + i * 16;
                split_tf32(frag<T, C::BM, AK>(sA, r, k8 + t), ah[i][0], al[i][0]);
                split_tf32(frag<T, C::BM, AK>(sA, r + 8, k8 + t), ah[i][1], al[i][1]);
                split_tf32(frag<T, C::BM, AK>(sA, r, k8 + t + 4), ah[i][2], al[i][2]);
                split_tf32(frag<T, C::BM, AK>(sA, r + 8, k8 + t + 4), ah[i][3], al[i][3]);
            }
#pragma unroll
            for (int j = 0; j < C::FN; ++j) {
                const int n = c0 + j * 8;
                split_tf32(frag<T, C::BN, BK>(sB, n, k8 + t), bh[j][0], bl[j][0]);
                split_tf32(frag<T, C::BN, BK>(sB, n, k8 + t + 4), bh[j][1], bl[j][1]);
            }
#pragma unroll
            for (int i = 0; i < C::FM; ++i)
#pragma unroll
                for (int j = 0; j < C::FN; ++j) {
                    mma_tf32_1688(acc.v[i][j], al[i], bh[j]);
                    mma_tf32_1688(acc.v[i][j], ah[i], bl[j]);
                    mma_tf32_1688(acc.v[i][j], ah[i], bh[j]);
                }
        }
    }
}

template <class C, bool AK, bool BK>
__device__ void cta_gemm_impl(Acc<C> &acc, const ViewT<typename C::T> &A, const ViewT<typename C::T> &B, int M,
                              int N, int K, typename C::T *smem, bool alA, bool alB) {
    using T = typename C::T;
    constexpr int ST = C::ST;
    T *sA = smem, *sB = smem + ST * C::SA;
    const int nk = (K + KC - 1) / KC;
    // prologue: stages 0 .. ST-2 in flight (one commit group each, possibly empty)
#pragma unroll
    for (int st = 0; st < ST - 1; ++st) {
        if (st < nk) {
            load_stage<T, C::BM, AK>(sA + st * C::SA, A, M, K, st * KC, alA);
            load_stage<T, C::BN, BK>(sB + st * C::SB, B, N, K, st * KC, alB);
        }
        cp_async_commit();
    }
    for (int c = 0; c < nk; ++c) {
        const int nxt = c + ST - 1;
        if (nxt < nk) {
            const int slot = nxt % ST;
            load_stage<T, C::BM, AK>(sA + slot * C::SA, A, M, K, nxt * KC, alA);
            load_stage<T, C::BN, BK>(sB + slot * C::SB, B, N, K, nxt * KC, alB);
        }
        cp_async_commit();
        cp_async_wait<ST - 1>();   // stage c has landed
        __syncthreads();
        const int slot = c % ST;
        mma_stage<C, AK, BK>(acc, sA + slot * C::SA, sB + slot * C::SB);
        __syncthreads();
    }
    cp_async_wait<0>();
}

template <class T>
__device__ __forceinline__ bool view_aligned(const ViewT<T> &V) {
    const int64_t ld = V.rs == 1 ? V.cs : V.rs;
    return ((reinterpret_cast<uintptr_t>(V.p) & 15) == 0) && ((ld % Geom<T>::VEC) == 0);
}

// acc(i,j) += sum_{k<K} A(i,k) B(j,k), i < M <= BM, j < N <= BN.  All threads
// of the CTA call it; shared memory `smem` holds C::SMEM_BYTES.  Ends with a
// barrier, so `smem` may be reused right after.
template <class C>
__device__ void cta_gemm(Acc<C> &acc, const ViewT<typename C::T> &A, const ViewT<typename C::T> &B, int M, int N,
                         int K, typename C::T *smem) {
    if (K <= 0 || M <= 0 || N <= 0) return;
    const bool ak = (A.rs != 1), bk = (B.rs != 1);
    const bool alA = view_aligned(A), alB = view_aligned(B);
    if (!ak && !bk) cta_gemm_impl<C, false, false>(acc, A, B, M, N, K, smem, alA, alB);
    else if (!ak && bk) cta_gemm_impl<C, false, true>(acc, A, B, M, N, K, smem, alA, alB);
    else if (ak && !bk) cta_gemm_impl<C, true, false>(acc, A, B, M, N, K, smem, alA, alB);
    else cta_gemm_impl<C, true, true>(acc, A, B, M, N, K, smem, alA, alB);
}

// ---------------------------------------------------------------------------
// Inner-block triangular inverse in shared memory.  sD: n x n (n <= IB)
// column-major with leading dimension LDD, lower triangle valid.
// ---------------------------------------------------------------------------
// sInv = L^{-1} for L = lower triangle of sD (n x n): row sweep, row i from
// rows < i; 4 threads per column split the dot product (shuffle combine).
template <class T>
__device__ inline void blk_inv(const T *sD, T *sInv, int n, bool unit = false) {
    // sInv has room for IB x LDD elements: the sweep works at stride LDD
    // (conflict-free column reads), then compacts to stride IB in place.
    const int tid = threadIdx.x;
    for (int idx = tid; idx < IB * LDD; idx += NT_CTA) sInv[idx] = T(0);
    __syncthreads();
    const int c = tid >> 2, part = tid & 3;   // 64 columns x 4 parts
    for (int i = 0; i < n; ++i) {
        T s = T(0);
        if (c < i) {
            for (int k = c + part; k < i; k += 4) s += sD[i + k * LDD] * sInv[k + c * LDD];
        }
        s += __shfl_down_sync(0xffffffffu, s, 2, 4);
        s += __shfl_down_sync(0xffffffffu, s, 1, 4);
        if (part == 0 && c <= i) {
            const T rhs = (c == i) ? T(1) : T(0);
            sInv[i + c * LDD] = unit ? (rhs - s) : (rhs - s) / sD[i + i * LDD];
        }
        __syncthreads();
    }
    // compact columns 1..63 from stride LDD to stride IB (ascending: each
    // destination range starts before its source range, ranges of one column
    // do not overlap earlier compacted columns)
    for (int col = 1; col < IB; ++col) {
        T v = T(0);
        if (tid < IB) v = sInv[tid + col * LDD];
        __syncthreads();
        if (tid < IB) sInv[tid + col * IB] = v;
        __syncthreads();
    }
}

// Copy an IB x IB lower inverse from shared (ld IB) to global (ld IB).
template <class T>
__device__ __forceinline__ void store_inv(T *g, const T *sInv) {
    for (int idx = threadIdx.x; idx < IB * IB; idx += NT_CTA) g[idx] = sInv[idx];
}

// ---------------------------------------------------------------------------
// Row-block right solve:  X <- X * L^{-T}  for X = rows x n (rows <= 128),
// L lower n x n with inverted diagonal blocks invd[b] (IB x IB, ld IB,
// column-major) -- the panel TRSM Right/Lower/Trans/NonUnit of
// coreblas/compute/core_ztrsm.c as used by compute/pzpotrf.c:100-105.
// Left-looking over inner blocks; all work in cta_gemm.
// ---------------------------------------------------------------------------
template <class T, int SP>
__device__ inline void trsm_rows(const ViewT<T> &X, int rows, const ViewT<T> &L, int n, const T *invd, T *smem) {
    using C = Cfg12864<T, SP>;
    for (int jb = 0; jb < n; jb += IB) {
        const int nbk = min(IB, n - jb);
        Acc<C> acc;
        if (jb > 0) {
            acc.zero();
            cta_gemm(acc, X, L.sub(jb, 0), rows, nbk, jb, smem);
            acc.sub_from(X.sub(0, jb), rows, nbk, false);
            cta_sync();
        }
        acc.zero();
        const ViewT<T> Inv{const_cast<T *>(invd) + (int64_t)(jb / IB) * IB * IB, 1, IB};
        cta_gemm(acc, X.sub(0, jb), Inv, rows, nbk, nbk, smem);
        acc.store_to(X.sub(0, jb), rows, nbk);
        cta_sync();
    }
}

// ---------------------------------------------------------------------------
// Left solve on a column strip:  X <- op(L)^{-1} X,  X = n x w (w <= 64),
// op = N (forward) or T (backward); inverted diagonal blocks as above.
// The solves of compute/pztrsm.c:58-200 (Left, Lower, {NoTrans, Trans}) on
// one diagonal tile.
// ---------------------------------------------------------------------------
template <class T, int SP, class C = Cfg64<T, SP>>
__device__ inline void trsm_left(const ViewT<T> &X, int w, const ViewT<T> &L, int n, const T *invd, bool trans,
                                 T *smem) {
    const int nblk = (n + IB - 1) / IB;
    for (int s = 0; s < nblk; ++s) {
        const int b = trans ? (nblk - 1 - s) : s;
        const int jb = b * IB, nbk = min(IB, n - jb);
        Acc<C> acc;
        acc.zero();
        const bool had = (!trans && jb > 0) || (trans && jb + nbk < n);
        if (!trans && jb > 0) {
            // acc(i,c) = sum_k L(jb+i, k) X(k, c), k < jb
            cta_gemm(acc, L.sub(jb, 0), X.t(), nbk, w, jb, smem);
        } else if (trans && jb + nbk < n) {
            // acc(i,c) = sum_k L(jb+nbk+k, jb+i) X(jb+nbk+k, c)
            cta_gemm(acc, L.sub(jb + nbk, jb).t(), X.sub(jb + nbk, 0).t(), nbk, w, n - jb - nbk, smem);
        }
        const ViewT<T> Xj = X.sub(jb, 0);
        if (had) {
            acc.sub_from(Xj, nbk, w, false);
            cta_sync();
        }
        acc.zero();
        ViewT<T> Inv{const_cast<T *>(invd) + (int64_t)b * IB * IB, 1, IB};
        if (trans) Inv = Inv.t();
        // acc(i,c) = sum_k op(Inv)(i,k) Xj(k,c)
        cta_gemm(acc, Inv, Xj.t(), nbk, w, nbk, smem);
        acc.store_to(Xj, nbk, w);
        cta_sync();
    }
}

template <class T, int SP = SPLIT_BF16X3>
constexpr size_t tile_smem_elems() {
    return (Cfg128<T, SP>::SMEM_ELEMS > (Cfg12864<T, SP>::SMEM_ELEMS + 2 * IB * LDD)
                ? Cfg128<T, SP>::SMEM_ELEMS
                : (Cfg12864<T, SP>::SMEM_ELEMS + 2 * IB * LDD));
}
template <class T, int SP = SPLIT_BF16X3>
constexpr size_t tile_smem_bytes() {
    return sizeof(T) * tile_smem_elems<T, SP>() + 64;
}
constexpr size_t TILE_KERNEL_SMEM_BYTES = tile_smem_bytes<double>();

}  // namespace chb
