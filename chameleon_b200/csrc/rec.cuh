// rec.cuh -- recursive diagonal-tile Cholesky with the explicit tile inverse.
//
// The diagonal-tile POTRF is on the critical path of the tile Cholesky DAG
// (compute/pzpotrf.c: potrf(k) -> trsm(m,k) -> update(k+1,k+1) -> potrf(k+1)),
// so its latency, not its flops, bounds the factorization.  This variant
// factors an n x n tile (n <= 1024) by 2 x 2 recursion
//
//     [A11    ]   [L11    ]            L21 = A21 X11^T      (X11 = L11^-1)
//     [A21 A22] = [L21 L22] [..]^T,    A22 -= L21 L21^T,     L22 = chol(A22)
//
// and assembles the full inverse X = L^-1 on the way up
//
//     X21 = -X22 (L21 X11),
//
// so that every off-diagonal step is one GEMM-shaped pass (cta_gemm on the
// tensor cores).  The recursion ends in a 64 x 64 leaf made of two warp-level
// 32 x 32 Cholesky / inverse kernels that keep a column per lane in registers.
// With the full inverse, the panel solve A(m,k) <- A(m,k) L(k,k)^-T and the
// diagonal solves of the forward / backward substitutions are one GEMM each
// (apply_inv_right / apply_inv_left), done in place by ordering the output
// blocks so that no block is overwritten before it has been read.
//
// Using the explicit inverse of a whole tile trades the backward stability of
// a substitution for fewer dependent steps; the mixed-precision solver runs it
// in FP32 and its FP64 refinement restores the FP64 backward error.
#pragma once
#include "core.cuh"

namespace chb {
namespace rec {

constexpr int LDS = IB + 1;   // leaf shared-memory leading dimension (65)
constexpr unsigned FULL = 0xffffffffu;

// 1/sqrt(d) to working precision: hardware estimate + one Newton step.
__device__ __forceinline__ float rsqrt_wp(float d) {
    const float r = rsqrtf(d);
    return r * fmaf(-0.5f * d * r, r, 1.5f);
}
__device__ __forceinline__ double rsqrt_wp(double d) {
    const double r = rsqrt(d);
    return r * fma(-0.5 * d * r, r, 1.5);
}

// Cholesky of the 32 x 32 lower block at S (shared, ld LDS) by one warp, in
// place: lane i keeps row i in registers.  Each of the 32 steps needs the
// pivot, one reciprocal square root and the broadcast of column j.  Entries
// above the diagonal are updated too (no per-element predicates): they are
// never read back.  The block must be identity-padded beyond the matrix.
// Returns 0 or the 1-based column of the first non-positive pivot (uniform
// across the warp); after a failure the remaining steps run on a unit pivot
// so that the loop stays branch-free.  The loop is rolled (its ~1-2 KB of
// code stays in the instruction cache); register indices stay static by
// shifting: at step j, slot k of a lane holds the entry of column (row)
// j + k, and the update of slot k writes slot k - 1, so slot 0 is always the
// current column (row) and the shift costs no moves.
template <class T>
__device__ __noinline__ int warp_chol32r(T *S, T *bc) {
    const int lane = threadIdx.x & 31;
    T a[32];   // a[k]: entry (lane, j + k)
#pragma unroll
    for (int c = 0; c < 32; ++c) a[c] = (c <= lane) ? S[lane + c * LDS] : T(0);
    int info = 0;
    // pivot and reciprocal square root of step 0; every step computes those of
    // the next one right after the entry that holds it, so that the shuffle
    // and the square root overlap the rest of the update
    T d = __shfl_sync(FULL, a[0], 0);
    if (!(d > T(0))) {   // also catches NaN
        info = 1;
        d = T(1);
    }
    T r = rsqrt_wp(d);
#pragma unroll 1
    for (int j = 0; j < 32; ++j) {
        const T l = (lane == j) ? d * r : a[0] * r;
        if (lane >= j) S[lane + j * LDS] = l;
        // column j broadcast through bc (two buffers of 64 entries, by step
        // parity): buf[m] = l of lane m & 31, so that slot k reads buf[j + k]
        // at a fixed offset (one shared load per entry, no lane arithmetic);
        // the wrapped slots read the unused lanes' values, as shuffles would,
        // and are never read back
        T *buf = bc + ((j & 1) << 6);
        buf[lane] = l;
        buf[lane + 32] = l;
        __syncwarp();
        const T *col = buf + j;
        a[0] = a[1] - l * col[1];
        T dn = __shfl_sync(FULL, a[0], (j + 1) & 31);
#pragma unroll
        for (int k = 2; k < 32; ++k) a[k - 1] = a[k] - l * col[k];
        a[31] = T(0);
        if (!(dn > T(0))) {
            if (info == 0 && j + 1 < 32) info = j + 2;
            dn = T(1);
        }
        d = dn;
        r = rsqrt_wp(dn);
    }
    __syncwarp();
    return info;
}

// X = L^-1 for the 32 x 32 lower block at S, lane c = column c of X, slot k =
// row i + k at step i (the entries of columns of L are broadcast loads at
// fixed offsets from S(i, i): rows i + 1 .. i + 31, so up to 31 entries past
// row 31 of column i -- the wrapped slots, never read back; the caller keeps
// that range inside its shared memory: leaf64_core's sX follows sD).
template <class T>
__device__ __noinline__ void warp_trinv32r(const T *S, T *Xs) {
    const int lane = threadIdx.x & 31;
    T x[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) x[k] = (k == lane) ? T(1) : T(0);
    // the 32 diagonal reciprocals at once, off the step chain (lane i: 1 / L(i, i))
    const T rdl = T(1) / S[lane + lane * LDS];
#pragma unroll 1
    for (int i = 0; i < 32; ++i) {
        const T xi = x[0] * __shfl_sync(FULL, rdl, i);   // X(i, lane), final (zero above the diagonal)
        Xs[i + lane * LDS] = xi;
        const T *col = S + i * (LDS + 1);                 // S(i, i)
#pragma unroll
        for (int k = 1; k < 32; ++k) x[k - 1] = x[k] - col[k] * xi;
        x[31] = T(0);
    }
    __syncwarp();
}

// out(i, c) = sum_{k<32} P[i + k*LDS] * Q[c + k*LDS] (ROWS_Q: Q read as
// rows) or Q[k + c*LDS] (Q read as columns), 32 x 32 outputs spread over the
// CTA: thread (i = tid & 31, cg = tid >> 5) owns columns 4cg .. 4cg+3.
template <class T, bool QROWS>
__device__ __forceinline__ void small_mm32(const T *P, const T *Q, T (&o)[4]) {
    const int i = threadIdx.x & 31, cg = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = T(0);
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
        const T p = P[i + k * LDS];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = 4 * cg + q;
            o[q] += p * (QROWS ? Q[c + k * LDS] : Q[k + c * LDS]);
        }
    }
}

// 64 x 64 leaf on shared memory.  sD (ld LDS) holds the block, lower
// triangle, identity-padded beyond the matrix and zero above the diagonal.
// FACT: sD is factored in place (L), else it already holds L.  sX = sD + 64
// LDS (ld LDS) receives the full inverse (zeros above the diagonal); the
// inverse kernel's column reads run up to 29 entries past the end of sD, into
// sX.  Returns LAPACK info.  Called by all threads; ends with a barrier.
template <class T, bool FACT>
__device__ __noinline__ int leaf64_core(T *sD) {
    T *sX = sD + 64 * LDS;
    __shared__ int s_info;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) s_info = 0;
    __syncthreads();
    if (FACT) {
        if (warp == 0) {
            const int info = warp_chol32r(sD, sX);   // sX (2 columns) is free until the inverse
            if (tid == 0) s_info = info;
        }
        __syncthreads();
        if (s_info) return s_info;
    }
    if (warp == 0) warp_trinv32r(sD, sX);
    __syncthreads();
    T o[4];
    const int i = tid & 31, cg = tid >> 5;
    if (FACT) {
        // L21 = A21 X11^T
        small_mm32<T, true>(sD + 32, sX, o);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q) sD[32 + i + (4 * cg + q) * LDS] = o[q];
        __syncthreads();
        // A22 -= L21 L21^T (lower)
        small_mm32<T, true>(sD + 32, sD + 32, o);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = 4 * cg + q;
            if (c <= i) sD[32 + i + (32 + c) * LDS] -= o[q];
        }
        __syncthreads();
        if (warp == 0) {
            // the columns 32, 33 of sX are free until X22 and W are written
            const int info = warp_chol32r(sD + 32 + 32 * LDS, sX + 32 * LDS);
            if (tid == 0) s_info = info ? 32 + info : 0;
        }
        __syncthreads();
        if (s_info) return s_info;
    }
    if (warp == 1) warp_trinv32r(sD + 32 + 32 * LDS, sX + 32 + 32 * LDS);
    __syncthreads();
    // W = L21 X11 into the upper-right block of sX (zero in the inverse)
    small_mm32<T, false>(sD + 32, sX, o);
#pragma unroll
    for (int q = 0; q < 4; ++q) sX[i + (32 + 4 * cg + q) * LDS] = o[q];
    __syncthreads();
    // X21 = -X22 W
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = T(0);
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
        const T p = sX[32 + i + (32 + k) * LDS];
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] += p * sX[k + (32 + 4 * cg + q) * LDS];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) sX[32 + i + (4 * cg + q) * LDS] = -o[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) sX[i + (32 + 4 * cg + q) * LDS] = T(0);
    __syncthreads();
    return 0;
}

// Identity-padded load of the lower n x n block of A (n <= 64) into sD.
template <class T>
__device__ __forceinline__ void leaf64_load(const ViewT<T> &A, int n, T *sD) {
    for (int idx = threadIdx.x; idx < 64 * 64; idx += NT_CTA) {
        const int r = idx & 63, c = idx >> 6;
        T v = (r == c) ? T(1) : T(0);
        if (r < n && c < n) v = (r >= c) ? *A.at(r, c) : T(0);
        sD[r + c * LDS] = v;
    }
    __syncthreads();
}

// 64 x 64 leaf on global views: FACT factors the lower n x n block of A in
// place; the full inverse goes to X (n x n, written in full).
template <class T, bool FACT>
__device__ __noinline__ int leaf64(const ViewT<T> &A, const ViewT<T> &X, int n, T *smem) {
    T *sD = smem;              // 64 x LDS
    T *sX = smem + 64 * LDS;   // 64 x LDS
    leaf64_load(A, n, sD);
    const int info = leaf64_core<T, FACT>(sD);
    if (info) return info;
    for (int idx = threadIdx.x; idx < n * n; idx += NT_CTA) {
        const int r = idx % n, c = idx / n;
        if (FACT && r >= c) *A.at(r, c) = sD[r + c * LDS];
        *X.at(r, c) = sX[r + c * LDS];
    }
    cta_sync();
    return 0;
}

// Blocked left-looking diagonal-tile Cholesky (lower view Tv, n x n) with the
// 64-wide leaf: per inner block, one GEMM brings in the columns to its left,
// the leaf factors and inverts it in shared memory, and the rows below are
// updated and multiplied by the leaf's inverse.  Writes L into the lower
// triangle (upper untouched) and the inverted diagonal blocks (IB x IB, ld
// IB, zero outside the block) into invd.  Returns LAPACK info.  Same
// contract as CORE_dpotrf (coreblas/compute/core_zpotrf.c:75-81).
// ph (optional, tracing): thread 0 adds the clock cycles spent in the block-
// column updates, the leaves and the panels to ph[0..2].
// PR: rows of one panel step (128 or 64).  LEAN: the leaf's two 64 x 64
// blocks share the GEMM staging area instead of following it (the leaf runs
// between GEMMs), so that smem needs only lean_smem_elems() -- the footprint
// that lets several CTAs share an SM.
template <class T, int SP>
constexpr size_t lean_smem_elems() {
    return Cfg64<T, SP>::SMEM_ELEMS > 2 * IB * LDS ? Cfg64<T, SP>::SMEM_ELEMS : 2 * IB * LDS;
}
template <class T, int SP, int PR = 128, bool LEAN = false>
__device__ int tile_potrf_blk(const ViewT<T> &Tv, int n, T *invd, T *smem, unsigned *ph = nullptr) {
    static_assert(PR == 128 || PR == 64, "panel rows");
    using CP = typename std::conditional<PR == 128, Cfg12864<T, SP>, Cfg64<T, SP>>::type;
    using CD = Cfg64<T, SP>;
    T *sD = LEAN ? smem : smem + CP::SMEM_ELEMS;   // cta_gemm ends with a barrier
    T *sX = sD + IB * LDS;
    long long c0 = (ph && threadIdx.x == 0) ? clock64() : 0;
    auto lap = [&](int i) {
        if (ph && threadIdx.x == 0) {
            const long long c1 = clock64();
            ph[i] += (unsigned)(c1 - c0);
            c0 = c1;
        }
    };
    for (int jb = 0; jb < n; jb += IB) {
        const int nbk = min(IB, n - jb);
        Acc<CD> acc;
        acc.zero();
        if (jb > 0) cta_gemm(acc, Tv.sub(jb, 0), Tv.sub(jb, 0), nbk, nbk, jb, smem);
        leaf64_load(Tv.sub(jb, jb), nbk, sD);
        acc.for_each([&](int r, int c, T v) {
            if (r < nbk && c < nbk && r >= c) sD[r + c * LDS] -= v;
        });
        lap(0);
        const int info = leaf64_core<T, true>(sD);
        lap(1);
        if (info) return jb + info;
        T *inv = invd + (int64_t)(jb / IB) * IB * IB;
        for (int idx = threadIdx.x; idx < IB * IB; idx += NT_CTA) {
            const int r = idx % IB, c = idx / IB;
            if (r < nbk && c < nbk && r >= c) *Tv.at(jb + r, jb + c) = sD[r + c * LDS];
            inv[idx] = (r < nbk && c < nbk) ? sX[r + c * LDS] : T(0);
        }
        cta_sync();
        // panel below the inner diagonal block
        for (int r0 = jb + nbk; r0 < n; r0 += PR) {
            const int mr = min(PR, n - r0);
            Acc<CP> pa;
            if (jb > 0) {
                pa.zero();
                cta_gemm(pa, Tv.sub(r0, 0), Tv.sub(jb, 0), mr, nbk, jb, smem);
                pa.sub_from(Tv.sub(r0, jb), mr, nbk, false);
                cta_sync();
            }
            pa.zero();
            const ViewT<T> Inv{inv, 1, IB};
            cta_gemm(pa, Tv.sub(r0, jb), Inv, mr, nbk, nbk, smem);
            pa.store_to(Tv.sub(r0, jb), mr, nbk);
            cta_sync();
        }
        lap(2);
    }
    return 0;
}

// Inverted 64 x 64 diagonal blocks of an existing lower factor (n x n), for
// the solve-only executor mode.
template <class T>
__device__ void tile_inv_blk(const ViewT<T> &Tv, int n, T *invd, T *smem) {
    T *sD = smem;
    T *sX = sD + IB * LDS;
    for (int jb = 0; jb < n; jb += IB) {
        const int nbk = min(IB, n - jb);
        leaf64_load(Tv.sub(jb, jb), nbk, sD);
        leaf64_core<T, false>(sD);
        T *inv = invd + (int64_t)(jb / IB) * IB * IB;
        for (int idx = threadIdx.x; idx < IB * IB; idx += NT_CTA) {
            const int r = idx % IB, c = idx / IB;
            inv[idx] = (r < nbk && c < nbk) ? sX[r + c * LDS] : T(0);
        }
        __syncthreads();
    }
}

// Output block sizes of the GEMM passes.
template <class T, int SP>
using CB = Cfg128<T, SP>;   // 128 x 128

// A (rows x n) <- A X^T in place, X lower n x n: column blocks from the last
// (each reads columns < its end, which later blocks do not overwrite).
template <class T, int SP>
__device__ __noinline__ void apply_inv_right(const ViewT<T> &A, int rows, const ViewT<T> &X, int n, T *smem) {
    using C = CB<T, SP>;
    const int ncb = (n + C::BN - 1) / C::BN;
    for (int r0 = 0; r0 < rows; r0 += C::BM) {
        const int mr = min(C::BM, rows - r0);
        for (int cb = ncb - 1; cb >= 0; --cb) {
            const int c0 = cb * C::BN, w = min(C::BN, n - c0);
            Acc<C> acc;
            acc.zero();
            cta_gemm(acc, A.sub(r0, 0), X.sub(c0, 0), mr, w, c0 + w, smem);
            acc.store_to(A.sub(r0, c0), mr, w);
            cta_sync();
        }
    }
}

// B (n x w) <- X B (TRANS: X^T B) in place, X lower n x n: row blocks from the
// last (forward) or the first (transposed), so that no row of B is
// overwritten before every block that reads it is done.
template <class T, int SP, bool TRANS>
__device__ __noinline__ void apply_inv_left(const ViewT<T> &B, int w, const ViewT<T> &X, int n, T *smem) {
    using C = Cfg12864<T, SP>;
    const int nrb = (n + C::BM - 1) / C::BM;
    for (int s = 0; s < nrb; ++s) {
        const int rb = TRANS ? s : nrb - 1 - s;
        const int r0 = rb * C::BM, mr = min(C::BM, n - r0);
        for (int c0 = 0; c0 < w; c0 += C::BN) {
            const int wc = min(C::BN, w - c0);
            Acc<C> acc;
            acc.zero();
            if (!TRANS) cta_gemm(acc, X.sub(r0, 0), B.sub(0, c0).t(), mr, wc, r0 + mr, smem);
            else cta_gemm(acc, X.sub(r0, r0).t(), B.sub(r0, c0).t(), mr, wc, n - r0, smem);
            acc.store_to(B.sub(r0, c0), mr, wc);
            cta_sync();
        }
    }
}

// Split point of an n-wide recursion level: a multiple of 64, at least half.
__device__ __forceinline__ int split_point(int n) { return ((n / 2 + 63) / 64) * 64; }

// Recursive factor (FACT) or inverse-only (!FACT) of an n x n lower tile,
// n <= 64 << LVL.  A: the tile (lower triangle read / written, upper never
// touched); X: its inverse, n x n, written in full.
template <class T, int SP, bool FACT, int LVL>
__device__ __noinline__ int rec_tile(const ViewT<T> &A, const ViewT<T> &X, int n, T *smem) {
    if constexpr (LVL == 0) {
        return leaf64<T, FACT>(A, X, n, smem);
    } else {
        if (n <= (64 << (LVL - 1))) return rec_tile<T, SP, FACT, LVL - 1>(A, X, n, smem);
        using C = CB<T, SP>;
        const int n1 = split_point(n), n2 = n - n1;
        const ViewT<T> A21 = A.sub(n1, 0), A22 = A.sub(n1, n1);
        const ViewT<T> X11 = X, X21 = X.sub(n1, 0), X22 = X.sub(n1, n1);
        int info = rec_tile<T, SP, FACT, LVL - 1>(A, X11, n1, smem);
        if (info) return info;
        if (FACT) {
            apply_inv_right<T, SP>(A21, n2, X11, n1, smem);   // L21 = A21 X11^T
            // A22 -= L21 L21^T, lower blocks only
            for (int r0 = 0; r0 < n2; r0 += C::BM) {
                const int mr = min(C::BM, n2 - r0);
                for (int c0 = 0; c0 <= r0; c0 += C::BN) {
                    const int w = min(C::BN, n2 - c0);
                    Acc<C> acc;
                    acc.zero();
                    cta_gemm(acc, A21.sub(r0, 0), A21.sub(c0, 0), mr, w, n1, smem);
                    acc.sub_from(A22.sub(r0, c0), mr, w, r0 == c0);
                }
            }
            cta_sync();
        }
        info = rec_tile<T, SP, FACT, LVL - 1>(A22, X22, n2, smem);
        if (info) return n1 + info;
        // W = L21 X11 into the X21 block (X11 lower: column block c0 needs k >= c0)
        for (int r0 = 0; r0 < n2; r0 += C::BM) {
            const int mr = min(C::BM, n2 - r0);
            for (int c0 = 0; c0 < n1; c0 += C::BN) {
                const int w = min(C::BN, n1 - c0);
                Acc<C> acc;
                acc.zero();
                cta_gemm(acc, A21.sub(r0, c0), X11.sub(c0, c0).t(), mr, w, n1 - c0, smem);
                acc.store_to(X21.sub(r0, c0), mr, w);
            }
        }
        cta_sync();
        // X21 = -X22 W in place, row blocks from the last
        const int nrb = (n2 + C::BM - 1) / C::BM;
        for (int rb = nrb - 1; rb >= 0; --rb) {
            const int r0 = rb * C::BM, mr = min(C::BM, n2 - r0);
            for (int c0 = 0; c0 < n1; c0 += C::BN) {
                const int w = min(C::BN, n1 - c0);
                Acc<C> acc;
                acc.zero();
                cta_gemm(acc, X22.sub(r0, 0), X21.sub(0, c0).t(), mr, w, r0 + mr, smem);
                acc.for_each([&](int r, int c, T v) {
                    if (r < mr && c < w) *X21.at(r0 + r, c0 + c) = -v;
                });
                cta_sync();
            }
        }
        // the upper-right block of the inverse is zero
        for (int idx = threadIdx.x; idx < n1 * n2; idx += NT_CTA) *X.at(idx % n1, n1 + idx / n1) = T(0);
        cta_sync();
        return 0;
    }
}

constexpr int MAX_LVL = 4;   // tiles up to 64 << 4 = 1024

template <class T, int SP>
__device__ __forceinline__ int tile_potrf_inv(const ViewT<T> &A, const ViewT<T> &X, int n, T *smem) {
    return rec_tile<T, SP, true, MAX_LVL>(A, X, n, smem);
}
template <class T, int SP>
__device__ __forceinline__ void tile_trtri(const ViewT<T> &A, const ViewT<T> &X, int n, T *smem) {
    rec_tile<T, SP, false, MAX_LVL>(A, X, n, smem);
}

// Shared memory of the leaf (the GEMM passes use the tile kernels' stages).
constexpr size_t leaf_smem_elems() { return 2 * 64 * LDS; }

}  // namespace rec
}  // namespace chb
