// potrf_smem.cuh -- Cholesky of an FP32 diagonal tile of order n <= 256 held
// entirely in shared memory, with the inverted 64 x 64 diagonal blocks.
//
// The diagonal-tile factorization is the critical path of the tile Cholesky
// DAG (compute/pzpotrf.c: potrf(k) -> trsm(m,k) -> update(k+1,k+1) ->
// potrf(k+1)).  The blocked tile kernels (rec.cuh) stream the tile through L2
// once per 64-column step; under the load of the trailing updates every such
// round trip costs microseconds, and their fully unrolled warp leaves are
// fetched from a busy L2 instruction by instruction.  Here the whole lower
// triangle (160 KB at n = 256) is loaded once, factored on chip by all 256
// threads with small loops, and written back once.
//
// Layout: the lower triangle by 64-wide block columns; block column b holds
// rows 64 b .. n-1, column-major with a leading dimension rounded up to a
// multiple of 4 (float4 row loads).  Right-looking over block columns:
//   leaf:     D_bb = L_bb L_bb^T and X_b = L_bb^-1 (the warp-level 64 x 64
//             leaf of rec.cuh on a staged copy of the block)
//   panel:    L_ib = A_ib X_b^T                      (i > b)
//   trailing: A_ij -= L_ib L_jb^T                    (i >= j > b)
// Same contract as CORE_spotrf on a lower view (coreblas/compute/core_zpotrf.c
// :75-81): lower triangle overwritten by L, upper untouched, LAPACK info; the
// inverted blocks go to invd (IB x IB, ld IB, zero outside the block), as the
// executor's panel solves expect.
#pragma once
#include "core.cuh"
#include "rec.cuh"

namespace chb {
namespace psm {

constexpr int MAXN = 256;   // largest tile order
constexpr int BW = 64;      // block-column width (= IB)
constexpr int LDI = 65;     // leading dimension of the staged block and its inverse
static_assert(LDI == rec::LDS, "the staged leaf uses the leading dimension of rec.cuh");

__host__ __device__ constexpr int blk_ld(int n, int b) { return ((n - BW * b) + 3) & ~3; }
__host__ __device__ constexpr int blk_off(int n, int b) {
    int o = 0;
    for (int i = 0; i < b; ++i) o += BW * blk_ld(n, i);
    return o;
}
// Shared memory: the block columns, the staged diagonal block and its inverse
// (floats; 16-byte aligned base).
constexpr int SMEM_FLOATS = blk_off(MAXN, MAXN / BW) + 2 * BW * LDI + 8;
constexpr size_t SMEM_BYTES = (size_t)SMEM_FLOATS * sizeof(float);

// Cholesky of the nbk x nbk block (nbk <= 64) at D (column-major, ld ldd,
// lower triangle) in place, and its inverse into Xs (ld LDI, 64 x 64: zeros
// above the diagonal and outside nbk).  The block is staged, identity-padded,
// into sD (64 x LDI) for the warp-level 64 x 64 leaf of rec.cuh (32 x 32
// Cholesky and inverse kernels in rolled form).  Returns LAPACK info.  All 256
// threads; ends with a barrier.
static __device__ __noinline__ int leaf(float *D, int ldd, int nbk, float *sD) {
    float *Xs = sD + BW * LDI;   // the leaf's inverse follows the staged block
    for (int idx = threadIdx.x; idx < 64 * 64; idx += NT_CTA) {
        const int r = idx & 63, c = idx >> 6;
        float v = (r == c) ? 1.f : 0.f;
        if (r < nbk && c < nbk) v = (r >= c) ? D[c * ldd + r] : 0.f;
        sD[c * LDI + r] = v;
    }
    __syncthreads();
    const int info = rec::leaf64_core<float, true>(sD);
    if (info) return info;
    for (int idx = threadIdx.x; idx < 64 * 64; idx += NT_CTA) {
        const int r = idx & 63, c = idx >> 6;
        if (r < nbk && c < nbk) {
            if (r >= c) D[c * ldd + r] = sD[c * LDI + r];
        } else {
            Xs[c * LDI + r] = 0.f;   // the identity padding's inverse
        }
    }
    __syncthreads();
    return 0;
}

// acc(i, c) = sum_{k < K} Xm(i, k) Ym(c, k) for rows i < M (M <= 192) and
// columns c < 64.  Xm: column-major (ld ldx, multiple of 4; 16-byte aligned
// base), Ym(c, k) at Ym[k * ldy + c].  Thread mapping: columns tj + 16 q,
// rows 4 ti + e + 64 g (float4 loads of four rows).
struct Frag {
    float v[3][4][4];   // [row group g][row e][column q]
};
static __device__ __forceinline__ void gemm64(Frag &acc, const float *Xm, int ldx, int M, const float *Ym, int ldy, int K) {
    const int tj = threadIdx.x & 15, ti = threadIdx.x >> 4;
#pragma unroll
    for (int g = 0; g < 3; ++g)
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc.v[g][e][q] = 0.f;
    const int ng = (M + 63) / 64;
#pragma unroll 2
    for (int k = 0; k < K; ++k) {
        float y[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) y[q] = Ym[k * ldy + tj + 16 * q];
#pragma unroll
        for (int g = 0; g < 3; ++g) {
            if (g < ng) {
                const float4 xv = *reinterpret_cast<const float4 *>(Xm + k * ldx + 4 * ti + 64 * g);
                const float xs[4] = {xv.x, xv.y, xv.z, xv.w};
#pragma unroll
                for (int e = 0; e < 4; ++e)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc.v[g][e][q] = fmaf(xs[e], y[q], acc.v[g][e][q]);
            }
        }
    }
}

// Factor the n x n lower view T (n <= MAXN) through shared memory `sm`
// (SMEM_BYTES, 16-byte aligned); inverted blocks to invd.  Returns info.
// All 256 threads.
static __device__ int potrf(const ViewF &T, int n, float *invd, float *sm, unsigned *ph = nullptr) {
    const int tid = threadIdx.x;
    const int nb = (n + BW - 1) / BW;
    float *sDl = sm + blk_off(n, nb);   // staged leaf block, then its inverse
    float *Xs = sDl + BW * LDI;
    // tracing (ph != null): thread 0 adds the clock cycles of the leaves, the
    // panel products and the trailing updates (with the load and the
    // write-back) to ph[0..2]
    long long c0 = (ph && tid == 0) ? clock64() : 0;
    auto lap = [&](int i) {
        if (ph && tid == 0) {
            const long long c1 = clock64();
            ph[i] += (unsigned)(c1 - c0);
            c0 = c1;
        }
    };
    // Load block column b (rows 64 b .. n-1, all 64 columns; the part above
    // the diagonal is never read).  A column-major tile with 16-byte aligned
    // columns is copied with 16-byte cp.async, every copy of the tile in
    // flight at once; otherwise element by element, coalesced along the
    // contiguous direction, eight loads in flight per thread.
    const bool colmajor = (T.rs == 1);
    const bool vec = colmajor && ((reinterpret_cast<uintptr_t>(T.p) & 15) == 0) && (T.cs % 4 == 0);
    if (vec) {
        for (int b = 0; b < nb; ++b) {
            const int rows = n - BW * b, ld = blk_ld(n, b), nq = ld / 4, wb = min(BW, n - BW * b);
            float *Sb = sm + blk_off(n, b);
            for (int idx = tid; idx < nq * wb; idx += NT_CTA) {
                const int q = idx % nq, c = idx / nq, r = 4 * q;
                const int nv = max(0, min(4, rows - r));
                const float *src = T.at(BW * b + r, BW * b + c);
                cp_async16(Sb + c * ld + r, nv ? src : T.p, nv * 4);
            }
        }
        cp_async_commit();
        cp_async_wait<0>();
    } else {
        for (int idx0 = tid; idx0 < n * n; idx0 += 8 * NT_CTA) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = idx0 + u * NT_CTA;
                const int i = colmajor ? idx % n : idx / n, j = colmajor ? idx / n : idx % n;
                v[u] = (idx < n * n && i >= j) ? *T.at(i, j) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = idx0 + u * NT_CTA;
                const int i = colmajor ? idx % n : idx / n, j = colmajor ? idx / n : idx % n;
                if (idx < n * n && i >= j) {
                    const int b = j / BW;
                    sm[blk_off(n, b) + (j - BW * b) * blk_ld(n, b) + (i - BW * b)] = v[u];
                }
            }
        }
    }
    __syncthreads();
    lap(2);
    int info = 0;
    for (int b = 0; b < nb; ++b) {
        float *Sb = sm + blk_off(n, b);
        const int ldb = blk_ld(n, b), nbk = min(BW, n - BW * b);
        const int linfo = leaf(Sb, ldb, nbk, sDl);
        lap(0);
        if (linfo) {
            info = BW * b + linfo;
            break;
        }
        float *inv = invd + (int64_t)b * IB * IB;
        for (int idx = tid; idx < IB * IB; idx += NT_CTA) inv[idx] = Xs[(idx / IB) * LDI + (idx % IB)];
        const int M = n - BW * (b + 1);   // rows below the diagonal block
        if (M <= 0) break;
        // panel: L_ib = A_ib X_b^T, computed in registers, then stored in place
        {
            Frag acc;
            gemm64(acc, Sb + BW, ldb, M, Xs, LDI, nbk);   // X_b(c, k) at Xs[k * LDI + c]
            __syncthreads();
            const int tj = tid & 15, ti = tid >> 4;
#pragma unroll
            for (int g = 0; g < 3; ++g)
#pragma unroll
                for (int e = 0; e < 4; ++e)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int r = 4 * ti + e + 64 * g, c = tj + 16 * q;
                        if (r < M && c < nbk) Sb[c * ldb + BW + r] = acc.v[g][e][q];
                    }
            __syncthreads();
        }
        lap(1);
        // trailing: block columns c > b
        for (int cb = b + 1; cb < nb; ++cb) {
            float *Sc = sm + blk_off(n, cb);
            const int ldc = blk_ld(n, cb), Mc = n - BW * cb, wc = min(BW, n - BW * cb);
            Frag acc;
            // rows i >= 64 cb of panel b, against its rows 64 cb .. 64 cb + 63
            gemm64(acc, Sb + BW * (cb - b), ldb, Mc, Sb + BW * (cb - b), ldb, nbk);
            const int tj = tid & 15, ti = tid >> 4;
#pragma unroll
            for (int g = 0; g < 3; ++g)
#pragma unroll
                for (int e = 0; e < 4; ++e)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int r = 4 * ti + e + 64 * g, c = tj + 16 * q;
                        if (r < Mc && c < wc && r >= c) Sc[c * ldc + r] -= acc.v[g][e][q];
                    }
        }
        __syncthreads();
        lap(2);
    }
    // write back the lower triangle, block column by block column: groups of
    // four rows entirely below the diagonal as one 16-byte store when the tile
    // allows it, the rest element by element (the upper triangle is never
    // written)
    for (int b = 0; b < nb; ++b) {
        const int rows = n - BW * b, ld = blk_ld(n, b), nq = ld / 4, wb = min(BW, n - BW * b);
        const float *Sb = sm + blk_off(n, b);
        for (int idx = tid; idx < nq * wb; idx += NT_CTA) {
            const int q = colmajor ? idx % nq : idx / wb, c = colmajor ? idx / nq : idx % wb, r = 4 * q;
            if (vec && r >= c + 3 && r + 4 <= rows) {
                *reinterpret_cast<float4 *>(T.at(BW * b + r, BW * b + c)) =
                    *reinterpret_cast<const float4 *>(Sb + c * ld + r);
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (r + u < rows && r + u >= c) *T.at(BW * b + r + u, BW * b + c) = Sb[c * ld + r + u];
            }
        }
    }
    __syncthreads();
    lap(2);
    return info;
}

}  // namespace psm
}  // namespace chb
