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
//   leaf:     D_bb = L_bb L_bb^T and X_b = L_bb^-1 (64 x 64, registers: each
//             thread owns a 4 x 4 block; one barrier per column)
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
constexpr int LDI = 65;     // leading dimension of the block inverse in shared memory

__host__ __device__ constexpr int blk_ld(int n, int b) { return ((n - BW * b) + 3) & ~3; }
__host__ __device__ constexpr int blk_off(int n, int b) {
    int o = 0;
    for (int i = 0; i < b; ++i) o += BW * blk_ld(n, i);
    return o;
}
// Shared memory: the block columns, the block inverse, two 64-float broadcast
// buffers, the info word (floats; 16-byte aligned base).
constexpr int SMEM_FLOATS = blk_off(MAXN, MAXN / BW) + BW * LDI + 2 * BW + 8;
constexpr size_t SMEM_BYTES = (size_t)SMEM_FLOATS * sizeof(float);

// Cholesky of the nbk x nbk block (nbk <= 64) at D (column-major, ld ldd,
// lower triangle) in place, and its inverse into Xs (ld LDI, 64 x 64 written
// in full: zeros above the diagonal and outside nbk).  cbuf: 128 floats.
// Returns LAPACK info (1-based column of the first non-positive pivot).
// All 256 threads; ends with a barrier.
static __device__ __noinline__ int leaf(float *D, int ldd, int nbk, float *Xs, float *cbuf) {
    const int tid = threadIdx.x;
    const int r0 = 4 * (tid >> 4), c0 = 4 * (tid & 15);   // this thread's 4 x 4 block
    float a[4][4];
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const int r = r0 + e, c = c0 + f;
            a[e][f] = (r < nbk && c < nbk && r >= c) ? D[c * ldd + r] : 0.f;
        }
    if (c0 == 0) {
#pragma unroll
        for (int e = 0; e < 4; ++e) cbuf[r0 + e] = a[e][0];
    }
    __syncthreads();
    int info = 0;
    for (int j = 0; j < nbk; ++j) {
        const float *col = cbuf + (j & 1) * BW;   // column j after its j updates
        const float d = col[j];
        if (!(d > 0.f)) {   // uniform: every thread reads the same pivot (also catches NaN)
            info = j + 1;
            break;
        }
        const float rs = rec::rsqrt_wp(d);
        float li[4], lc[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) li[e] = col[r0 + e] * rs;
#pragma unroll
        for (int f = 0; f < 4; ++f) lc[f] = col[c0 + f] * rs;
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const int r = r0 + e, c = c0 + f;
                if (c > j && r >= c && r < nbk) a[e][f] -= li[e] * lc[f];
            }
        // column j is final: L(i, j) = col[i] / sqrt(d), L(j, j) = sqrt(d)
#pragma unroll
        for (int f = 0; f < 4; ++f)
            if (c0 + f == j) {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (r0 + e >= j) a[e][f] = (r0 + e == j) ? d * rs : li[e];
            }
        // column j + 1 (now updated by all j + 1 columns) to the other buffer
        if (j + 1 < nbk) {
#pragma unroll
            for (int f = 0; f < 4; ++f)
                if (c0 + f == j + 1) {
#pragma unroll
                    for (int e = 0; e < 4; ++e) cbuf[((j + 1) & 1) * BW + r0 + e] = a[e][f];
                }
        }
        __syncthreads();
    }
    if (info) return info;
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const int r = r0 + e, c = c0 + f;
            if (r < nbk && c < nbk && r >= c) D[c * ldd + r] = a[e][f];
        }
    __syncthreads();
    // X = L^-1 by rows: row i is final once divided by L(i, i); it then
    // updates the rows below (x(r, c) -= L(r, i) x(i, c)).
    float x[4][4];
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int f = 0; f < 4; ++f) x[e][f] = (r0 + e == c0 + f && r0 + e < nbk) ? 1.f : 0.f;
    for (int i = 0; i < nbk; ++i) {
        float *row = cbuf + (i & 1) * BW;
        if (i >= r0 && i < r0 + 4) {
            const float inv = 1.f / D[i * ldd + i];
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (r0 + e == i) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        x[e][f] *= inv;   // zero for c > i
                        row[c0 + f] = x[e][f];
                    }
                }
        }
        __syncthreads();
        float lr[4], xr[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) lr[e] = (r0 + e > i && r0 + e < nbk) ? D[i * ldd + r0 + e] : 0.f;
#pragma unroll
        for (int f = 0; f < 4; ++f) xr[f] = row[c0 + f];
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int f = 0; f < 4; ++f) x[e][f] -= lr[e] * xr[f];
    }
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int f = 0; f < 4; ++f) Xs[(c0 + f) * LDI + r0 + e] = x[e][f];
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
static __device__ int potrf(const ViewF &T, int n, float *invd, float *sm) {
    const int tid = threadIdx.x;
    const int nb = (n + BW - 1) / BW;
    float *Xs = sm + blk_off(n, nb);
    float *cbuf = Xs + BW * LDI;
    // load the lower triangle (coalesced along the contiguous direction of T)
    const bool colmajor = (T.rs == 1);
    for (int idx = tid; idx < n * n; idx += NT_CTA) {
        const int i = colmajor ? idx % n : idx / n, j = colmajor ? idx / n : idx % n;
        if (i >= j) {
            const int b = j / BW;
            sm[blk_off(n, b) + (j - BW * b) * blk_ld(n, b) + (i - BW * b)] = *T.at(i, j);
        }
    }
    __syncthreads();
    int info = 0;
    for (int b = 0; b < nb; ++b) {
        float *Sb = sm + blk_off(n, b);
        const int ldb = blk_ld(n, b), nbk = min(BW, n - BW * b);
        const int linfo = leaf(Sb, ldb, nbk, Xs, cbuf);
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
    }
    // write back the lower triangle
    for (int idx = tid; idx < n * n; idx += NT_CTA) {
        const int i = colmajor ? idx % n : idx / n, j = colmajor ? idx / n : idx % n;
        if (i >= j) {
            const int b = j / BW;
            *T.at(i, j) = sm[blk_off(n, b) + (j - BW * b) * blk_ld(n, b) + (i - BW * b)];
        }
    }
    __syncthreads();
    return info;
}

}  // namespace psm
}  // namespace chb
