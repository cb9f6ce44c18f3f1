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
// rows 64 b .. n-1, column-major with a padded leading dimension (blk_ld).  Right-looking over block columns:
//   leaf:     D_bb = L_bb L_bb^T and X_b = L_bb^-1 (the warp-level 64 x 64
//             leaf of rec.cuh on a staged copy of the block)
//   panel:    L_ib = A_ib X_b^T                      (i > b)
//   trailing: A_ij -= L_ib L_jb^T                    (i >= j > b)
// (the panel and trailing products on the tensor cores as 3xTF32)
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

// Leading dimension of block column b: its rows rounded up to 32, plus 8
// (8 mod 32: the tensor-core fragment loads -- 8 consecutive rows at 4
// columns -- then hit 32 distinct banks; a multiple of 4 keeps the columns
// 16-byte aligned for the vectorized load and write-back).
__host__ __device__ constexpr int blk_ld(int n, int b) { return (((n - BW * b) + 31) & ~31) + 8; }
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
// columns c < 64 on the tensor cores: mma.sync m16n8k8 TF32 with each operand
// split in two TF32 parts and three products (hi*hi + hi*lo + lo*hi, close to
// FP32 accuracy).  Xm: column-major (ld ldx), Ym(c, k) at Ym[k * ldy + c].
// Warp w owns rows 48 (w & 3) .. +47 (three 16-row tiles) and columns
// 32 (w >> 2) .. +31 (four 8-column tiles); rows >= M and k >= K read as
// zero, so no operand entry outside them is read.
struct Frag {
    float v[3][4][4];   // [row tile][column tile][mma accumulator]
};
static __device__ __forceinline__ void gemm64(Frag &acc, const float *Xm, int ldx, int M, const float *Ym, int ldy,
                                              int K) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = 48 * (w & 3), c0 = 32 * (w >> 2);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc.v[i][j][e] = 0.f;
    const int nm = M > r0 ? min(3, (M - r0 + 15) / 16) : 0;   // row tiles with rows < M (warp-uniform)
    if (nm == 0) return;
#pragma unroll 1
    for (int k8 = 0; k8 < K; k8 += 8) {
        const int ka = k8 + t, kb = k8 + t + 4;
        const bool va = ka < K, vb = kb < K;
        // the four column tiles' fragments stay live; each row tile's are
        // loaded just before its products (fewer live registers)
        uint32_t bh[4][2], bl[4][2];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + 8 * j + g;
            split_tf32(va ? Ym[ka * ldy + c] : 0.f, bh[j][0], bl[j][0]);
            split_tf32(vb ? Ym[kb * ldy + c] : 0.f, bh[j][1], bl[j][1]);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (i < nm) {
                const int ra = r0 + 16 * i + g, rb = ra + 8;
                uint32_t ah[4], al[4];
                split_tf32((va && ra < M) ? Xm[ka * ldx + ra] : 0.f, ah[0], al[0]);
                split_tf32((va && rb < M) ? Xm[ka * ldx + rb] : 0.f, ah[1], al[1]);
                split_tf32((vb && ra < M) ? Xm[kb * ldx + ra] : 0.f, ah[2], al[2]);
                split_tf32((vb && rb < M) ? Xm[kb * ldx + rb] : 0.f, ah[3], al[3]);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    mma_tf32_1688(acc.v[i][j], al, bh[j]);
                    mma_tf32_1688(acc.v[i][j], ah, bl[j]);
                    mma_tf32_1688(acc.v[i][j], ah, bh[j]);
                }
            }
        }
    }
}

// f(row, column, value) over this thread's accumulators (rows may be >= M:
// their values are zero and the caller's row guard skips them).
template <class F>
static __device__ __forceinline__ void frag_each(const Frag &acc, F &&f) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int r0 = 48 * (w & 3), c0 = 32 * (w >> 2);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = r0 + 16 * i + g, c = c0 + 8 * j + 2 * t;
            f(r, c, acc.v[i][j][0]);
            f(r, c + 1, acc.v[i][j][1]);
            f(r + 8, c, acc.v[i][j][2]);
            f(r + 8, c + 1, acc.v[i][j][3]);
        }
}

// Factor the n x n lower view T (n <= MAXN) through shared memory `sm`
// (SMEM_BYTES, 16-byte aligned); inverted blocks to invd.  Returns info.
// All 256 threads.
static __device__ __noinline__ int potrf(const ViewF &T, int n, float *invd, float *sm, unsigned *ph = nullptr) {
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
            frag_each(acc, [&](int r, int c, float v) {
                if (r < M && c < nbk) Sb[c * ldb + BW + r] = v;
            });
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
            frag_each(acc, [&](int r, int c, float v) {
                if (r < Mc && c < wc && r >= c) Sc[c * ldc + r] -= v;
            });
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
