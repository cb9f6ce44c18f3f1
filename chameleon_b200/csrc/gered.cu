// gered.cu -- adaptive per-tile precision of a symmetric matrix (gered) and
// its restoration (gerst).
//
// Reference: CHAMELEON_zgered_Tile / chameleon_pzgered (compute/zgered.c,
// compute/pzgered.c:160-260) and the conversion rule of INSERT_TASK_zgered
// (runtime/starpu/codelets/codelet_zgered.c, the CUDA build in double
// precision); CHAMELEON_zgerst_Tile / chameleon_pzgerst (compute/pzgerst.c).
//   gnorm      = Frobenius norm of the referenced triangle of A
//   eps        = prec if prec >= 0, else the FP64 unit roundoff (dlamch 'e')
//   threshold  = eps gnorm / min(MT, NT); on the diagonal tiles the same, or
//                the FP32 unit roundoff in place of eps when eps is larger
//   tile (m,n) of the triangle, of Frobenius norm |A_mn| (diagonal tiles:
//   their referenced triangle):
//     |A_mn| < threshold / 1e-4          -> FP16
//     else |A_mn| < threshold / slamch   -> FP32
//     else                               -> FP64 (unchanged)
// The reference stores a reduced tile in the lower precision (the tile's
// flttype changes, and later kernels read it as such).  Here the descriptor
// keeps its FP64 layout: a reduced tile is rounded in place to the values of
// its precision (round to nearest even, FP16 overflow to +-inf as the
// conversion does) and carries a precision tag, read back with
// CHAM_B200_Tile_Precision; gerst resets the tags to FP64 (the values stay
// rounded, as the reference's conversion back to FP64 leaves them).
// The norms: one CTA per tile, scaled sums of squares (LAPACK's scale/ssq
// pairs, so no overflow), combined on the host.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "core.cuh"
#include "internal.h"

namespace chb {

struct GeredTile {
    int64_t off;
    int ld, rows, cols;
    int tri;   // 0: full tile, 1: lower triangle, 2: upper triangle
};

// out[2 i] = max |a|, out[2 i + 1] = sum (a / max)^2 over the tile's part.
__global__ void tile_ssq_kernel(const GeredTile *tiles, const double *A, double *out) {
    const GeredTile t = tiles[blockIdx.x];
    const double *a = A + t.off;
    __shared__ double red[NT_CTA / 32];
    auto inside = [&](int r, int c) { return t.tri == 0 || (t.tri == 1 ? r >= c : r <= c); };
    double mx = 0.0;
    for (int idx = threadIdx.x; idx < t.rows * t.cols; idx += blockDim.x) {
        const int r = idx % t.rows, c = idx / t.rows;
        if (inside(r, c)) mx = fmax(mx, fabs(a[r + (int64_t)c * t.ld]));
    }
    for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    mx = 0.0;
    for (int w = 0; w < NT_CTA / 32; ++w) mx = fmax(mx, red[w]);
    __syncthreads();
    double s = 0.0;
    if (mx > 0.0) {
        for (int idx = threadIdx.x; idx < t.rows * t.cols; idx += blockDim.x) {
            const int r = idx % t.rows, c = idx / t.rows;
            if (inside(r, c)) {
                const double v = a[r + (int64_t)c * t.ld] / mx;
                s += v * v;
            }
        }
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < NT_CTA / 32; ++w) tot += red[w];
        out[2 * blockIdx.x] = mx;
        out[2 * blockIdx.x + 1] = tot;
    }
}

// Round every entry of the tiles to their precision (1: FP32, 2: FP16).
__global__ void tile_round_kernel(const GeredTile *tiles, const int *prec, double *A) {
    const GeredTile t = tiles[blockIdx.x];
    const int p = prec[blockIdx.x];
    if (p == 0) return;
    double *a = A + t.off;
    for (int idx = threadIdx.x; idx < t.rows * t.cols; idx += blockDim.x) {
        const int r = idx % t.rows, c = idx / t.rows;
        double &v = a[r + (int64_t)c * t.ld];
        v = (p == 1) ? (double)__double2float_rn(v) : (double)__half2float(__double2half(v));
    }
}

namespace {

// Tiles of the uplo triangle (tile-wise, as pzgered walks them).
std::vector<GeredTile> triangle_tiles(const CHAM_desc_t *A, cham_uplo_t uplo, std::vector<std::pair<int, int>> *mn) {
    std::vector<GeredTile> out;
    for (int m = 0; m < A->mt; ++m) {
        const int nmin = uplo == ChamUpper ? m : 0;
        const int nmax = uplo == ChamLower ? std::min(m + 1, A->nt) : A->nt;
        for (int n = nmin; n < nmax; ++n) {
            const int tri = (m == n && uplo != ChamUpperLower) ? (uplo == ChamLower ? 1 : 2) : 0;
            out.push_back(GeredTile{desc_tile_off(A, m, n), desc_tile_ld(A, m), desc_tile_rows(A, m),
                                    desc_tile_cols(A, n), tri});
            if (mn) mn->push_back({m, n});
        }
    }
    return out;
}

std::vector<signed char> &tags_of(CHAM_desc_t *A) {
    DescPriv *pv = priv(A);
    if (pv->prec.size() != (size_t)A->mt * A->nt) pv->prec.assign((size_t)A->mt * A->nt, 0);
    return pv->prec;
}

}  // namespace
}  // namespace chb

using namespace chb;

extern "C" {

int CHAMELEON_dgered_Tile(cham_uplo_t uplo, double prec, CHAM_desc_t *A) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || A->dtyp != ChamRealDouble) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (uplo != ChamUpper && uplo != ChamLower && uplo != ChamUpperLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    std::vector<std::pair<int, int>> mn;
    std::vector<GeredTile> tiles = triangle_tiles(A, uplo, &mn);
    if (tiles.empty()) return 0;
    cudaStream_t s = ctx().stream;
    const size_t nt = tiles.size();
    GeredTile *d_tiles = (GeredTile *)dev_alloc(nt * sizeof(GeredTile));
    double *d_ssq = (double *)dev_alloc(2 * nt * sizeof(double));
    int *d_prec = (int *)dev_alloc(nt * sizeof(int));
    if (!d_tiles || !d_ssq || !d_prec) {
        dev_free(d_tiles);
        dev_free(d_ssq);
        dev_free(d_prec);
        return CHAMELEON_ERR_OUT_OF_RESOURCES;
    }
    std::vector<double> ssq(2 * nt);
    std::vector<int> pr(nt, 0);
    rc = 0;
    if (cudaMemcpyAsync(d_tiles, tiles.data(), nt * sizeof(GeredTile), cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = CHAMELEON_ERR_UNEXPECTED;
    if (!rc) {
        tile_ssq_kernel<<<(unsigned)nt, NT_CTA, 0, s>>>(d_tiles, (const double *)A->mat, d_ssq);
        CHB_LAUNCHED(1);
        if (cudaMemcpyAsync(ssq.data(), d_ssq, 2 * nt * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            rc = CHAMELEON_ERR_UNEXPECTED;
    }
    if (!rc) {
        // combine the (scale, ssq) pairs: gnorm^2 = sum_t (scale_t)^2 ssq_t
        double big = 0.0;
        for (size_t i = 0; i < nt; ++i) big = std::max(big, ssq[2 * i]);
        double acc = 0.0;
        if (big > 0.0)
            for (size_t i = 0; i < nt; ++i) {
                const double r = ssq[2 * i] / big;
                acc += r * r * ssq[2 * i + 1];
            }
        const double gnorm = big * std::sqrt(acc);
        const double eps = prec < 0.0 ? 0x1p-53 : prec;
        const double eps_diag = 0x1p-24;   // FP32 unit roundoff (slamch 'e')
        const double mnt = (double)std::min(A->mt, A->nt);
        const double threshold = eps * gnorm / mnt;
        const double threshold_diag = (eps < eps_diag) ? threshold : eps_diag * gnorm / mnt;
        std::vector<signed char> &tags = tags_of(A);
        for (size_t i = 0; i < nt; ++i) {
            const int m = mn[i].first, n = mn[i].second;
            const double lnorm = ssq[2 * i] * std::sqrt(ssq[2 * i + 1]);
            const double th = (m == n) ? threshold_diag : threshold;
            int p = 0;
            if (lnorm < th / 1e-4) p = 2;
            else if (lnorm < th / eps_diag) p = 1;
            // a tile already reduced keeps its lower precision
            const int cur = tags[m + (size_t)A->mt * n];
            if (cur > p) p = 0;
            pr[i] = p;
            if (p) tags[m + (size_t)A->mt * n] = (signed char)p;
        }
        if (cudaMemcpyAsync(d_prec, pr.data(), nt * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = CHAMELEON_ERR_UNEXPECTED;
        if (!rc) {
            tile_round_kernel<<<(unsigned)nt, NT_CTA, 0, s>>>(d_tiles, d_prec, (double *)A->mat);
            CHB_LAUNCHED(1);
            if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
                rc = CHAMELEON_ERR_UNEXPECTED;
        }
    }
    dev_free(d_tiles);
    dev_free(d_ssq);
    dev_free(d_prec);
    if (rc) return rc;
    return desc_sync_to_host(A);
}

int CHAMELEON_dgerst_Tile(cham_uplo_t uplo, CHAM_desc_t *A) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || A->dtyp != ChamRealDouble) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (uplo != ChamUpper && uplo != ChamLower && uplo != ChamUpperLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    std::vector<signed char> &tags = tags_of(A);
    for (int m = 0; m < A->mt; ++m) {
        const int nmin = uplo == ChamUpper ? m : 0;
        const int nmax = uplo == ChamLower ? std::min(m + 1, A->nt) : A->nt;
        for (int n = nmin; n < nmax; ++n) tags[m + (size_t)A->mt * n] = 0;
    }
    return 0;
}

int CHAM_B200_Tile_Precision(const CHAM_desc_t *A, int m, int n) {
    if (!A || m < 0 || n < 0 || m >= A->mt || n >= A->nt) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const DescPriv *pv = priv(A);
    const int p = pv->prec.size() == (size_t)A->mt * A->nt ? pv->prec[m + (size_t)A->mt * n] : 0;
    return p == 2 ? ChamRealHalf : p == 1 ? ChamRealFloat : ChamRealDouble;
}

}  // extern "C"
