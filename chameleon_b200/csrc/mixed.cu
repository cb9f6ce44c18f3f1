// mixed.cu -- mixed-precision Cholesky solve with FP64 iterative refinement.
//
// The reference has no working mixed solver: zcposv / zcgesv are commented out
// of its build (compute/CMakeLists.txt:211-212, include/chameleon/chameleon_zc.h
// :33-42); only the tile casts chameleon_pzlag2c / pclag2z exist
// (compute/pzlag2c.c:33-104).  This file restates LAPACK's dsposv scheme (the
// CPU comparator, LAPACKE_dsposv) on the B200 path:
//
//   A32 = float(A)                        (tile cast, overflow -> FP64 fallback)
//   L32 = chol(A32)                       (tile-DAG executor, FP32 storage,
//                                          BF16x3 or TF32x3 tensor-core GEMMs)
//   X   = double(L32^-T L32^-1 float(B))
//   repeat: R = B - A X (FP64, DMMA)      converged when, for every column,
//           max|R| <= max|X| * ||A||_inf * eps * sqrt(N)   (dsposv's test)
//           X += double(L32^-T L32^-1 float(R))
//   after REFINE_MAXITER iterations without convergence: FP64 dposv on A.
//
// ITER follows LAPACK: >= 0 iterations used; -2 overflow in the cast; -3 the
// low-precision factorization failed; -(maxiter+1) refinement did not
// converge.  On fallback A holds the FP64 factor (as in dsposv).
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "core.cuh"
#include "internal.h"

namespace chb {

struct TileMapD {
    void *base;
    const int64_t *off;
    const int *ld;
    int mt, mb, nb;
    template <class T>
    __device__ T *at(int i, int j) const {
        const int m = i / mb, n = j / nb;
        return static_cast<T *>(base) + off[m + (int64_t)mt * n] + (i - m * mb) + (int64_t)(j - n * nb) * ld[m];
    }
};

// Device tile map of a descriptor.  Its offset table must be on the device
// already (desc_upload); every workspace descriptor is uploaded at creation.
static TileMapD tmap(CHAM_desc_t *d) {
    return TileMapD{d->mat, priv(d)->dev.off, priv(d)->dev.ld, d->mt, d->mb, d->nb};
}
static bool uploaded(const CHAM_desc_t *d) { return priv(d)->dev.off != nullptr && priv(d)->dev.ld != nullptr; }

// Flat cast of tile storage with identical layout (CCRB -> CCRB, same tiling):
// element offsets coincide, so the cast is one coalesced pass over the storage.
__global__ void cast_d2s_flat(const double *__restrict__ src, float *__restrict__ dst, size_t n, int *overflow) {
    size_t i = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) * 4;
    const size_t stride = (size_t)gridDim.x * blockDim.x * 4;
    int ovf = 0;
    for (; i + 3 < n; i += stride) {
        const double2 a = *reinterpret_cast<const double2 *>(src + i);
        const double2 b = *reinterpret_cast<const double2 *>(src + i + 2);
        ovf |= (fabs(a.x) > 3.4028234663852886e38) | (fabs(a.y) > 3.4028234663852886e38) |
               (fabs(b.x) > 3.4028234663852886e38) | (fabs(b.y) > 3.4028234663852886e38);
        *reinterpret_cast<float4 *>(dst + i) =
            make_float4(__double2float_rn(a.x), __double2float_rn(a.y), __double2float_rn(b.x), __double2float_rn(b.y));
    }
    for (; i < n; ++i) {   // tail (only the last thread range)
        ovf |= fabs(src[i]) > 3.4028234663852886e38;
        dst[i] = __double2float_rn(src[i]);
    }
    if (ovf && overflow) *overflow = 1;
}

// Generic element-wise cast through the two tile maps (any layouts).
template <class S, class D>
__global__ void cast_tiles(TileMapD s, TileMapD d, int M, int N, int *overflow) {
    const int64_t total = (int64_t)M * N;
    int ovf = 0;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        const double v = (double)*s.at<S>(i, j);
        if (overflow) ovf |= fabs(v) > 3.4028234663852886e38;
        *d.at<D>(i, j) = (D)v;
    }
    if (ovf && overflow) *overflow = 1;
}

// X += double(D) on N x nrhs tile-layout operands.
__global__ void add_correction(TileMapD x, TileMapD d, int M, int N) {
    const int64_t total = (int64_t)M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        *x.at<double>(i, j) += (double)*d.at<float>(i, j);
    }
}

// Logical lower tile (m,n), m >= n, of a symmetric matrix stored in `uplo`.
// Only the `uplo` triangle is referenced (LAPACK convention): the diagonal
// tiles are read through `diag`, full symmetric copies made by sym_diag_kernel.
struct SymTiles {
    double *A;
    const int64_t *off;
    const int *ld;
    int NT, N, NB, upper;
    double *diag;   // NT tiles of NB x NB, column-major, ld NB
    __device__ int tm(int m) const { return (m == NT - 1) ? N - m * NB : NB; }
    __device__ View L(int m, int n) const {
        if (!upper) return View{A + off[m + NT * n], 1, ld[m]};
        return View{A + off[n + NT * m], ld[n], 1};
    }
    __device__ View D(int m) const { return View{diag + (int64_t)m * NB * NB, 1, NB}; }
};

// diag[m] = the full symmetric diagonal tile (m,m), from its `uplo` triangle.
__global__ void sym_diag_kernel(SymTiles a) {
    const int m = blockIdx.y;
    const int n = a.tm(m);
    const View L = a.L(m, m);
    double *d = a.diag + (int64_t)m * a.NB * a.NB;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
        const int i = idx % n, j = idx / n;
        d[i + (int64_t)j * a.NB] = (i >= j) ? *L.at(i, j) : *L.at(j, i);
    }
}

// Residual GEMM tile: 128 x 64 FP64 outputs, 2-stage cp.async pipeline, two
// CTAs per SM (16 warps feed the DMMA pipe; 111 KB of stages each).
using CfgRes = GemmCfg<double, 128, 64, 4, 2, SPLIT_BF16X3, 2>;
constexpr int RES_CTAS_PER_SM = 2;

// R = B - A X for symmetric A (one triangle stored), FP64 on DMMA.  One CTA
// per (tile row m, 128-row block, 64-column block of the right-hand sides, K
// part): it sweeps tile columns [kp NT / ksplit, (kp + 1) NT / ksplit) of the
// block row of A.  ksplit == 1: writes R and the per-column max |R|; else the
// partial product goes to part[kp] (N x nrhs, ld N) for residual_reduce_kernel,
// which adds the parts in a fixed order (deterministic).
__global__ void __launch_bounds__(NT_CTA, RES_CTAS_PER_SM) sym_residual_kernel(SymTiles a, TileMapD xb, TileMapD bb, TileMapD rb,
                                                                 int nrhs, int nrb, int ncb, int ksplit,
                                                                 double *part, unsigned long long *rmax) {
    extern __shared__ __align__(128) double smem[];
    const int kp = blockIdx.x % ksplit;
    const int task = blockIdx.x / ksplit;
    const int cb = task % ncb;            // 64-column block, aligned to the tile columns of X
    const int mr = task / ncb;            // (m, row block) flattened
    const int m = mr / nrb, rblk = mr % nrb;
    const int r0 = rblk * 128;
    if (m >= a.NT || r0 >= a.tm(m)) return;
    const int rows = min(128, a.tm(m) - r0);
    const int per_tile = (xb.nb + 63) / 64;
    const int bn = cb / per_tile;
    const int c0 = bn * xb.nb + (cb % per_tile) * 64;
    const int w = min(min(64, (bn + 1) * xb.nb - c0), nrhs - c0);
    if (w <= 0) return;
    Acc<CfgRes> acc;
    acc.zero();
    const int n0 = kp * a.NT / ksplit, n1 = (kp + 1) * a.NT / ksplit;
    for (int n = n0; n < n1; ++n) {
        const View An = (n < m) ? a.L(m, n).sub(r0, 0) : (n == m) ? a.D(m).sub(r0, 0) : a.L(n, m).t().sub(r0, 0);
        // X tile n, columns c0..c0+w: view of the N x nrhs operand in tile layout
        double *xp = xb.at<double>(n * a.NB, c0);
        const View Xn{xp, 1, xb.ld[n]};
        cta_gemm(acc, An, Xn.t(), rows, w, a.tm(n), smem);
    }
    const int gi0 = m * a.NB + r0;
    if (ksplit > 1) {
        double *P = part + (size_t)kp * a.N * nrhs;
        acc.for_each([&](int r, int c, double v) {
            if (r < rows && c < w) P[(gi0 + r) + (size_t)(c0 + c) * a.N] = v;
        });
        return;
    }
    __shared__ unsigned long long cmax[64];
    if (threadIdx.x < 64) cmax[threadIdx.x] = 0ull;
    __syncthreads();
    // R = B - acc: B and R are different arrays; all B loads go first
    Acc<CfgRes> bv;
    acc.for_each_idx([&](int a2, int b2, int e, int r, int c, double) {
        bv.v[a2][b2][e] = (r < rows && c < w) ? __ldcg(bb.at<double>(gi0 + r, c0 + c)) : 0.0;
    });
    acc.for_each_idx([&](int a2, int b2, int e, int r, int c, double v) {
        if (r < rows && c < w) {
            const double res = bv.v[a2][b2][e] - v;
            *rb.at<double>(gi0 + r, c0 + c) = res;
            atomicMax(&cmax[c], (unsigned long long)__double_as_longlong(fabs(res)));
        }
    });
    __syncthreads();
    if (threadIdx.x < w) atomicMax(&rmax[c0 + threadIdx.x], cmax[threadIdx.x]);
}

// R = B - sum_kp part[kp] (parts added in order), and per-column max |R|:
// block (bx, j) handles a strided share of column j's rows.
__global__ void residual_reduce_kernel(const double *part, int ksplit, int N, TileMapD bb, TileMapD rb,
                                       unsigned long long *rmax) {
    __shared__ unsigned long long red[32];
    const int j = blockIdx.y;
    unsigned long long mx = 0ull;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        double sum = 0.0;
        for (int kp = 0; kp < ksplit; ++kp) sum += part[(size_t)kp * N * gridDim.y + i + (size_t)j * N];
        const double res = *bb.at<double>(i, j) - sum;
        *rb.at<double>(i, j) = res;
        const unsigned long long v = (unsigned long long)__double_as_longlong(fabs(res));
        mx = v > mx ? v : mx;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = v > mx ? v : mx;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        mx = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long v = __shfl_xor_sync(0xffffffffu, mx, o);
            mx = v > mx ? v : mx;
        }
        if (threadIdx.x == 0 && mx) atomicMax(&rmax[j], mx);
    }
}

// Per-column max |X| of an M x N operand: block (bx, j) reduces a strided
// share of column j's rows in registers and a warp/block tree, then issues one
// atomic (non-negative doubles order like their bit patterns).
__global__ void colmax_kernel(TileMapD x, int M, int N, unsigned long long *out) {
    __shared__ unsigned long long red[32];
    const int j = blockIdx.y;
    unsigned long long m = 0ull;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
        const unsigned long long v = (unsigned long long)__double_as_longlong(fabs(*x.at<double>(i, j)));
        m = v > m ? v : m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, m, o);
        m = v > m ? v : m;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long v = __shfl_xor_sync(0xffffffffu, m, o);
            m = v > m ? v : m;
        }
        if (threadIdx.x == 0 && m) atomicMax(&out[j], m);
    }
}

// Infinity norm (= one norm) of the symmetric matrix stored in its `uplo`
// triangle and, when a32.base is set, the FP32 copy of that triangle's tiles,
// in one pass over the referenced tiles only.  One CTA per stored tile (p, q)
// of the triangle, read in its stored orientation: warp w takes stored rows
// w*32 + lane (+256, ...) and walks the columns, so every read is one
// coalesced 256-byte row segment.  Row sums stay in registers, column sums are
// warp-reduced into shared memory; each goes to the row it belongs to by
// symmetry (stored row i of tile p -> row p*NB + i, stored column j of tile q
// -> row q*NB + j).  On a diagonal tile only the referenced triangle counts:
// row sums without the diagonal, column sums with it.  overflow is set when a
// referenced value does not fit FP32.  Dynamic shared memory: NB doubles.
__global__ void __launch_bounds__(256) sym_cast_norm_kernel(SymTiles a, TileMapD a32, double *colsum,
                                                            int *overflow) {
    extern __shared__ double s_col[];
    int t = blockIdx.x;
    int m = 0;
    while (t > m) { t -= m + 1; ++m; }   // t-th lower tile (m, n) in row-major order
    const int n = t;
    const int p = a.upper ? n : m, q = a.upper ? m : n;   // stored tile
    const double *src = a.A + a.off[p + (int64_t)a.NT * q];
    const int lds = a.ld[p];
    const int rows = a.tm(p), cols = a.tm(q);
    const bool diag = (p == q);
    // the FP32 copy may use a finer tiling (tile size a32.mb dividing NB):
    // stored tile (p, q) covers sub-tiles (p r + i / mb, q r + j / mb)
    const int fb = a32.base ? a32.mb : a.NB;
    const int rsub = a.NB / fb;
    for (int j = threadIdx.x; j < cols; j += blockDim.x) s_col[j] = 0.0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int ovf = 0;
    for (int r0 = warp * 32; r0 < rows; r0 += 256) {
        const int i = r0 + lane;
        const bool rv = i < rows;
        const int rt = p * rsub + i / fb;   // sub-tile row of the FP32 copy
        const int ldd = (a32.base && rv) ? a32.ld[rt] : 0;
        double rs = 0.0;
        for (int jb = 0; jb < cols; jb += fb) {
            float *dst = (a32.base && rv)
                             ? static_cast<float *>(a32.base) + a32.off[rt + (int64_t)a32.mt * (q * rsub + jb / fb)] +
                                   (i % fb)
                             : nullptr;
            const int je = min(cols, jb + fb);
#pragma unroll 4
            for (int j = jb; j < je; ++j) {
                const double v = rv ? src[i + (int64_t)j * lds] : 0.0;
                if (dst) dst[(int64_t)(j - jb) * ldd] = __double2float_rn(v);
                const bool ref = rv && (!diag || (a.upper ? i <= j : i >= j));
                const double av = ref ? fabs(v) : 0.0;
                ovf |= av > 3.4028234663852886e38;
                if (!diag || i != j) rs += av;
                double cs = av;
#pragma unroll
                for (int o = 16; o; o >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, o);
                if (lane == 0 && cs != 0.0) atomicAdd(&s_col[j], cs);
            }
        }
        if (rv && rs != 0.0) atomicAdd(&colsum[(int64_t)p * a.NB + i], rs);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cols; j += blockDim.x)
        if (s_col[j] != 0.0) atomicAdd(&colsum[(int64_t)q * a.NB + j], s_col[j]);
    if (ovf && overflow) *overflow = 1;
}

static int ew_grid(int64_t total) {
    const int64_t b = (total + 255) / 256;
    return (int)std::min<int64_t>(std::max<int64_t>(b, 1), (int64_t)ctx().num_sms * 16);
}

namespace {
MixedWs g_mws;   // workspace of the synchronous API entry points

// Grow-only buffer of a workspace: replaced (stream-ordered) when too small.
static bool grow(void **buf, size_t *cap, size_t bytes) {
    if (bytes <= *cap) return true;
    dev_free(*buf);
    *cap = 0;
    *buf = dev_alloc(bytes);
    if (!*buf) return false;
    *cap = bytes;
    return true;
}

}  // namespace

// Tile size of the FP32 factorization for an FP64 tile size NB: the
// configured factor tile size when it divides NB (a finer tiling shortens the
// chain of diagonal-tile steps, the factorization's critical path), else NB.
int factor_tile(int NB) {
    const int f = ctx().factor_nb;
    return (f > 0 && f < NB && NB % f == 0) ? f : NB;
}

namespace {
int mixed_reserve(MixedWs &m, int N, int NB, int nrhs) {
    const int NBf = factor_tile(NB);
    if (m.N != N || m.NB != NB || m.NBf != NBf) {
        if (m.A32) CHAMELEON_Desc_Destroy(&m.A32);
        if (!grow(&m.a32_buf, &m.a32_cap, (size_t)N * N * sizeof(float))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        if (int rc = desc_create_tiled_on(&m.A32, ChamRealFloat, m.a32_buf, NBf, N, N)) return rc;
        m.N = N;
        m.NB = NB;
        m.NBf = NBf;
        m.nrhs = -1;
    }
    if (m.nrhs != nrhs) {
        if (m.B32) CHAMELEON_Desc_Destroy(&m.B32);
        if (m.R) CHAMELEON_Desc_Destroy(&m.R);
        if (!grow(&m.b32_buf, &m.b32_cap, (size_t)N * nrhs * sizeof(float)) ||
            !grow(&m.r_buf, &m.r_cap, (size_t)N * nrhs * sizeof(double)))
            return CHAMELEON_ERR_OUT_OF_RESOURCES;
        // B32 is tiled like the FP32 factor's tile rows; R like B
        if (int rc = desc_create_tiled_on(&m.B32, ChamRealFloat, m.b32_buf, NBf, N, nrhs)) return rc;
        if (int rc = desc_create_tiled_on(&m.R, ChamRealDouble, m.r_buf, NB, N, nrhs)) return rc;
        m.nrhs = nrhs;
    }
    if (nrhs > m.cap_rhs) {
        dev_free(m.rmax);
        dev_free(m.xmax);
        m.rmax = (unsigned long long *)dev_alloc(nrhs * sizeof(unsigned long long));
        m.xmax = (unsigned long long *)dev_alloc(nrhs * sizeof(unsigned long long));
        if (!m.rmax || !m.xmax) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        m.cap_rhs = nrhs;
    }
    const size_t diag_bytes = (size_t)((N + NB - 1) / NB) * NB * NB * sizeof(double);
    if (!grow((void **)&m.diag, &m.diag_cap, diag_bytes)) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    if (N > m.cap_n) {
        dev_free(m.colsum);
        if (!(m.colsum = (double *)dev_alloc(N * sizeof(double)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        m.cap_n = N;
    }
    if (!m.flag && !(m.flag = (int *)dev_alloc(sizeof(int)))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    if (!m.e0) {
        CHB_CUDA(cudaEventCreate(&m.e0));
        CHB_CUDA(cudaEventCreate(&m.e1));
    }
    return 0;
}

bool g_res_attr = false;
}  // namespace

static SymTiles symtiles(CHAM_desc_t *A, cham_uplo_t uplo, double *diag = nullptr) {
    return SymTiles{(double *)A->mat, priv(A)->dev.off, priv(A)->dev.ld, A->nt, A->n, A->nb, uplo == ChamUpper,
                    diag};
}

// Symmetric copies of the diagonal tiles of A for the residuals of this solve.
static void sym_diag(CHAM_desc_t *A, cham_uplo_t uplo, cudaStream_t s, MixedWs &m) {
    sym_diag_kernel<<<dim3(std::max(1, std::min(64, (A->nb * A->nb + 255) / 256)), A->nt), 256, 0, s>>>(
        symtiles(A, uplo, m.diag));
    CHB_LAUNCHED(1);
}

// ||A||_inf of the symmetric A (its `uplo` triangle); with a32 (same tiling as
// A) the referenced tiles are cast into it in the same pass, overflow flagged
// in *ovf.  Also makes the symmetric diagonal-tile copies for the residuals.
double sym_norm_inf(CHAM_desc_t *A, cham_uplo_t uplo, cudaStream_t s, MixedWs &m, CHAM_desc_t *a32, int *ovf) {
    if (desc_upload(A) || mixed_reserve(m, A->n, A->nb, std::max(1, m.nrhs))) return -1.0;
    if (a32 && (desc_upload(a32) || a32->nb != a32->mb || A->nb % a32->nb != 0 || a32->n != A->n)) return -1.0;
    const int NT = A->nt;
    cudaMemsetAsync(m.colsum, 0, A->n * sizeof(double), s);
    const TileMapD t32 = a32 ? tmap(a32) : TileMapD{nullptr, nullptr, nullptr, 0, 0, 0};
    sym_cast_norm_kernel<<<NT * (NT + 1) / 2, 256, A->nb * sizeof(double), s>>>(symtiles(A, uplo), t32, m.colsum,
                                                                              ovf);
    sym_diag(A, uplo, s, m);
    CHB_LAUNCHED(1);
    std::vector<double> h(A->n);
    cudaMemcpyAsync(h.data(), m.colsum, A->n * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double r = 0;
    for (double v : h) r = std::max(r, v);
    return r;
}

// R = B - A X and the per-column max |R|, max |X| (host copies).
static int residual(CHAM_desc_t *A, cham_uplo_t uplo, CHAM_desc_t *B, CHAM_desc_t *X, cudaStream_t s,
                    std::vector<double> &rn, std::vector<double> &xn, MixedWs &m) {
    if (!uploaded(A) || !uploaded(B) || !uploaded(X) || !uploaded(m.R)) return CHAMELEON_ERR_UNEXPECTED;
    if (!g_res_attr) {
        CHB_CUDA(cudaFuncSetAttribute(sym_residual_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)CfgRes::SMEM_BYTES));
        g_res_attr = true;
    }
    const int nrhs = B->n;
    const int nrb = (A->nb + 127) / 128;
    const int ncb = X->nt * ((X->nb + 63) / 64);
    // split the K sweep so that the working CTAs fill whole waves of SMs
    const int sms = ctx().num_sms * RES_CTAS_PER_SM;
    int nwork = 0;
    for (int mm = 0; mm < A->nt; ++mm) nwork += (desc_tile_rows(A, mm) + 127) / 128;
    nwork *= (nrhs + 63) / 64;
    int ksplit = 1;
    double best = 0;
    for (int k = 1; k <= std::min(8, std::max(1, A->nt / 4)); ++k) {
        const double eff = (double)nwork * k / ((double)((nwork * k + sms - 1) / sms) * sms);
        if (eff > best + 0.02) {
            best = eff;
            ksplit = k;
        }
    }
    if (ksplit > 1) {
        const size_t bytes = (size_t)ksplit * A->n * nrhs * sizeof(double);
        if (bytes > m.part_cap) {
            dev_free(m.part);
            m.part_cap = 0;
            if (!(m.part = (double *)dev_alloc(bytes))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
            m.part_cap = bytes;
        }
    }
    CHB_CUDA(cudaMemsetAsync(m.rmax, 0, nrhs * sizeof(unsigned long long), s));
    CHB_CUDA(cudaMemsetAsync(m.xmax, 0, nrhs * sizeof(unsigned long long), s));
    sym_residual_kernel<<<A->nt * nrb * ncb * ksplit, NT_CTA, CfgRes::SMEM_BYTES, s>>>(
        symtiles(A, uplo, m.diag), tmap(X), tmap(B), tmap(m.R), nrhs, nrb, ncb, ksplit, m.part, m.rmax);
    if (ksplit > 1) {
        residual_reduce_kernel<<<dim3(std::max(1, std::min(32, (A->n + 4095) / 4096)), nrhs), 256, 0, s>>>(
            m.part, ksplit, A->n, tmap(B), tmap(m.R), m.rmax);
        CHB_LAUNCHED(1);
    }
    colmax_kernel<<<dim3(std::max(1, std::min(32, (X->m + 4095) / 4096)), nrhs), 256, 0, s>>>(tmap(X), X->m, nrhs,
                                                                                           m.xmax);
    CHB_LAUNCHED(2);
    CHB_CUDA(cudaGetLastError());
    std::vector<unsigned long long> hr(nrhs), hx(nrhs);
    CHB_CUDA(cudaMemcpyAsync(hr.data(), m.rmax, nrhs * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaMemcpyAsync(hx.data(), m.xmax, nrhs * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaStreamSynchronize(s));
    rn.resize(nrhs);
    xn.resize(nrhs);
    for (int j = 0; j < nrhs; ++j) {
        memcpy(&rn[j], &hr[j], 8);
        memcpy(&xn[j], &hx[j], 8);
    }
    return 0;
}

// dsposv's stopping test on every column, and the normwise backward error
// max_j ||r_j||_inf / (||A||_inf ||x_j||_inf) of the current iterate.
static bool converged(const std::vector<double> &rn, const std::vector<double> &xn, double cte, double anrm,
                      double *berr) {
    bool ok = true;
    double b = 0;
    for (size_t j = 0; j < rn.size(); ++j) {
        if (!(rn[j] <= xn[j] * cte)) ok = false;
        if (xn[j] > 0 && anrm > 0) b = std::max(b, rn[j] / (anrm * xn[j]));
    }
    if (berr) *berr = b;
    return ok;
}

static int cast_desc(CHAM_desc_t *src, CHAM_desc_t *dst, cudaStream_t s, int *overflow_flag) {
    if (desc_upload(src) || desc_upload(dst)) return CHAMELEON_ERR_UNEXPECTED;
    const bool same_layout = !priv(src)->cm_view && !priv(dst)->cm_view && src->mb == dst->mb && src->nb == dst->nb &&
                             src->lm == dst->lm && src->ln == dst->ln;
    if (src->dtyp == ChamRealDouble && dst->dtyp == ChamRealFloat && same_layout) {
        const size_t n = (size_t)src->lm * src->ln;
        cast_d2s_flat<<<ctx().num_sms * 8, 256, 0, s>>>((const double *)src->mat, (float *)dst->mat, n,
                                                      overflow_flag);
    } else if (src->dtyp == ChamRealDouble && dst->dtyp == ChamRealFloat) {
        cast_tiles<double, float><<<ew_grid((int64_t)src->m * src->n), 256, 0, s>>>(tmap(src), tmap(dst), src->m,
                                                                                     src->n, overflow_flag);
    } else if (src->dtyp == ChamRealFloat && dst->dtyp == ChamRealDouble) {
        cast_tiles<float, double><<<ew_grid((int64_t)src->m * src->n), 256, 0, s>>>(tmap(src), tmap(dst), src->m,
                                                                                     src->n, nullptr);
    } else {
        cast_tiles<double, double><<<ew_grid((int64_t)src->m * src->n), 256, 0, s>>>(tmap(src), tmap(dst), src->m,
                                                                                      src->n, nullptr);
    }
    CHB_CUDA(cudaGetLastError());
    CHB_LAUNCHED(1);
    return 0;
}

// Accumulates the device time of host-delimited phases on one stream.
struct PhaseClock {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit PhaseClock(cudaStream_t st) : s(st) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~PhaseClock() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    void tic() { cudaEventRecord(a, s); }
    void toc(float &acc) {
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        acc += ms;
    }
};

// The refinement driver.  A: FP64 (uplo triangle), B: N x nrhs FP64, X: output.
void free_mixed_ws(MixedWs &m) {
    if (m.A32) CHAMELEON_Desc_Destroy(&m.A32);
    if (m.B32) CHAMELEON_Desc_Destroy(&m.B32);
    if (m.R) CHAMELEON_Desc_Destroy(&m.R);
    dev_free(m.a32_buf);
    dev_free(m.b32_buf);
    dev_free(m.r_buf);
    dev_free(m.rmax);
    dev_free(m.xmax);
    dev_free(m.colsum);
    dev_free(m.diag);
    dev_free(m.part);
    dev_free(m.flag);
    if (m.e0) cudaEventDestroy(m.e0);
    if (m.e1) cudaEventDestroy(m.e1);
    m = MixedWs();
}

int mixed_posv_ws(cham_uplo_t uplo, int precision, CHAM_desc_t *A, CHAM_desc_t *B, CHAM_desc_t *X, int *iter_out,
                  CHAM_b200_refine_info_t *info, cudaStream_t s, MixedWs &m, ExecWs *ews, int grid, bool factored,
                  const TriStream *tri) {
    Context &c = ctx();
    const int N = A->n, nrhs = B->n, NB = A->nb;
    int iter = 0;
    CHAM_b200_refine_info_t inf{};
    inf.precision = precision;
    if (int rc0 = mixed_reserve(m, N, NB, nrhs)) return rc0;
    cudaEvent_t e0 = m.e0, e1 = m.e1;
    cudaEventRecord(e0, s);
    int rc = 0;
    ExecResult res;
    bool fallback = (precision == CHAM_B200_PREC_FP64);
    double berr = 0;
    MixedStats st;
    PhaseClock clk(s);
    if (!fallback) {
        if ((rc = desc_upload(A)) || (rc = desc_upload(B)) || (rc = desc_upload(X))) return rc;
        clk.tic();
        CHB_CUDA(cudaMemsetAsync(m.flag, 0, sizeof(int), s));
        if ((rc = cast_desc(B, m.B32, s, m.flag))) return rc;
        const int split = (precision == CHAM_B200_PREC_FP32) ? SPLIT_TF32X3 : SPLIT_BF16X3;
        double anrm = 0;
        int ovf = 0;
        if (!tri) {
            // the norm pass also casts A's referenced tiles to FP32 (unless the
            // FP32 factor is kept from an earlier call)
            anrm = sym_norm_inf(A, uplo, s, m, factored ? nullptr : m.A32, m.flag);
            if (anrm < 0) return CHAMELEON_ERR_UNEXPECTED;
            CHB_CUDA(cudaMemcpyAsync(&ovf, m.flag, sizeof(int), cudaMemcpyDeviceToHost, s));
        } else {
            // A is still arriving: the factorization launch casts its tiles as
            // their columns land and accumulates the norm
            CHB_CUDA(cudaMemsetAsync(m.colsum, 0, (size_t)N * sizeof(double), s));
        }
        clk.toc(st.cast_ms);
        if (ovf) {
            iter = -2;
            fallback = true;
        }
        if (!fallback) {
            CastIn cin{};
            if (tri) {
                if (desc_upload(m.A32)) return CHAMELEON_ERR_UNEXPECTED;
                cin = CastIn{tri->dA, tri->ld, tri->arrive, tri->epoch, m.colsum, m.flag, tri->h2d_gbs};
            }
            rc = run_cholesky_dag(factored ? MODE_SOLVE : (MODE_FACT | MODE_SOLVE), uplo, m.A32, m.B32, s, &res, split,
                                  ews, grid, EXEC_REUSE_INV, tri ? &cin : nullptr);
            if (tri) {
                // every column has landed (each cast waited for its column); order
                // the FP64 readers of A after the copies all the same
                if (cudaStreamWaitEvent(s, tri->done, 0) != cudaSuccess) rc = rc ? rc : CHAMELEON_ERR_UNEXPECTED;
            }
            if (rc) return rc;
            st.factor_ms += res.ms;
            if (res.error) return res.error;
            if (tri) {
                sym_diag(A, uplo, s, m);
                std::vector<double> h(N);
                CHB_CUDA(cudaMemcpyAsync(h.data(), m.colsum, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, s));
                CHB_CUDA(cudaMemcpyAsync(&ovf, m.flag, sizeof(int), cudaMemcpyDeviceToHost, s));
                CHB_CUDA(cudaStreamSynchronize(s));
                for (double v : h) anrm = std::max(anrm, v);
                if (ovf) {
                    iter = -2;
                    fallback = true;
                }
            }
            if (!fallback && res.info) {
                iter = -3;
                fallback = true;
            }
        }
        const double cte = anrm * 1.1102230246251565e-16 * sqrt((double)N);
        if (!fallback) {
            if ((rc = cast_desc(m.B32, X, s, nullptr))) return rc;
            std::vector<double> rn, xn;
            clk.tic();
            if ((rc = residual(A, uplo, B, X, s, rn, xn, m))) return rc;
            clk.toc(st.residual_ms);
            bool ok = converged(rn, xn, cte, anrm, &berr);
            int it = 0;
            while (!ok && it < c.refine_maxiter) {
                ++it;
                clk.tic();
                if ((rc = cast_desc(m.R, m.B32, s, nullptr))) return rc;
                clk.toc(st.cast_ms);
                if ((rc = run_cholesky_dag(MODE_SOLVE, uplo, m.A32, m.B32, s, &res, split, ews, grid, EXEC_REUSE_INV)))
                    return rc;
                st.refine_solve_ms += res.ms;
                if (res.error) return res.error;
                if (!uploaded(X) || !uploaded(m.B32)) return CHAMELEON_ERR_UNEXPECTED;
                clk.tic();
                add_correction<<<ew_grid((int64_t)N * nrhs), 256, 0, s>>>(tmap(X), tmap(m.B32), N, nrhs);
                CHB_LAUNCHED(1);
                CHB_CUDA(cudaGetLastError());
                clk.toc(st.cast_ms);
                clk.tic();
                if ((rc = residual(A, uplo, B, X, s, rn, xn, m))) return rc;
                clk.toc(st.residual_ms);
                ok = converged(rn, xn, cte, anrm, &berr);
            }
            if (ok) {
                iter = it;
            } else {
                iter = -(c.refine_maxiter + 1);
                fallback = true;
            }
        }
    }
    if (fallback) {
        if ((rc = cast_desc(B, X, s, nullptr))) return rc;
        if ((rc = run_cholesky_dag(MODE_FACT | MODE_SOLVE, uplo, A, X, s, &res, 0, ews, grid))) return rc;
        if (res.error) return res.error;
        if (res.info) return res.info;
        inf.fallback = (precision != CHAM_B200_PREC_FP64);
        if (iter == 0 && precision == CHAM_B200_PREC_FP64) iter = 0;
        berr = 0;
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    st.total_ms = ms;
    st.iterations = iter;
    st.fallback = fallback ? 1 : 0;
    if (&m == &g_mws) g_mixed_stats = st;
    inf.iterations = iter;
    inf.backward_error = berr;
    inf.seconds = ms * 1e-3;
    if (iter_out) *iter_out = iter;
    if (info) *info = inf;
    if (fallback) desc_sync_to_host(A);
    return desc_sync_to_host(X);
}

int mixed_posv(cham_uplo_t uplo, int precision, CHAM_desc_t *A, CHAM_desc_t *B, CHAM_desc_t *X, int *iter_out,
               CHAM_b200_refine_info_t *info, const TriStream *tri = nullptr) {
    return mixed_posv_ws(uplo, precision, A, B, X, iter_out, info, ctx().stream, g_mws, nullptr, 0, false, tri);
}

// The referenced triangle of a host matrix is copied to the device one tile
// column (of the FP32 factor's tiling) at a time on a copy stream, each
// column followed by a 4-byte arrival flag from pinned host memory (the copy
// engine executes the two in order), so that the factorization can start on
// the first columns while the others are still on the way.  Column q of the
// lower triangle is rows [q nb, N) of columns [q nb, q nb + w); for the upper
// triangle, rows [q nb, q nb + w) of columns [q nb, N) (the same tiles of the
// symmetric matrix).  Only the triangle moves: half the bytes of the matrix.
int tri_stream_start(TriStreamState &ts, cham_uplo_t uplo, const double *hA, int lda, double *dA, int N, int nb,
                     TriStream *out) {
    const int NT = (N + nb - 1) / nb;
    if (!ts.cs) {
        CHB_CUDA(cudaStreamCreateWithFlags(&ts.cs, cudaStreamNonBlocking));
        CHB_CUDA(cudaEventCreateWithFlags(&ts.done, cudaEventDisableTiming));
        CHB_CUDA(cudaHostAlloc((void **)&ts.h_epoch, sizeof(int), cudaHostAllocDefault));
    }
    if (NT > ts.cap) {
        // the flags keep counting up across calls (epochs), so a fresh array
        // starts from zero once and is never reset
        if (ts.d_arrive) cudaFree(ts.d_arrive);
        ts.d_arrive = nullptr;
        ts.cap = 0;
        const int cap = std::max(NT, 256);
        CHB_CUDA(cudaMalloc(&ts.d_arrive, (size_t)cap * sizeof(int)));
        // zeros from host memory: a copy, not a memset kernel (which could wait
        // for SMs that other streams' persistent launches hold)
        std::vector<int> zeros(cap, 0);
        CHB_CUDA(cudaMemcpy(ts.d_arrive, zeros.data(), (size_t)cap * sizeof(int), cudaMemcpyHostToDevice));
        ts.cap = cap;
        ts.epoch = 0;
    }
    // the previous call's copies read *h_epoch; they are done (synchronous API)
    CHB_CUDA(cudaStreamSynchronize(ts.cs));
    *ts.h_epoch = ++ts.epoch;
    for (int q = 0; q < NT; ++q) {
        const int c0 = q * nb, w = std::min(nb, N - c0);
        const size_t off_d = (size_t)c0 + (size_t)c0 * N, off_h = (size_t)c0 + (size_t)c0 * lda;
        if (uplo == ChamLower)
            CHB_CUDA(cudaMemcpy2DAsync(dA + off_d, (size_t)N * 8, hA + off_h, (size_t)lda * 8, (size_t)(N - c0) * 8, w,
                                       cudaMemcpyHostToDevice, ts.cs));
        else
            CHB_CUDA(cudaMemcpy2DAsync(dA + off_d, (size_t)N * 8, hA + off_h, (size_t)lda * 8, (size_t)w * 8, N - c0,
                                       cudaMemcpyHostToDevice, ts.cs));
        CHB_CUDA(cudaMemcpyAsync(ts.d_arrive + q, ts.h_epoch, sizeof(int), cudaMemcpyHostToDevice, ts.cs));
    }
    CHB_CUDA(cudaEventRecord(ts.done, ts.cs));
    *out = TriStream{dA, (int64_t)N, ts.d_arrive, ts.epoch, ts.done, ctx().h2d_gbs};
    return 0;
}
TriStreamState g_tri;

void free_tri_stream(TriStreamState &ts) {
    if (ts.cs) {
        cudaStreamSynchronize(ts.cs);
        cudaStreamDestroy(ts.cs);
    }
    if (ts.done) cudaEventDestroy(ts.done);
    if (ts.d_arrive) cudaFree(ts.d_arrive);
    if (ts.h_epoch) cudaFreeHost(ts.h_epoch);
    ts = TriStreamState();
}

}  // namespace chb

using namespace chb;

extern "C" {

static int check_mixed_args(CHAM_desc_t *A, CHAM_desc_t *B, CHAM_desc_t *X) {
    if (!A || !B || !X) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (A->dtyp != ChamRealDouble || B->dtyp != ChamRealDouble || X->dtyp != ChamRealDouble)
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (A->m != A->n || A->mb != A->nb || B->m != A->n || X->m != A->n || B->n != X->n || B->mb != A->mb ||
        X->mb != A->mb || X->nb != B->nb)
        return CHAMELEON_ERR_ILLEGAL_VALUE;
    return 0;
}

// Tile-layout dsposv (the reference's commented-out zcposv_Tile prototype,
// include/chameleon/chameleon_zc.h:42, in d/s precision).
int CHAMELEON_dsposv_Tile(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B, CHAM_desc_t *X, int *ITER) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if ((rc = check_mixed_args(A, B, X))) return rc;
    if (A->n == 0 || B->n == 0) return 0;
    const int prec = ctx().precision == CHAM_B200_PREC_FP64 ? CHAM_B200_PREC_BF16X3 : ctx().precision;
    return mixed_posv(uplo, prec, A, B, X, ITER, nullptr);
}

int CHAMELEON_B200_dposv_mixed_Tile(cham_uplo_t uplo, int precision, CHAM_desc_t *A, CHAM_desc_t *B,
                                    CHAM_desc_t *X, CHAM_b200_refine_info_t *info) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (precision < CHAM_B200_PREC_FP64 || precision > CHAM_B200_PREC_BF16X3) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if ((rc = check_mixed_args(A, B, X))) return rc;
    if (A->n == 0 || B->n == 0) return 0;
    return mixed_posv(uplo, precision, A, B, X, nullptr, info);
}

// LAPACK-layout dsposv (chameleon_zc.h:34 prototype, d/s precision): A, B, X
// column-major host or device arrays.
int CHAMELEON_dsposv(cham_uplo_t uplo, int N, int NRHS, double *A, int LDA, double *B, int LDB, double *X, int LDX,
                     int *ITER) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (N < 0) return -2;
    if (NRHS < 0) return -3;
    if (LDA < std::max(1, N)) return -5;
    if (LDB < std::max(1, N)) return -7;
    if (LDX < std::max(1, N)) return -9;
    if (N == 0 || NRHS == 0) {
        if (ITER) *ITER = 0;
        return 0;
    }
    Context &c = ctx();
    cudaStream_t s = c.stream;
    cudaPointerAttributes at;
    auto on_dev = [&](const void *p) {
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
    };
    const bool ad = on_dev(A), bd = on_dev(B), xd = on_dev(X);
    // host arrays are staged densely (ld = N): only the N x cols block moves;
    // a host A streams its referenced triangle in while the factorization
    // runs (tri_stream_start)
    double *dA = A, *dB = B, *dX = X;
    int lda = LDA, ldb = LDB, ldx = LDX;
    TriStream tri{};
    const int prec0 = c.precision == CHAM_B200_PREC_FP64 ? CHAM_B200_PREC_BF16X3 : c.precision;
    const int nbf = factor_tile(c.tile_size);
    const bool stream_a = !ad && prec0 == CHAM_B200_PREC_BF16X3 && c.use_tcgen05 && nbf % 64 == 0 && N > nbf;
    if (!ad) {
        if (stream_a) {
            if (!(dA = staging(0, std::max<size_t>((size_t)N * N * sizeof(double), 16))))
                return CHAMELEON_ERR_OUT_OF_RESOURCES;
            if ((rc = tri_stream_start(g_tri, uplo, A, LDA, dA, N, nbf, &tri))) return rc;
        } else if (!(dA = stage_in(0, A, LDA, N, N, s))) {
            return CHAMELEON_ERR_OUT_OF_RESOURCES;
        }
        lda = N;
    }
    if (!bd) {
        if (!(dB = stage_in(1, B, LDB, N, NRHS, s))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        ldb = N;
    }
    if (!xd) {
        if (!(dX = staging(2, (size_t)N * NRHS * 8))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        ldx = N;
    }
    CHAM_desc_t *Ad, *Bd, *Xd;
    desc_create_cm(&Ad, dA, lda, N, N, c.tile_size);
    desc_create_cm(&Bd, dB, ldb, N, NRHS, c.tile_size);
    desc_create_cm(&Xd, dX, ldx, N, NRHS, c.tile_size);
    int iter = 0;
    rc = mixed_posv(uplo, prec0, Ad, Bd, Xd, &iter, nullptr, stream_a ? &tri : nullptr);
    if (stream_a) cudaStreamSynchronize(g_tri.cs);   // the staging buffer is free again
    if (ITER) *ITER = iter;
    if (!xd) stage_out(X, LDX, dX, N, NRHS, s);
    if (!ad && iter < 0) stage_out(A, LDA, dA, N, N, s);
    cudaStreamSynchronize(s);
    CHAMELEON_Desc_Destroy(&Ad);
    CHAMELEON_Desc_Destroy(&Bd);
    CHAMELEON_Desc_Destroy(&Xd);
    return rc;
}

// Diagnostics: only the first phase of the mixed solve (casts + the FP32
// factor-and-solve DAG launch), returning that launch's device time.
int CHAM_B200_Mixed_Factor_Only(cham_uplo_t uplo, int precision, CHAM_desc_t *A, CHAM_desc_t *B, float *ms) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || !B || precision == CHAM_B200_PREC_FP64) return CHAMELEON_ERR_ILLEGAL_VALUE;
    cudaStream_t s = ctx().stream;
    if ((rc = mixed_reserve(g_mws, A->n, A->nb, B->n))) return rc;
    CHB_CUDA(cudaMemsetAsync(g_mws.flag, 0, sizeof(int), s));
    if ((rc = cast_desc(A, g_mws.A32, s, g_mws.flag)) || (rc = cast_desc(B, g_mws.B32, s, g_mws.flag))) return rc;
    ExecResult res;
    const int split = (precision == CHAM_B200_PREC_FP32) ? SPLIT_TF32X3 : SPLIT_BF16X3;
    rc = run_cholesky_dag(MODE_FACT | MODE_SOLVE, uplo, g_mws.A32, g_mws.B32, s, &res, split);
    if (ms) *ms = res.ms;
    return rc ? rc : (res.error ? res.error : res.info);
}

}  // extern "C"
