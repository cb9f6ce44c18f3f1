// control.cu -- context, descriptors, layout translation, generators, norms and
// the public Cholesky drivers of the B200 library.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "core.cuh"
#include "gen.cuh"
#include "internal.h"

namespace chb {

Context &ctx() {
    static Context c;
    return c;
}

std::atomic<unsigned long long> g_launch_count{0};
MixedStats g_mixed_stats;

void report_cuda_error(const char *what, cudaError_t e, const char *file, int line) {
    fprintf(stderr, "[chameleon_b200] CUDA error %s (%d) in %s at %s:%d\n", cudaGetErrorString(e), (int)e,
            what, file, line);
}

void warning(const char *func, const char *msg) {
    if (ctx().warnings) fprintf(stderr, "CHAMELEON_B200 WARNING: %s(): %s\n", func, msg);
}

int ensure_init() {
    Context &c = ctx();
    if (!c.initialized) {
        fprintf(stderr, "CHAMELEON_B200 ERROR: CHAMELEON not initialized\n");
        return CHAMELEON_ERR_NOT_INITIALIZED;
    }
    // The entry points compute on the library's own non-blocking stream, which
    // the legacy default stream does not order.  A caller that filled its
    // device matrix with work on the default stream (an asynchronous copy, a
    // kernel of its own) must see that work finish before the call reads the
    // matrix, as with a synchronous library: make the stream wait for
    // everything the default stream holds at the time of the call.
    if (c.order_event && (cudaEventRecord(c.order_event, cudaStreamLegacy) != cudaSuccess ||
                          cudaStreamWaitEvent(c.stream, c.order_event, 0) != cudaSuccess)) {
        cudaGetLastError();
        return CHAMELEON_ERR_UNEXPECTED;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Descriptor layout (control/descriptor.c:318-375, control/descriptor_helpers.c
// :450-577): tile-major CCRB with the full tiles first (A11), then the ragged
// last tile row (A21), the ragged last tile column (A12) and the corner (A22).
// ---------------------------------------------------------------------------
DescPriv *priv(const CHAM_desc_t *d) { return (DescPriv *)d->schedopt; }

int desc_tile_rows(const CHAM_desc_t *d, int m) { return (m == d->mt - 1) ? d->m - m * d->mb : d->mb; }
int desc_tile_cols(const CHAM_desc_t *d, int n) { return (n == d->nt - 1) ? d->n - n * d->nb : d->nb; }

int64_t desc_tile_off(const CHAM_desc_t *d, int m, int n) {
    if (priv(d)->cm_view) return (int64_t)m * d->mb + (int64_t)n * d->nb * d->lda;
    const int64_t mm = m, nn = n;
    if (mm < d->llm1) {
        if (nn < d->lln1) return (int64_t)d->bsiz * (mm + (int64_t)d->llm1 * nn);
        return (int64_t)d->A12 + (int64_t)d->mb * (d->ln % d->nb) * mm;
    }
    if (nn < d->lln1) return (int64_t)d->A21 + (int64_t)(d->lm % d->mb) * d->nb * nn;
    return (int64_t)d->A22;
}

int desc_tile_ld(const CHAM_desc_t *d, int m) {
    if (priv(d)->cm_view) return d->lda;
    return ((m + 1) == d->lmt && (d->lm % d->mb) != 0) ? d->lm % d->mb : d->mb;
}

static size_t elt_size(cham_flttype_t t) { return t == ChamRealFloat ? 4 : (t == ChamRealHalf ? 2 : 8); }

static void *host_getaddr(const CHAM_desc_t *d, int m, int n) {
    return (char *)d->mat + desc_tile_off(d, m, n) * elt_size(d->dtyp);
}
static int host_getldd(const CHAM_desc_t *d, int m) { return desc_tile_ld(d, m); }

static void fill_tiles(CHAM_desc_t *d) {
    d->tiles = (CHAM_tile_t *)calloc((size_t)d->mt * d->nt, sizeof(CHAM_tile_t));
    for (int n = 0; n < d->nt; ++n)
        for (int m = 0; m < d->mt; ++m) {
            CHAM_tile_t *t = &d->tiles[m + (size_t)d->mt * n];
            t->mat = host_getaddr(d, m, n);
            t->m = desc_tile_rows(d, m);
            t->n = desc_tile_cols(d, n);
            t->ld = desc_tile_ld(d, m);
            t->format = 1;
            t->flttype = d->dtyp;
        }
}

static void layout_init(CHAM_desc_t *d, cham_flttype_t dtyp, int mb, int nb, int bsiz, int lm, int ln,
                        int m, int n) {
    d->dtyp = dtyp;
    d->styp = ChamCCRB;
    d->mb = mb; d->nb = nb; d->bsiz = bsiz;
    d->lm = lm; d->ln = ln; d->i = 0; d->j = 0; d->m = m; d->n = n;
    d->lmt = (lm + mb - 1) / mb;
    d->lnt = (ln + nb - 1) / nb;
    d->mt = (m + mb - 1) / mb;
    d->nt = (n + nb - 1) / nb;
    d->llm1 = lm / mb;
    d->lln1 = ln / nb;
    const int64_t llm = lm, lln = ln;
    d->A21 = (size_t)(llm - llm % mb) * (size_t)(lln - lln % nb);
    d->A12 = (size_t)(llm % mb) * (size_t)(lln - lln % nb) + d->A21;
    d->A22 = (size_t)(llm - llm % mb) * (size_t)(lln % nb) + d->A12;
    d->get_blkaddr = host_getaddr;
    d->get_blkldd = host_getldd;
}

cudaStream_t meta_stream() {
    static std::once_flag once;
    static cudaStream_t ms = nullptr;
    std::call_once(once, [] { cudaStreamCreateWithFlags(&ms, cudaStreamNonBlocking); });
    return ms;
}

// Stream-ordered workspace memory: allocation and release go through the
// meta stream, so neither waits for kernels running on other streams (a plain
// cudaFree synchronizes the whole device).  dev_alloc returns memory usable on
// any stream (contents undefined); dev_free requires that no queued work still
// uses the memory.
// The library's own memory pool: freed blocks stay mapped for reuse (release
// threshold = max), so workspace churn never returns memory to the driver and
// re-maps it -- which can stall every stream of the device.  The pool is an
// object of this process; no device setting changes.
static cudaMemPool_t lib_pool() {
    static std::once_flag once;
    static cudaMemPool_t pool = nullptr;
    std::call_once(once, [] {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx().device;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            pool = nullptr;
            return;
        }
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    });
    return pool;
}

void *dev_alloc(size_t bytes) {
    void *p = nullptr;
    cudaStream_t ms = meta_stream();
    cudaMemPool_t pool = lib_pool();
    const cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 16), pool, ms)
                               : cudaMallocAsync(&p, std::max<size_t>(bytes, 16), ms);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    // no fill: a memset is a kernel, and on a device whose SMs are all held by
    // other streams' persistent launches it would wait for them (callers
    // write or clear their buffers on their own streams before reading them)
    if (cudaStreamSynchronize(ms) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(p, ms);
        return nullptr;
    }
    return p;
}

void dev_free(void *p) {
    if (p) cudaFreeAsync(p, meta_stream());
}

// Maps `bytes` of device memory into the library pool ahead of use (one
// allocation, freed at once: the pool keeps the memory), so that later
// workspace growth is served from mapped memory.  Growing the pool maps new
// physical memory, which took hundreds of milliseconds while persistent
// launches occupied the device.
int pool_reserve(size_t bytes) {
    cudaMemPool_t pool = lib_pool();
    if (!pool || bytes == 0) return 0;
    size_t have = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &have);
    if (have >= bytes) return 0;
    void *p = nullptr;
    cudaStream_t ms = meta_stream();
    if (cudaMallocFromPoolAsync(&p, bytes - have, pool, ms) != cudaSuccess) {
        cudaGetLastError();
        return CHAMELEON_ERR_OUT_OF_RESOURCES;
    }
    cudaFreeAsync(p, ms);
    return cudaStreamSynchronize(ms) == cudaSuccess ? 0 : CHAMELEON_ERR_UNEXPECTED;
}

int desc_create_tiled_on(CHAM_desc_t **desc, cham_flttype_t dtyp, void *storage, int nb, int m, int n) {
    CHAM_desc_t *d = (CHAM_desc_t *)calloc(1, sizeof(CHAM_desc_t));
    layout_init(d, dtyp, nb, nb, nb * nb, m, n, m, n);
    d->mat = storage;
    d->alloc_mat = 0;
    d->schedopt = new DescPriv();
    d->id = ctx().desc_ids++;
    fill_tiles(d);
    *desc = d;
    return desc_upload(d);
}

static int desc_upload_tables(CHAM_desc_t *d, const int64_t *off, const int *ld);

// A descriptor over tiles addressed by caller tables: tile (m, n) at
// base + off[m + mt n], leading dimension ld[m] (a runtime plugin's view of
// another library's descriptor); uploaded, storage not owned.
int desc_create_from_tables(CHAM_desc_t **desc, double *base, int mb, int m, int n, const int64_t *off,
                            const int *ld, int nb) {
    if (nb <= 0) nb = mb;
    CHAM_desc_t *d = (CHAM_desc_t *)calloc(1, sizeof(CHAM_desc_t));
    layout_init(d, ChamRealDouble, mb, nb, mb * nb, m, n, m, n);
    d->mat = base;
    d->alloc_mat = 0;
    d->schedopt = new DescPriv();
    d->id = ctx().desc_ids++;
    fill_tiles(d);
    *desc = d;
    return desc_upload_tables(d, off, ld);
}

int desc_upload(CHAM_desc_t *d) {
    DescPriv *pv = priv(d);
    if (pv->dev.off) return 0;
    const size_t nt = (size_t)d->mt * d->nt;
    std::vector<int64_t> off(nt);
    std::vector<int> ld(d->mt);
    for (int n = 0; n < d->nt; ++n)
        for (int m = 0; m < d->mt; ++m) off[m + (size_t)d->mt * n] = desc_tile_off(d, m, n);
    for (int m = 0; m < d->mt; ++m) ld[m] = desc_tile_ld(d, m);
    return desc_upload_tables(d, off.data(), ld.data());
}

static int desc_upload_tables(CHAM_desc_t *d, const int64_t *off_h, const int *ld_h) {
    DescPriv *pv = priv(d);
    const size_t nt = (size_t)d->mt * d->nt;
    // Stream-ordered allocation on a private stream: creating and destroying
    // descriptors does not synchronize the device (cudaFree would), so
    // concurrent solvers on other streams keep running.
    cudaStream_t ms = meta_stream();
    cudaMemPool_t pool = lib_pool();
    if (pool) {
        CHB_CUDA(cudaMallocFromPoolAsync((void **)&pv->dev.off, nt * sizeof(int64_t), pool, ms));
        CHB_CUDA(cudaMallocFromPoolAsync((void **)&pv->dev.ld, d->mt * sizeof(int), pool, ms));
    } else {
        CHB_CUDA(cudaMallocAsync(&pv->dev.off, nt * sizeof(int64_t), ms));
        CHB_CUDA(cudaMallocAsync(&pv->dev.ld, d->mt * sizeof(int), ms));
    }
    CHB_CUDA(cudaMemcpyAsync(pv->dev.off, off_h, nt * sizeof(int64_t), cudaMemcpyHostToDevice, ms));
    CHB_CUDA(cudaMemcpyAsync(pv->dev.ld, ld_h, d->mt * sizeof(int), cudaMemcpyHostToDevice, ms));
    CHB_CUDA(cudaStreamSynchronize(ms));
    return 0;
}

static bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int desc_create_cm(CHAM_desc_t **desc, double *dA, int lda, int m, int n, int nb) {
    CHAM_desc_t *d = (CHAM_desc_t *)calloc(1, sizeof(CHAM_desc_t));
    layout_init(d, ChamRealDouble, nb, nb, nb * nb, m, n, m, n);
    d->styp = ChamCM;
    d->lda = lda;
    d->mat = dA;
    d->alloc_mat = 0;
    d->schedopt = new DescPriv();
    priv(d)->cm_view = 1;
    d->id = ctx().desc_ids++;
    fill_tiles(d);
    *desc = d;
    return 0;
}

int desc_sync_to_host(CHAM_desc_t *d) {
    if (!d->host_mat) return 0;
    const size_t bytes = (size_t)d->lm * d->ln * elt_size(d->dtyp);
    CHB_CUDA(cudaMemcpy(d->host_mat, d->mat, bytes, cudaMemcpyDeviceToHost));
    return 0;
}

static int desc_sync_from_host(CHAM_desc_t *d) {
    if (!d->host_mat) return 0;
    const size_t bytes = (size_t)d->lm * d->ln * elt_size(d->dtyp);
    CHB_CUDA(cudaMemcpy(d->mat, d->host_mat, bytes, cudaMemcpyHostToDevice));
    return 0;
}

// ---------------------------------------------------------------------------
// Kernels: layout translation, generators, norms
// ---------------------------------------------------------------------------
struct TileMap {
    double *base;
    const int64_t *off;
    const int *ld;
    int mt, mb, nb;
    __device__ double *at(int i, int j) const {
        const int m = i / mb, n = j / nb;
        return base + off[m + (int64_t)mt * n] + (i - m * mb) + (int64_t)(j - n * nb) * ld[m];
    }
};

__device__ __forceinline__ bool in_uplo(int uplo, int i, int j) {
    return uplo == ChamUpperLower || (uplo == ChamUpper && i <= j) || (uplo == ChamLower && i >= j);
}

__global__ void lap2tile_kernel(TileMap t, const double *A, int64_t lda, int M, int N, int uplo, int to_tile) {
    const int64_t total = (int64_t)M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        if (!in_uplo(uplo, i, j)) continue;
        double *tp = t.at(i, j);
        double *ap = const_cast<double *>(A) + i + j * lda;
        if (to_tile) *tp = *ap;
        else *ap = *tp;
    }
}

// dplgsy: element (i,j) of the global matrix, i >= j, is the value of state
// i + j*bigM of the stream seeded by `seed`; the upper triangle mirrors it and
// the diagonal adds `bump` (coreblas/compute/core_zplgsy.c:38-112; real
// precision uses one state per element).  Tiles entirely in the triangle
// opposite to `uplo` are skipped as chameleon_pzplgsy does
// (compute/pzplgsy.c:57-66).
__global__ void plgsy_kernel(TileMap t, int M, int N, double bump, int bigM, int m0, int n0,
                             unsigned long long seed, int uplo) {
    const int64_t total = (int64_t)M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        const int tm = i / t.mb, tn = j / t.nb;
        const int tile_m0 = tm * t.mb, tile_n0 = tn * t.nb;
        const int tmm = min(t.mb, M - tile_m0), tnn = min(t.nb, N - tile_n0);
        if (uplo == ChamLower && tile_n0 + n0 >= tile_m0 + m0 + tmm) continue;
        if (uplo == ChamUpper && tile_m0 + m0 >= tile_n0 + n0 + tnn) continue;
        const long long gi = (long long)i + m0, gj = (long long)j + n0;
        unsigned long long pos;
        if (gi >= gj) pos = (unsigned long long)gi + (unsigned long long)gj * (unsigned long long)bigM;
        else pos = (unsigned long long)gj + (unsigned long long)gi * (unsigned long long)bigM;
        double v = lcg_value(lcg_skip(pos, seed));
        if (gi == gj) v = __dadd_rn(v, bump);
        *t.at(i, j) = v;
    }
}

// dplrnt: element (i,j) = value of state i + j*bigM (coreblas/compute/core_zplrnt.c).
__global__ void plrnt_kernel(TileMap t, int M, int N, int bigM, int m0, int n0, unsigned long long seed) {
    const int64_t total = (int64_t)M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        const unsigned long long pos =
            (unsigned long long)(i + m0) + (unsigned long long)(j + n0) * (unsigned long long)bigM;
        *t.at(i, j) = lcg_value(lcg_skip(pos, seed));
    }
}

// Column sums of |A| for a symmetric matrix stored in one triangle (one and
// infinity norms are equal), or max |a_ij|; general matrices use sym = 0.
__global__ void abs_colsum_kernel(TileMap t, int M, int N, int uplo, int sym, double *colsum,
                                  double *rowsum, unsigned long long *maxbits) {
    const int64_t total = (int64_t)M * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % M), j = (int)(idx / M);
        if (sym && !in_uplo(uplo, i, j)) continue;
        const double v = fabs(*t.at(i, j));
        atomicAdd(&colsum[j], v);
        if (rowsum) atomicAdd(&rowsum[i], v);
        if (sym && i != j) atomicAdd(&colsum[i], v);
        atomicMax(maxbits, (unsigned long long)__double_as_longlong(v));
    }
}

static int grid_for(int64_t total) {
    const int64_t blocks = (total + 255) / 256;
    return (int)std::min<int64_t>(std::max<int64_t>(blocks, 1), (int64_t)ctx().num_sms * 32);
}

static TileMap tilemap(CHAM_desc_t *d) {
    return TileMap{(double *)d->mat, priv(d)->dev.off, priv(d)->dev.ld, d->mt, d->mb, d->nb};
}

}  // namespace chb

using namespace chb;

// ---------------------------------------------------------------------------
// Public C API
// ---------------------------------------------------------------------------
extern "C" {

int __chameleon_init(int nworkers, int ncudas) {
    (void)nworkers;
    Context &c = ctx();
    if (c.initialized) {
        warning("CHAMELEON_Init", "CHAMELEON already initialized");
        return CHAMELEON_ERR_REINITIALIZED;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        fprintf(stderr, "CHAMELEON_B200 ERROR: no CUDA device available\n");
        return CHAMELEON_ERR_NOT_INITIALIZED;
    }
    (void)ncudas;
    CHB_CUDA(cudaGetDevice(&c.device));
    CHB_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device));
    CHB_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    CHB_CUDA(cudaEventCreateWithFlags(&c.order_event, cudaEventDisableTiming));
    if (const char *s = getenv("CHAMELEON_TILE_SIZE")) c.tile_size = std::max(1, atoi(s));
    if (const char *s = getenv("CHAMELEON_B200_PRECISION")) {
        if (!strcmp(s, "fp64")) c.precision = CHAM_B200_PREC_FP64;
        else if (!strcmp(s, "fp32")) c.precision = CHAM_B200_PREC_FP32;
        else if (!strcmp(s, "bf16x3")) c.precision = CHAM_B200_PREC_BF16X3;
    }
    if (const char *s = getenv("CHAMELEON_B200_REFINE_MAXITER")) c.refine_maxiter = std::max(1, atoi(s));
    c.initialized = true;
    return CHAMELEON_SUCCESS;
}

int __chameleon_finalize(void) {
    Context &c = ctx();
    if (!c.initialized) return CHAMELEON_ERR_NOT_INITIALIZED;
    cudaStreamSynchronize(c.stream);
    c.initialized = false;
    return CHAMELEON_SUCCESS;
}

int CHAMELEON_Initialized(void) { return ctx().initialized ? 1 : 0; }

int CHAM_B200_Init(void) {
    if (ctx().initialized) return 0;
    return __chameleon_init(0, 1);
}

int CHAMELEON_Set(int param, int value) {
    Context &c = ctx();
    if (!c.initialized) return CHAMELEON_ERR_NOT_INITIALIZED;
    switch (param) {
    case CHAMELEON_TILE_SIZE:
        if (value <= 0) return CHAMELEON_ERR_ILLEGAL_VALUE;
        c.tile_size = value;
        return 0;
    case CHAMELEON_INNER_BLOCK_SIZE:
        if (value <= 0) return CHAMELEON_ERR_ILLEGAL_VALUE;
        c.inner_block = value;
        return 0;
    case CHAMELEON_B200_PRECISION:
        if (value < CHAM_B200_PREC_FP64 || value > CHAM_B200_PREC_BF16X3) return CHAMELEON_ERR_ILLEGAL_VALUE;
        c.precision = value;
        return 0;
    case CHAMELEON_B200_REFINE_MAXITER:
        if (value <= 0) return CHAMELEON_ERR_ILLEGAL_VALUE;
        c.refine_maxiter = value;
        return 0;
    case CHAMELEON_B200_WAIT_BUDGET_MS:
        if (value <= 0) return CHAMELEON_ERR_ILLEGAL_VALUE;
        c.wait_budget_us = (long long)value * 1000;
        return 0;
    case CHAMELEON_B200_WAIT_BUDGET_US:
        if (value <= 0) return CHAMELEON_ERR_ILLEGAL_VALUE;
        c.wait_budget_us = value;
        return 0;
    case CHAMELEON_B200_TCGEN05:
        c.use_tcgen05 = (value != 0);
        return 0;
    case CHAMELEON_B200_REC_TILE:
        c.rec_tile = (value != 0);
        return 0;
    case CHAMELEON_B200_XINV_SOLVE:
        c.xinv_solve = (value != 0);
        return 0;
    case CHAMELEON_B200_POTRF_CTA:
        c.potrf_cta = (value != 0);
        return 0;
    case CHAMELEON_B200_UPD_GROUP_F64:
    case CHAMELEON_B200_UPD_GROUP_F32:
    case CHAMELEON_B200_UPD_GROUP_TC:
        if (value < 1 || value > 64) return CHAMELEON_ERR_ILLEGAL_VALUE;
        (param == CHAMELEON_B200_UPD_GROUP_F64 ? c.kgroup_f64
                                               : param == CHAMELEON_B200_UPD_GROUP_F32 ? c.kgroup_f32 : c.kgroup_tc) =
            value;
        return 0;
    case CHAMELEON_B200_UPD_TAIL_F64:
        if (value < 0 || value > 8) return CHAMELEON_ERR_ILLEGAL_VALUE;
        c.utail_f64 = value;
        return 0;
    case CHAMELEON_B200_FACTOR_NB:
        if (value < 0 || (value > 0 && value % 64 != 0)) return CHAMELEON_ERR_ILLEGAL_VALUE;
        c.factor_nb = value;
        return 0;
    case CHAMELEON_TRANSLATION_MODE:
    case CHAMELEON_LOOKAHEAD:
    case CHAMELEON_CONCURRENCY:
        return 0;
    }
    return CHAMELEON_ERR_ILLEGAL_VALUE;
}

int CHAMELEON_Get(int param, int *value) {
    Context &c = ctx();
    if (!c.initialized) return CHAMELEON_ERR_NOT_INITIALIZED;
    switch (param) {
    case CHAMELEON_TILE_SIZE: *value = c.tile_size; return 0;
    case CHAMELEON_INNER_BLOCK_SIZE: *value = c.inner_block; return 0;
    case CHAMELEON_B200_PRECISION: *value = c.precision; return 0;
    case CHAMELEON_B200_REFINE_MAXITER: *value = c.refine_maxiter; return 0;
    case CHAMELEON_B200_WAIT_BUDGET_MS: *value = (int)(c.wait_budget_us / 1000); return 0;
    case CHAMELEON_B200_WAIT_BUDGET_US: *value = (int)std::min<long long>(c.wait_budget_us, INT_MAX); return 0;
    case CHAMELEON_B200_TCGEN05: *value = c.use_tcgen05 ? 1 : 0; return 0;
    case CHAMELEON_B200_REC_TILE: *value = c.rec_tile ? 1 : 0; return 0;
    case CHAMELEON_B200_XINV_SOLVE: *value = c.xinv_solve ? 1 : 0; return 0;
    case CHAMELEON_B200_POTRF_CTA: *value = c.potrf_cta ? 1 : 0; return 0;
    case CHAMELEON_B200_UPD_GROUP_F64: *value = c.kgroup_f64; return 0;
    case CHAMELEON_B200_UPD_GROUP_F32: *value = c.kgroup_f32; return 0;
    case CHAMELEON_B200_UPD_GROUP_TC: *value = c.kgroup_tc; return 0;
    case CHAMELEON_B200_FACTOR_NB: *value = c.factor_nb; return 0;
    case CHAMELEON_B200_UPD_TAIL_F64: *value = c.utail_f64; return 0;
    }
    return CHAMELEON_ERR_ILLEGAL_VALUE;
}

int CHAMELEON_Enable(int option) {
    if (option == CHAMELEON_WARNINGS || option == CHAMELEON_ERRORS) { ctx().warnings = 1; return 0; }
    if (option == CHAMELEON_AUTOTUNING) return 0;
    return CHAMELEON_ERR_ILLEGAL_VALUE;
}
int CHAMELEON_Disable(int option) {
    if (option == CHAMELEON_WARNINGS || option == CHAMELEON_ERRORS) { ctx().warnings = 0; return 0; }
    if (option == CHAMELEON_AUTOTUNING) return 0;
    return CHAMELEON_ERR_ILLEGAL_VALUE;
}

const char *CHAMELEON_B200_Strerror(int code) {
    switch (code) {
    case CHAMELEON_SUCCESS: return "success";
    case CHAMELEON_ERR_NOT_INITIALIZED: return "not initialized";
    case CHAMELEON_ERR_REINITIALIZED: return "reinitialized";
    case CHAMELEON_ERR_NOT_SUPPORTED: return "not supported";
    case CHAMELEON_ERR_ILLEGAL_VALUE: return "illegal value";
    case CHAMELEON_ERR_NOT_FOUND: return "not found";
    case CHAMELEON_ERR_OUT_OF_RESOURCES: return "out of resources";
    case CHAMELEON_ERR_INTERNAL_LIMIT: return "internal limit";
    case CHAMELEON_ERR_UNALLOCATED: return "unallocated";
    case CHAMELEON_ERR_FILESYSTEM: return "filesystem";
    case CHAMELEON_ERR_UNEXPECTED: return "unexpected";
    case CHAMELEON_ERR_SEQUENCE_FLUSHED: return "sequence flushed";
    case CHAMELEON_ERR_DEVICE_TIMEOUT: return "device dependency wait timed out";
    }
    return code > 0 ? "matrix not positive definite" : "unknown";
}

int CHAMELEON_Desc_Create(CHAM_desc_t **descptr, void *mat, cham_flttype_t dtyp, int mb, int nb, int bsiz,
                          int lm, int ln, int i, int j, int m, int n, int p, int q) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!descptr) return CHAMELEON_ERR_ILLEGAL_VALUE;
    *descptr = nullptr;
    if (dtyp != ChamRealDouble && dtyp != ChamRealFloat) return CHAMELEON_ERR_NOT_SUPPORTED;
    if (mb <= 0 || nb <= 0 || lm < 0 || ln < 0 || m < 0 || n < 0 || bsiz < mb * nb) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (i != 0 || j != 0 || m > lm || n > ln) return CHAMELEON_ERR_NOT_SUPPORTED;   // submatrices: not on this path
    if (p != 1 || q != 1) return CHAMELEON_ERR_NOT_SUPPORTED;                       // single-GPU process grid
    CHAM_desc_t *d = (CHAM_desc_t *)calloc(1, sizeof(CHAM_desc_t));
    layout_init(d, dtyp, mb, nb, bsiz, lm, ln, m, n);
    d->schedopt = new DescPriv();
    d->id = ctx().desc_ids++;
    const size_t bytes = std::max<size_t>((size_t)lm * ln * elt_size(dtyp), 16);
    // As in the reference (control/descriptor.c:183-199), a caller-provided
    // matrix is a column-major lm x ln array (ChamCM, ld = lm); only
    // library-allocated storage uses the tile-major CCRB layout.
    const bool user_mat = !(mat == CHAMELEON_MAT_ALLOC_TILE || mat == CHAMELEON_MAT_ALLOC_GLOBAL);
    if (user_mat) {
        d->styp = ChamCM;
        d->lda = std::max(lm, 1);
        priv(d)->cm_view = 1;
    }
    if (!user_mat) {
        if (cudaMalloc(&d->mat, bytes) != cudaSuccess) {
            cudaGetLastError();
            delete priv(d);
            free(d);
            return CHAMELEON_ERR_OUT_OF_RESOURCES;
        }
        cudaMemset(d->mat, 0, bytes);
        d->alloc_mat = 1;
    } else if (is_device_ptr(mat)) {
        d->mat = mat;
    } else {
        if (cudaMalloc(&d->mat, bytes) != cudaSuccess) {
            cudaGetLastError();
            delete priv(d);
            free(d);
            return CHAMELEON_ERR_OUT_OF_RESOURCES;
        }
        d->alloc_mat = 1;
        d->host_mat = mat;
        desc_sync_from_host(d);
    }
    fill_tiles(d);
    *descptr = d;
    return CHAMELEON_SUCCESS;
}

int CHAMELEON_Desc_Destroy(CHAM_desc_t **descptr) {
    if (!descptr || !*descptr) return CHAMELEON_ERR_UNALLOCATED;
    CHAM_desc_t *d = *descptr;
    if (d->alloc_mat && d->mat) cudaFree(d->mat);
    DescPriv *pv = priv(d);
    if (pv) {
        // the caller has synchronized the work that used the tables
        if (pv->dev.off) cudaFreeAsync(pv->dev.off, meta_stream());
        if (pv->dev.ld) cudaFreeAsync(pv->dev.ld, meta_stream());
        delete pv;
    }
    free(d->tiles);
    free(d);
    *descptr = nullptr;
    return CHAMELEON_SUCCESS;
}

int CHAMELEON_Desc_Flush(const CHAM_desc_t *desc, const RUNTIME_sequence_t *sequence) {
    (void)sequence;
    if (!desc) return CHAMELEON_ERR_UNALLOCATED;
    cudaStreamSynchronize(ctx().stream);
    return desc_sync_to_host(const_cast<CHAM_desc_t *>(desc));
}
int CHAMELEON_Desc_Acquire(const CHAM_desc_t *desc) { return CHAMELEON_Desc_Flush(desc, nullptr); }
int CHAMELEON_Desc_Release(const CHAM_desc_t *desc) {
    if (!desc) return CHAMELEON_ERR_UNALLOCATED;
    return desc_sync_from_host(const_cast<CHAM_desc_t *>(desc));
}

static int lap_desc_copy(cham_uplo_t uplo, void *A, int LDA, CHAM_desc_t *d, int to_tile) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!d || !A) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (d->dtyp != ChamRealDouble) return CHAMELEON_ERR_NOT_SUPPORTED;
    if (LDA < std::max(1, d->m)) return CHAMELEON_ERR_ILLEGAL_VALUE;
    rc = desc_upload(d);
    if (rc) return rc;
    cudaStream_t s = ctx().stream;
    double *dA = (double *)A;
    double *tmp = nullptr;
    const size_t bytes = (size_t)LDA * d->n * sizeof(double);
    if (!is_device_ptr(A)) {
        CHB_CUDA(cudaMalloc(&tmp, std::max<size_t>(bytes, 16)));
        if (to_tile) CHB_CUDA(cudaMemcpyAsync(tmp, A, bytes, cudaMemcpyHostToDevice, s));
        else CHB_CUDA(cudaMemcpyAsync(tmp, A, bytes, cudaMemcpyHostToDevice, s));   // keep untouched triangle
        dA = tmp;
    }
    const int64_t total = (int64_t)d->m * d->n;
    if (total > 0)
        lap2tile_kernel<<<grid_for(total), 256, 0, s>>>(tilemap(d), dA, LDA, d->m, d->n, (int)uplo, to_tile),
            CHB_LAUNCHED(1);
    CHB_CUDA(cudaGetLastError());
    if (tmp) {
        if (!to_tile) CHB_CUDA(cudaMemcpyAsync(A, tmp, bytes, cudaMemcpyDeviceToHost, s));
        CHB_CUDA(cudaStreamSynchronize(s));
        cudaFree(tmp);
    } else {
        CHB_CUDA(cudaStreamSynchronize(s));
    }
    if (to_tile) return desc_sync_to_host(d);
    return 0;
}

int CHAMELEON_Lap2Desc(cham_uplo_t uplo, void *A, int LDA, CHAM_desc_t *descA) {
    return lap_desc_copy(uplo, A, LDA, descA, 1);
}
int CHAMELEON_Desc2Lap(cham_uplo_t uplo, CHAM_desc_t *descA, void *A, int LDA) {
    return lap_desc_copy(uplo, A, LDA, descA, 0);
}

int CHAMELEON_Sequence_Create(RUNTIME_sequence_t **sequence) {
    *sequence = (RUNTIME_sequence_t *)calloc(1, sizeof(RUNTIME_sequence_t));
    return *sequence ? 0 : CHAMELEON_ERR_OUT_OF_RESOURCES;
}
int CHAMELEON_Sequence_Destroy(RUNTIME_sequence_t *sequence) {
    free(sequence);
    return 0;
}
int CHAMELEON_Sequence_Wait(RUNTIME_sequence_t *sequence) {
    cudaStreamSynchronize(ctx().stream);
    return sequence ? sequence->status : CHAMELEON_ERR_UNALLOCATED;
}

// ---- generators -------------------------------------------------------------
int CHAMELEON_dplgsy_Tile(double bump, cham_uplo_t uplo, CHAM_desc_t *A, unsigned long long int seed) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || A->dtyp != ChamRealDouble) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (A->mb != A->nb) return CHAMELEON_ERR_ILLEGAL_VALUE;
    rc = desc_upload(A);
    if (rc) return rc;
    const int64_t total = (int64_t)A->m * A->n;
    if (total > 0)
        plgsy_kernel<<<grid_for(total), 256, 0, ctx().stream>>>(tilemap(A), A->m, A->n, bump, A->m, 0, 0, seed,
                                                                (int)uplo),
            CHB_LAUNCHED(1);
    CHB_CUDA(cudaGetLastError());
    CHB_CUDA(cudaStreamSynchronize(ctx().stream));
    return desc_sync_to_host(A);
}

int CHAMELEON_dplrnt_Tile(CHAM_desc_t *A, unsigned long long int seed) {
    int rc = ensure_init();
    if (rc) return rc;
    if (!A || A->dtyp != ChamRealDouble) return CHAMELEON_ERR_ILLEGAL_VALUE;
    rc = desc_upload(A);
    if (rc) return rc;
    const int64_t total = (int64_t)A->m * A->n;
    if (total > 0)
        plrnt_kernel<<<grid_for(total), 256, 0, ctx().stream>>>(tilemap(A), A->m, A->n, A->m, 0, 0, seed),
            CHB_LAUNCHED(1);
    CHB_CUDA(cudaGetLastError());
    CHB_CUDA(cudaStreamSynchronize(ctx().stream));
    return desc_sync_to_host(A);
}

// LAPACK-layout generators (compute/zplgsy.c, compute/zplrnt.c): A may be a
// host or a device array.
int CHAMELEON_dplgsy(double bump, cham_uplo_t uplo, int N, double *A, int LDA, unsigned long long int seed) {
    int rc = ensure_init();
    if (rc) return rc;
    if (N < 0) return -3;
    if (LDA < std::max(1, N)) return -5;
    if (N == 0) return 0;
    CHAM_desc_t *d = nullptr;
    rc = CHAMELEON_Desc_Create(&d, CHAMELEON_MAT_ALLOC_TILE, ChamRealDouble, ctx().tile_size, ctx().tile_size,
                               ctx().tile_size * ctx().tile_size, N, N, 0, 0, N, N, 1, 1);
    if (rc) return rc;
    rc = CHAMELEON_dplgsy_Tile(bump, uplo, d, seed);
    if (!rc) rc = CHAMELEON_Desc2Lap(uplo, d, A, LDA);
    CHAMELEON_Desc_Destroy(&d);
    return rc;
}

int CHAMELEON_dplrnt(int M, int N, double *A, int LDA, unsigned long long int seed) {
    int rc = ensure_init();
    if (rc) return rc;
    if (M < 0) return -1;
    if (N < 0) return -2;
    if (LDA < std::max(1, M)) return -4;
    if (M == 0 || N == 0) return 0;
    CHAM_desc_t *d = nullptr;
    rc = CHAMELEON_Desc_Create(&d, CHAMELEON_MAT_ALLOC_TILE, ChamRealDouble, ctx().tile_size, ctx().tile_size,
                               ctx().tile_size * ctx().tile_size, M, N, 0, 0, M, N, 1, 1);
    if (rc) return rc;
    rc = CHAMELEON_dplrnt_Tile(d, seed);
    if (!rc) rc = CHAMELEON_Desc2Lap(ChamUpperLower, d, A, LDA);
    CHAMELEON_Desc_Destroy(&d);
    return rc;
}

// ---- norms -----------------------------------------------------------------
static double norm_impl(cham_normtype_t norm, cham_uplo_t uplo, CHAM_desc_t *A, int sym) {
    if (ensure_init() || !A || desc_upload(A)) return -1.0;
    const int M = A->m, N = A->n;
    if (M == 0 || N == 0) return 0.0;
    double *col = nullptr, *row = nullptr;
    unsigned long long *mx = nullptr;
    cudaStream_t s = ctx().stream;
    if (cudaMalloc(&col, sizeof(double) * (size_t)std::max(M, N)) != cudaSuccess) return -1.0;
    if (cudaMalloc(&row, sizeof(double) * (size_t)std::max(M, N)) != cudaSuccess) { cudaFree(col); return -1.0; }
    if (cudaMalloc(&mx, sizeof(unsigned long long)) != cudaSuccess) { cudaFree(col); cudaFree(row); return -1.0; }
    cudaMemsetAsync(col, 0, sizeof(double) * std::max(M, N), s);
    cudaMemsetAsync(row, 0, sizeof(double) * std::max(M, N), s);
    cudaMemsetAsync(mx, 0, sizeof(unsigned long long), s);
    abs_colsum_kernel<<<grid_for((int64_t)M * N), 256, 0, s>>>(tilemap(A), M, N, (int)uplo, sym, col,
                                                               sym ? nullptr : row, mx);
    std::vector<double> hc(std::max(M, N)), hr(std::max(M, N));
    unsigned long long hm = 0;
    cudaMemcpyAsync(hc.data(), col, sizeof(double) * N, cudaMemcpyDeviceToHost, s);
    if (!sym) cudaMemcpyAsync(hr.data(), row, sizeof(double) * M, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&hm, mx, sizeof(hm), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    cudaFree(col); cudaFree(row); cudaFree(mx);
    double r = 0;
    switch (norm) {
    case ChamOneNorm:
        for (int j = 0; j < N; ++j) r = std::max(r, hc[j]);
        break;
    case ChamInfNorm:
        if (sym) for (int j = 0; j < N; ++j) r = std::max(r, hc[j]);
        else for (int i = 0; i < M; ++i) r = std::max(r, hr[i]);
        break;
    case ChamMaxNorm: {
        double v;
        memcpy(&v, &hm, sizeof v);
        r = v;
        break;
    }
    default:
        return -1.0;
    }
    return r;
}

double CHAMELEON_dlansy_Tile(cham_normtype_t norm, cham_uplo_t uplo, CHAM_desc_t *A) {
    return norm_impl(norm, uplo, A, 1);
}
double CHAMELEON_dlange_Tile(cham_normtype_t norm, CHAM_desc_t *A) {
    return norm_impl(norm, ChamUpperLower, A, 0);
}

// ---- Cholesky drivers --------------------------------------------------------
static int check_square_desc(const CHAM_desc_t *A, const char *fn) {
    if (!A) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (A->dtyp != ChamRealDouble) { warning(fn, "only real double descriptors"); return CHAMELEON_ERR_ILLEGAL_VALUE; }
    if (A->nb != A->mb) { warning(fn, "only square tiles supported"); return CHAMELEON_ERR_ILLEGAL_VALUE; }
    if (A->m != A->n) { warning(fn, "only square matrices"); return CHAMELEON_ERR_ILLEGAL_VALUE; }
    return 0;
}

static int finish(int rc, const ExecResult &res, RUNTIME_sequence_t *seq) {
    int status = rc ? rc : (res.error ? res.error : res.info);
    if (seq) seq->status = status;
    return status;
}

int CHAMELEON_dpotrf_Tile_Async(cham_uplo_t uplo, CHAM_desc_t *A, RUNTIME_sequence_t *sequence,
                                RUNTIME_request_t *request) {
    (void)request;
    int rc = ensure_init();
    if (rc) return rc;
    if ((rc = check_square_desc(A, "CHAMELEON_dpotrf_Tile"))) return finish(rc, ExecResult{}, sequence);
    if (uplo != ChamUpper && uplo != ChamLower) return finish(CHAMELEON_ERR_ILLEGAL_VALUE, ExecResult{}, sequence);
    ExecResult res;
    rc = run_cholesky_dag(MODE_FACT, uplo, A, nullptr, ctx().stream, &res);
    if (!rc) rc = desc_sync_to_host(A);
    return finish(rc, res, sequence);
}
int CHAMELEON_dpotrf_Tile(cham_uplo_t uplo, CHAM_desc_t *A) {
    RUNTIME_sequence_t seq{};
    return CHAMELEON_dpotrf_Tile_Async(uplo, A, &seq, nullptr);
}

int CHAMELEON_dpotrs_Tile_Async(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B, RUNTIME_sequence_t *sequence,
                                RUNTIME_request_t *request) {
    (void)request;
    int rc = ensure_init();
    if (rc) return rc;
    if ((rc = check_square_desc(A, "CHAMELEON_dpotrs_Tile"))) return finish(rc, ExecResult{}, sequence);
    if (!B || B->dtyp != ChamRealDouble || B->mb != A->mb || B->m != A->n)
        return finish(CHAMELEON_ERR_ILLEGAL_VALUE, ExecResult{}, sequence);
    if (uplo != ChamUpper && uplo != ChamLower) return finish(CHAMELEON_ERR_ILLEGAL_VALUE, ExecResult{}, sequence);
    ExecResult res;
    rc = run_cholesky_dag(MODE_SOLVE, uplo, A, B, ctx().stream, &res);
    if (!rc) rc = desc_sync_to_host(B);
    return finish(rc, res, sequence);
}
int CHAMELEON_dpotrs_Tile(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B) {
    RUNTIME_sequence_t seq{};
    return CHAMELEON_dpotrs_Tile_Async(uplo, A, B, &seq, nullptr);
}

int CHAMELEON_dposv_Tile_Async(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B, RUNTIME_sequence_t *sequence,
                               RUNTIME_request_t *request) {
    (void)request;
    int rc = ensure_init();
    if (rc) return rc;
    if ((rc = check_square_desc(A, "CHAMELEON_dposv_Tile"))) return finish(rc, ExecResult{}, sequence);
    if (!B || B->dtyp != ChamRealDouble || B->mb != A->mb || B->m != A->n)
        return finish(CHAMELEON_ERR_ILLEGAL_VALUE, ExecResult{}, sequence);
    if (uplo != ChamUpper && uplo != ChamLower) return finish(CHAMELEON_ERR_ILLEGAL_VALUE, ExecResult{}, sequence);
    ExecResult res;
    rc = run_cholesky_dag(MODE_FACT | MODE_SOLVE, uplo, A, B, ctx().stream, &res);
    if (!rc) rc = desc_sync_to_host(A);
    if (!rc) rc = desc_sync_to_host(B);
    return finish(rc, res, sequence);
}
int CHAMELEON_dposv_Tile(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B) {
    RUNTIME_sequence_t seq{};
    return CHAMELEON_dposv_Tile_Async(uplo, A, B, &seq, nullptr);
}

// LAPACK layout (compute/zposv.c:93-172, zpotrf.c:81, zpotrs.c:78): the user
// arrays are viewed in place through column-major tile addressing
// (control/compute_z.h:471-506, InPlace translation); host arrays are staged
// to the device and back.
}  // extern "C"

namespace chb {
// Device staging buffers of the LAPACK-layout entry points (grow-only, kept
// for the life of the process so repeated calls do not re-allocate).
static double *g_stage[3] = {nullptr, nullptr, nullptr};
static size_t g_stage_bytes[3] = {0, 0, 0};
double *staging(int slot, size_t bytes) {
    if (bytes > g_stage_bytes[slot]) {
        // the previous call that used the buffer is done (synchronous API);
        // pool memory: no device-wide synchronization
        cudaStreamSynchronize(ctx().stream);
        dev_free(g_stage[slot]);
        g_stage[slot] = nullptr;
        g_stage_bytes[slot] = 0;
        if (!(g_stage[slot] = (double *)dev_alloc(bytes))) return nullptr;
        g_stage_bytes[slot] = bytes;
    }
    return g_stage[slot];
}
bool is_device_ptr_pub(const void *p) { return is_device_ptr(p); }

double *stage_in(int slot, const double *host, int ld, int rows, int cols, cudaStream_t s) {
    double *d = staging(slot, std::max<size_t>((size_t)rows * cols * sizeof(double), 16));
    if (!d) return nullptr;
    if (rows > 0 && cols > 0 &&
        cudaMemcpy2DAsync(d, (size_t)rows * 8, host, (size_t)ld * 8, (size_t)rows * 8, cols, cudaMemcpyHostToDevice,
                          s) != cudaSuccess)
        return nullptr;
    return d;
}

int stage_out(double *host, int ld, const double *dev, int rows, int cols, cudaStream_t s) {
    if (rows <= 0 || cols <= 0) return 0;
    CHB_CUDA(cudaMemcpy2DAsync(host, (size_t)ld * 8, dev, (size_t)rows * 8, (size_t)rows * 8, cols,
                               cudaMemcpyDeviceToHost, s));
    return 0;
}

}  // namespace chb

extern "C" {

static int lapack_call(int mode, cham_uplo_t uplo, int N, int NRHS, double *A, int LDA, double *B, int LDB,
                       float *ms_out) {
    Context &c = ctx();
    cudaStream_t s = c.stream;
    const bool a_dev = is_device_ptr(A);
    const bool b_dev = (NRHS > 0 && B) ? is_device_ptr(B) : true;
    double *dA = A, *dB = B;
    // host arrays are staged densely (ld = N): only the N x cols block moves
    int lda = LDA, ldb = LDB;
    if (!a_dev) {
        if (!(dA = stage_in(0, A, LDA, N, N, s))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        lda = N;
    }
    if (!b_dev) {
        if (!(dB = stage_in(1, B, LDB, N, NRHS, s))) return CHAMELEON_ERR_OUT_OF_RESOURCES;
        ldb = N;
    }
    CHAM_desc_t *dAd = nullptr, *dBd = nullptr;
    desc_create_cm(&dAd, dA, lda, N, N, c.tile_size);
    if (NRHS > 0 && (mode & MODE_SOLVE)) desc_create_cm(&dBd, dB, ldb, N, NRHS, c.tile_size);
    ExecResult res;
    int rc = run_cholesky_dag(mode, uplo, dAd, dBd, s, &res);
    if (ms_out) *ms_out = res.ms;
    if (!a_dev && (mode & MODE_FACT)) stage_out(A, LDA, dA, N, N, s);
    if (!b_dev && (mode & MODE_SOLVE)) stage_out(B, LDB, dB, N, NRHS, s);
    cudaStreamSynchronize(s);
    CHAMELEON_Desc_Destroy(&dAd);
    if (dBd) CHAMELEON_Desc_Destroy(&dBd);
    if (rc) return rc;
    return res.error ? res.error : res.info;
}

int CHAMELEON_dposv(cham_uplo_t uplo, int N, int NRHS, double *A, int LDA, double *B, int LDB) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (N < 0) return -2;
    if (NRHS < 0) return -3;
    if (LDA < std::max(1, N)) return -5;
    if (LDB < std::max(1, N)) return -7;
    if (N == 0 || NRHS == 0) return 0;
    return lapack_call(MODE_FACT | MODE_SOLVE, uplo, N, NRHS, A, LDA, B, LDB, nullptr);
}

int CHAMELEON_dpotrf(cham_uplo_t uplo, int N, double *A, int LDA) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (N < 0) return -2;
    if (LDA < std::max(1, N)) return -4;
    if (N == 0) return 0;
    return lapack_call(MODE_FACT, uplo, N, 0, A, LDA, nullptr, 1, nullptr);
}

int CHAMELEON_dpotrs(cham_uplo_t uplo, int N, int NRHS, double *A, int LDA, double *B, int LDB) {
    int rc = ensure_init();
    if (rc) return rc;
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (N < 0) return -2;
    if (NRHS < 0) return -3;
    if (LDA < std::max(1, N)) return -5;
    if (LDB < std::max(1, N)) return -7;
    if (N == 0 || NRHS == 0) return 0;
    return lapack_call(MODE_SOLVE, uplo, N, NRHS, A, LDA, B, LDB, nullptr);
}

// Device time (ms) of the last executor launch of a LAPACK-layout dposv on
// device arrays: used by the benchmark to separate kernel time from staging.
int CHAM_B200_dposv_timed(cham_uplo_t uplo, int N, int NRHS, double *A, int LDA, double *B, int LDB,
                          float *device_ms) {
    int rc = ensure_init();
    if (rc) return rc;
    return lapack_call(MODE_FACT | MODE_SOLVE, uplo, N, NRHS, A, LDA, B, LDB, device_ms);
}

// ---- measurement hooks (benchmark) ------------------------------------------
// Device events on the library's stream: slot 0..7.
static cudaEvent_t g_ev[8] = {};
int CHAM_B200_Event_Record(int slot) {
    if (ensure_init() || slot < 0 || slot >= 8) return CHAMELEON_ERR_ILLEGAL_VALUE;
    if (!g_ev[slot]) CHB_CUDA(cudaEventCreate(&g_ev[slot]));
    CHB_CUDA(cudaEventRecord(g_ev[slot], ctx().stream));
    return 0;
}
float CHAM_B200_Event_Elapsed(int a, int b) {
    if (a < 0 || b < 0 || a >= 8 || b >= 8 || !g_ev[a] || !g_ev[b]) return -1.f;
    cudaEventSynchronize(g_ev[b]);
    float ms = -1.f;
    cudaEventElapsedTime(&ms, g_ev[a], g_ev[b]);
    return ms;
}
unsigned long long CHAM_B200_Launch_Count(void) { return g_launch_count.load(); }
int CHAM_B200_Device_Sync(void) {
    return cudaStreamSynchronize(ctx().stream) == cudaSuccess ? 0 : CHAMELEON_ERR_UNEXPECTED;
}
// Phase breakdown of the last mixed solve: out[7] = {factor, refine_solve,
// residual, cast, total (ms), iterations, fallback}.
int CHAM_B200_Mixed_Stats(double *out) {
    const MixedStats &m = g_mixed_stats;
    out[0] = m.factor_ms; out[1] = m.refine_solve_ms; out[2] = m.residual_ms; out[3] = m.cast_ms;
    out[4] = m.total_ms; out[5] = m.iterations; out[6] = m.fallback;
    return 0;
}

}  // extern "C"
