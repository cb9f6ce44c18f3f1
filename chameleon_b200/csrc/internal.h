// internal.h -- host-side internals shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/chameleon_b200.h"
#include "executor.cuh"

namespace chb {

// Library context: the reference keeps one global context
// (control/context.c:145-221); so does this library.
struct Context {
    bool initialized = false;
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t order_event = nullptr;   // orders `stream` after the caller's default stream
    int tile_size = 384;          // CHAMELEON_TILE_SIZE default (control/context.c:162)
    int inner_block = 48;
    int warnings = 1;
    int precision = CHAM_B200_PREC_BF16X3;
    int refine_maxiter = 30;
    long long wait_budget_us = 20000000;
    bool use_tcgen05 = true;      // tcgen05 trailing updates in the BF16x3 factorization
    bool rec_tile = false;        // FP32 factorization: recursive tile POTRF with full tile inverses
    bool xinv_solve = true;       // FP32 substitutions with full diagonal-tile inverses
    bool potrf_cta = false;        // one executor CTA dedicated to the diagonal-tile factorizations
    // update group sizes (panels applied per trailing-update task) per path:
    // FP64 DMMA, FP32 split products on mma.sync, FP32 on tcgen05
    int kgroup_f64 = 8, kgroup_f32 = 1, kgroup_tc = 8;
    int utail_f64 = 2;             // single-panel update groups closing each tile column, FP64 path
    // tile size of the mixed solver's FP32 copy of A (0: A's own tile size);
    // used when it divides A's tile size
    int factor_nb = 256;
    // expected host-to-device copy bandwidth (GB/s): orders the tasks of a
    // factorization that starts while its matrix is still arriving
    int h2d_gbs = 50;
    int desc_ids = 0;
    std::mutex mu;
};
Context &ctx();

// Count of this library's kernel launches (reported by the benchmark).
extern std::atomic<unsigned long long> g_launch_count;
#define CHB_LAUNCHED(n) (::chb::g_launch_count += (n))

// Phase breakdown of the last mixed-precision solve (device times, ms).
struct MixedStats {
    float factor_ms = 0;        // FP32 factorization + first solve (one DAG launch)
    float refine_solve_ms = 0;  // correction solves
    float residual_ms = 0;      // FP64 residuals
    float cast_ms = 0;          // casts + norm
    float total_ms = 0;
    int iterations = 0;
    int fallback = 0;
};
extern MixedStats g_mixed_stats;

#define CHB_CUDA(call)                                                                 \
    do {                                                                               \
        cudaError_t _e = (call);                                                       \
        if (_e != cudaSuccess) {                                                       \
            chb::report_cuda_error(#call, _e, __FILE__, __LINE__);                     \
            return CHAMELEON_ERR_UNEXPECTED;                                           \
        }                                                                              \
    } while (0)

void report_cuda_error(const char *what, cudaError_t e, const char *file, int line);
void warning(const char *func, const char *msg);
int ensure_init();

// Device-resident view of a descriptor's tile addressing (cached per descriptor).
struct DescDev {
    int64_t *off = nullptr;   // mt*nt element offsets
    int *ld = nullptr;        // mt leading dimensions
};
struct DescPriv {
    DescDev dev;
    int cm_view = 0;          // 1: column-major user array view (LAPACK-layout entry points)
    std::vector<signed char> prec;   // per tile (m + mt n): 0 FP64, 1 FP32, 2 FP16 values (gered.cu)
};
DescPriv *priv(const CHAM_desc_t *d);
int desc_tile_rows(const CHAM_desc_t *d, int m);
int desc_tile_cols(const CHAM_desc_t *d, int n);
int64_t desc_tile_off(const CHAM_desc_t *d, int m, int n);
int desc_tile_ld(const CHAM_desc_t *d, int m);
int desc_upload(CHAM_desc_t *d);
// Descriptor over tiles addressed by caller tables (host arrays): tile (m, n)
// at base + off[m + mt n], leading dimension ld[m]; mb x nb tiles (nb <= 0: mb).
int desc_create_from_tables(CHAM_desc_t **desc, double *base, int mb, int m, int n, const int64_t *off,
                            const int *ld, int nb = 0);
cudaStream_t meta_stream();   // private stream of descriptor metadata uploads
// Workspace memory allocated / released in stream order on the meta stream
// (no device-wide synchronization, no kernel); contents undefined.
void *dev_alloc(size_t bytes);
void dev_free(void *p);
// Map `bytes` of device memory into the library pool ahead of use.
int pool_reserve(size_t bytes);
// Tile-layout (CCRB) m x n descriptor on caller-owned device storage of at
// least m * n elements (not freed by Desc_Destroy); uploaded.
int desc_create_tiled_on(CHAM_desc_t **desc, cham_flttype_t dtyp, void *storage, int nb, int m, int n);
// Create a descriptor viewing a device column-major array (ld = lda) with
// tile size nb: tile (m,n) at A + m*nb + n*nb*lda (control/descriptor.h:238-252).
int desc_create_cm(CHAM_desc_t **desc, double *dA, int lda, int m, int n, int nb);
int desc_sync_to_host(CHAM_desc_t *d);
double *staging(int slot, size_t bytes);   // LAPACK-layout staging buffers (0: A, 1: B, 2: X)
// Copy the rows x cols block of a host array (leading dimension ld) into
// staging slot `slot` with leading dimension rows; and back.
double *stage_in(int slot, const double *host, int ld, int rows, int cols, cudaStream_t s);
int stage_out(double *host, int ld, const double *dev, int rows, int cols, cudaStream_t s);

// Device workspace of one executor stream: dependency counters, inverted
// diagonal blocks, split-BF16 panel chunks (tcgen05 path), state, events.
// Grow-only; one per concurrent caller (the synchronous API uses a global one).
struct ExecWs {
    uint8_t *split = nullptr;
    size_t split_bytes = 0;
    void *xinv = nullptr;               // full inverses of the diagonal tiles (FP32 solves)
    size_t xinv_bytes = 0;
    const void *xinv_owner = nullptr;   // factor storage the inverses belong to (nullptr: none)
    int xinv_n = 0, xinv_nt = 0, xinv_nb = 0;
    void *y = nullptr;                  // forward-substitution results (MODE_XINV)
    size_t y_bytes = 0;
    size_t ctr_bytes = 0, inv_bytes = 0;
    void *ctr = nullptr;
    void *inv = nullptr;
    ExecState *st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

// Workspace of one mixed-precision solve stream (mixed.cu).
struct MixedWs {
    CHAM_desc_t *A32 = nullptr, *B32 = nullptr, *R = nullptr;   // views on the buffers below
    void *a32_buf = nullptr, *b32_buf = nullptr, *r_buf = nullptr;   // grow-only (dev_alloc)
    size_t a32_cap = 0, b32_cap = 0, r_cap = 0;
    int N = -1, NB = -1, NBf = -1, nrhs = -1;   // NBf: tile size of A32 / B32 (factor_tile(NB))
    unsigned long long *rmax = nullptr, *xmax = nullptr;
    double *colsum = nullptr;
    double *diag = nullptr;       // symmetric copies of the diagonal tiles (residuals)
    size_t diag_cap = 0;
    double *part = nullptr;       // split-K partial products of the residual
    size_t part_cap = 0;
    int *flag = nullptr;
    int cap_rhs = 0, cap_n = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

// Batched dposv (batch.cu): one item per independent system; offsets in
// elements into the batch's A / B arrays.
struct BatchItem {
    int64_t a_off, b_off;
    int n, nrhs, lda, ldb;   // nrhs == 0: factor only
    int info_idx;
    int pad;
};
// Device workspace of one batch stream (grow-only).
struct BatchWs {
    void *items = nullptr;
    size_t items_bytes = 0;
    double *scratch = nullptr;
    size_t scratch_bytes = 0;
    int *cursor = nullptr;
    int *info = nullptr;
    size_t info_n = 0;
    cudaStream_t side = nullptr;          // small-bin stream (joined back before return)
    cudaEvent_t fork = nullptr, join = nullptr;
};
extern BatchWs g_bws;   // the synchronous API's
int bws_reserve(BatchWs &ws, size_t item_bytes, size_t scratch_bytes, size_t ninfo);
// One persistent launch over `items` (sorted in place, largest first).
int launch_posv_batch(std::vector<BatchItem> &items, double *A, double *B, int upper, int *info, cudaStream_t s,
                      BatchWs &ws);

// Release every buffer and descriptor of a workspace (its stream is idle).
void free_mixed_ws(MixedWs &m);
void free_exec_ws(ExecWs &w);

// A factorization whose FP32 tiles are cast inside the launch from an FP64
// column-major copy of A that the copy engine is still writing (MODE_CAST):
// tile column q has arrived once arrive[q] >= epoch.  colsum (N doubles,
// zeroed by the caller) receives the row sums of |A| (symmetric), ovf is set
// when a referenced value does not fit FP32.  h2d_gbs: expected copy
// bandwidth, for the order of the task list.
struct CastIn {
    const double *src;
    int64_t ld;
    const int *arrive;
    int epoch;
    double *colsum;
    int *ovf;
    int h2d_gbs;
};

// Executor entry (executor.cu).
struct ExecResult {
    int info = 0;     // >0: LAPACK-style order of the failing minor
    int error = 0;    // CHAMELEON_ERR_*
    float ms = 0.f;   // device time of the launch
};
// A, B: double descriptors (FP64 path) or float descriptors (split-precision
// path, `split` = SPLIT_BF16X3 or SPLIT_TF32X3 from core.cuh).
// ws: workspace (nullptr: the global one of the synchronous API); grid:
// number of persistent CTAs (0: one per SM).
// flags: EXEC_REUSE_INV -- a solve-only launch may reuse the full diagonal-tile
// inverses a previous launch on the same workspace computed for this factor.
enum ExecFlags : int { EXEC_REUSE_INV = 1 };
int run_cholesky_dag(int mode, cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B, cudaStream_t s,
                     ExecResult *res, int split = 0, ExecWs *ws = nullptr, int grid = 0, int flags = 0,
                     const CastIn *cin = nullptr);

// Tile size of the mixed solver's FP32 factorization for FP64 tile size NB (mixed.cu).
int factor_tile(int NB);

// A host matrix whose referenced triangle is being copied to dA (column-major,
// ld) one tile column at a time; column q has landed once arrive[q] >= epoch
// (tri_stream_start, mixed.cu); `done` is recorded after the last copy.
struct TriStream {
    double *dA;
    int64_t ld;
    const int *arrive;
    int epoch;
    cudaEvent_t done;
    int h2d_gbs;
};
// Copy stream, flags and pinned epoch word of the triangle streaming.
struct TriStreamState {
    cudaStream_t cs = nullptr;
    cudaEvent_t done = nullptr;
    int *d_arrive = nullptr;
    int cap = 0;
    int *h_epoch = nullptr;
    int epoch = 0;
};
int tri_stream_start(TriStreamState &ts, cham_uplo_t uplo, const double *hA, int lda, double *dA, int N, int nb,
                     TriStream *out);
void free_tri_stream(TriStreamState &ts);

// Mixed-precision solve on an explicit stream and workspaces (mixed.cu).
// factored = true: m.A32 already holds the low-precision factor of A (resident
// factor re-use); only the solve and refinement run.
// tri: A (FP64, column-major view of tri->dA) is still arriving from the host;
// its tiles are cast inside the factorization launch (MODE_CAST).
int mixed_posv_ws(cham_uplo_t uplo, int precision, CHAM_desc_t *A, CHAM_desc_t *B, CHAM_desc_t *X, int *iter_out,
                  CHAM_b200_refine_info_t *info, cudaStream_t s, MixedWs &m, ExecWs *ews, int grid, bool factored,
                  const TriStream *tri = nullptr);

}  // namespace chb
