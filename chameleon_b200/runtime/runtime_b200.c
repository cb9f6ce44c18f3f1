/*
 * runtime_b200.c -- a Chameleon runtime plugin ("runtime/b200") on the B200
 * persistent tile-DAG executor.
 *
 * Chameleon's algorithms (compute/pz*.c) submit their work through a runtime
 * interface: INSERT_TASK_* per tile kernel (include/chameleon/tasks_z.h:64-380)
 * and the RUNTIME_* services (include/chameleon/runtime.h:51-714: context,
 * sequences, descriptors, options).  StarPU, PaRSEC, QUARK and OpenMP each
 * implement it (runtime/<name>/).  This file implements it for the B200:
 *
 *   * INSERT_TASK_dpotrf / dtrsm / dsyrk / dgemm append one record per call to
 *     the sequence's DAG (CHAM_B200_Dag_Record), in the logical lower-triangle
 *     coordinates of the executor;
 *   * RUNTIME_sequence_wait runs the recorded DAG in ONE persistent launch
 *     (CHAM_B200_Dag_Run) over the descriptors' tiles, and stores LAPACK's info
 *     in the sequence status, as the reference's codelets do
 *     (runtime/starpu/codelets/codelet_zpotrf.c:72-74);
 *   * descriptor tiles live in CUDA managed memory (RUNTIME_malloc), so that
 *     the host-side descriptor code and the kernels share them.
 *
 * chameleon_pdpotrf and chameleon_pdtrsm (compute/pzpotrf.c:84-194,
 * compute/pztrsm.c:58-200, d precision) and the public drivers above them
 * (compute/zposv.c, zpotrf.c, zpotrs.c) run unchanged on this runtime.  Tile
 * kernels outside the Cholesky path have no INSERT_TASK here.
 *
 * Built against the Chameleon sources (their headers define CHAM_desc_t,
 * RUNTIME_option_t, CHAM_context_t); it links libchameleon_b200.so and calls
 * only its CHAM_B200_* entry points, declared below with plain C types.
 *
 * Recording without running: with CHAMELEON_B200_RUNTIME_RECORD_ONLY=1 in the
 * environment (or chameleon_b200_runtime_record_only(1)), sequence waits keep
 * the records for inspection (chameleon_b200_runtime_last_dag) instead of
 * running them, and RUNTIME_malloc uses host memory -- this needs no GPU.
 */
#include "control/common.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <cuda_runtime.h>

/* libchameleon_b200.so (include/chameleon_b200.h), plain C types */
typedef struct cham_b200_dag_s *b200_dag_t;
int CHAM_B200_Init(void);
int CHAM_B200_Dag_Create(b200_dag_t *dag);
int CHAM_B200_Dag_Destroy(b200_dag_t dag);
int CHAM_B200_Dag_Clear(b200_dag_t dag);
int CHAM_B200_Dag_Record(b200_dag_t dag, int kind, int m, int n, int k, int bn);
int CHAM_B200_Dag_Size(b200_dag_t dag);
int CHAM_B200_Dag_Get(b200_dag_t dag, int *out, int cap);
int CHAM_B200_Dag_Run(b200_dag_t dag, int uplo, int N, int NB, double *A, const int64_t *a_off, const int *a_ld,
                      int nrhs, int NBB, double *B, const int64_t *b_off, const int *b_ld, int *info);
enum { DAG_POTRF = 1, DAG_PANEL = 2, DAG_UPDATE = 3, DAG_FWD_SOLVE = 4, DAG_FWD_UPDATE = 5, DAG_BWD_SOLVE = 6,
       DAG_BWD_UPDATE = 7 };

/* ------------------------------------------------------------------------- */
/* Plugin state                                                              */
/* ------------------------------------------------------------------------- */
static int g_record_only = -1;   /* -1: read the environment at first use */
static int g_gpu = 0;            /* the B200 library is initialized       */

/* The records of the last sequence waited on in record-only mode. */
static int *g_last = NULL;
static int g_last_n = 0;

int chameleon_b200_runtime_record_only(int on) {
    g_record_only = on ? 1 : 0;
    return 0;
}

static int record_only(void) {
    if (g_record_only < 0) {
        const char *e = getenv("CHAMELEON_B200_RUNTIME_RECORD_ONLY");
        g_record_only = (e && *e && *e != '0') ? 1 : 0;
    }
    return g_record_only;
}

/* Copies the records of the last sequence waited on in record-only mode (5
 * ints each: kind, m, n, k, bn); returns their count. */
int chameleon_b200_runtime_last_dag(int *out, int cap) {
    const int n = g_last_n < cap ? g_last_n : cap;
    if (out && n > 0) memcpy(out, g_last, sizeof(int) * 5 * (size_t)n);
    return g_last_n;
}

/* Per-sequence state (RUNTIME_sequence_t.schedopt) */
typedef struct b200_seq_s {
    b200_dag_t dag;
    const CHAM_desc_t *A;   /* the factored matrix / the triangular factor */
    const CHAM_desc_t *B;   /* the right-hand sides (solves) */
    int uplo;
    int unsupported;        /* a task the executor cannot run was submitted */
} b200_seq_t;

static b200_seq_t *seq_state(const RUNTIME_option_t *options) {
    if (!options || !options->sequence) return NULL;
    return (b200_seq_t *)options->sequence->schedopt;
}

static void record(b200_seq_t *s, int kind, int m, int n, int k, int bn) {
    if (!s || s->unsupported) return;
    if (CHAM_B200_Dag_Record(s->dag, kind, m, n, k, bn) != 0) s->unsupported = 1;
}

/* ------------------------------------------------------------------------- */
/* Context, control                                                           */
/* ------------------------------------------------------------------------- */
void RUNTIME_context_create(CHAM_context_t *ctxt) {
    /* the reference's runtime ids have no value for this runtime: it is a
     * shared-memory runtime with eagerly allocated tiles, as OpenMP's */
    ctxt->scheduler = RUNTIME_SCHED_OPENMP;
}
void RUNTIME_context_destroy(CHAM_context_t *ctxt) { (void)ctxt; }
void RUNTIME_enable(void *runtime_ctxt, int option) { (void)runtime_ctxt; (void)option; }
void RUNTIME_disable(void *runtime_ctxt, int option) { (void)runtime_ctxt; (void)option; }

int RUNTIME_init(CHAM_context_t *ctxt, int ncpus, int ncudas, int nthreads_per_worker) {
    ctxt->nworkers = ncpus > 0 ? ncpus : 1;
    ctxt->ncudas = 0;   /* the algorithms' host-side CUDA paths are not used */
    ctxt->nthreads_per_worker = nthreads_per_worker;
    (void)ncudas;
    g_gpu = !record_only() && CHAM_B200_Init() == 0;
    return (g_gpu || record_only()) ? CHAMELEON_SUCCESS : CHAMELEON_ERR_NOT_INITIALIZED;
}
void RUNTIME_finalize(CHAM_context_t *ctxt) { (void)ctxt; }
void RUNTIME_pause(CHAM_context_t *ctxt) { ctxt->runtime_paused = CHAMELEON_TRUE; }
void RUNTIME_resume(CHAM_context_t *ctxt) { ctxt->runtime_paused = CHAMELEON_FALSE; }
void RUNTIME_barrier(CHAM_context_t *ctxt) {
    (void)ctxt;
    if (g_gpu) cudaDeviceSynchronize();
}
void RUNTIME_progress(CHAM_context_t *ctxt) { (void)ctxt; }
int RUNTIME_thread_rank(const CHAM_context_t *ctxt) { (void)ctxt; return 0; }
int RUNTIME_thread_size(const CHAM_context_t *ctxt) { (void)ctxt; return 1; }
int RUNTIME_comm_rank(const CHAM_context_t *ctxt) { (void)ctxt; return 0; }
int RUNTIME_comm_size(const CHAM_context_t *ctxt) { (void)ctxt; return 1; }
void RUNTIME_flush(CHAM_context_t *ctxt) { (void)ctxt; }
void RUNTIME_set_minmax_submitted_tasks(int min, int max) { (void)min; (void)max; }

double RUNTIME_get_time(void) {
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}
void RUNTIME_iteration_push(CHAM_context_t *ctxt, unsigned long iteration) { (void)ctxt; (void)iteration; }
void RUNTIME_iteration_pop(CHAM_context_t *ctxt) { (void)ctxt; }
void RUNTIME_start_profiling(void) {}
void RUNTIME_stop_profiling(void) {}
void RUNTIME_start_stats(void) {}
void RUNTIME_stop_stats(void) {}
void RUNTIME_schedprofile_display(void) {}
void RUNTIME_kernelprofile_display(void) {}

/* ------------------------------------------------------------------------- */
/* Sequences: the DAG of a sequence runs when it is waited on                 */
/* ------------------------------------------------------------------------- */
int RUNTIME_sequence_create(CHAM_context_t *ctxt, RUNTIME_sequence_t *sequence) {
    (void)ctxt;
    b200_seq_t *s = (b200_seq_t *)calloc(1, sizeof(b200_seq_t));
    if (!s || CHAM_B200_Dag_Create(&s->dag) != 0) {
        free(s);
        return CHAMELEON_ERR_OUT_OF_RESOURCES;
    }
    sequence->schedopt = s;
    return CHAMELEON_SUCCESS;
}

int RUNTIME_sequence_destroy(CHAM_context_t *ctxt, RUNTIME_sequence_t *sequence) {
    (void)ctxt;
    b200_seq_t *s = (b200_seq_t *)sequence->schedopt;
    if (s) {
        CHAM_B200_Dag_Destroy(s->dag);
        free(s);
    }
    sequence->schedopt = NULL;
    return CHAMELEON_SUCCESS;
}

/* Element offsets (from the first tile) and leading dimensions of the tiles
 * of a descriptor, as the executor addresses them. */
static int tile_tables(const CHAM_desc_t *d, double **base, int64_t **off, int **ld) {
    *base = (double *)d->get_blkaddr(d, 0, 0);
    *off = (int64_t *)malloc(sizeof(int64_t) * (size_t)d->mt * (size_t)d->nt);
    *ld = (int *)malloc(sizeof(int) * (size_t)d->mt);
    if (!*off || !*ld) return CHAMELEON_ERR_OUT_OF_RESOURCES;
    for (int n = 0; n < d->nt; ++n)
        for (int m = 0; m < d->mt; ++m)
            (*off)[m + (size_t)d->mt * n] = (double *)d->get_blkaddr(d, m, n) - *base;
    for (int m = 0; m < d->mt; ++m) (*ld)[m] = d->get_blkldd(d, m);
    return CHAMELEON_SUCCESS;
}

static int run_sequence(b200_seq_t *s, RUNTIME_sequence_t *sequence) {
    const int n = CHAM_B200_Dag_Size(s->dag);
    if (n <= 0) return CHAMELEON_SUCCESS;
    if (s->unsupported) return CHAMELEON_ERR_NOT_SUPPORTED;
    if (record_only()) {
        free(g_last);
        g_last = (int *)malloc(sizeof(int) * 5 * (size_t)n);
        g_last_n = g_last ? CHAM_B200_Dag_Get(s->dag, g_last, n) : 0;
        return CHAMELEON_SUCCESS;
    }
    const CHAM_desc_t *A = s->A, *B = s->B;
    if (!A || A->dtyp != ChamRealDouble || A->m != A->n || A->mb != A->nb || (B && (B->mb != A->mb || B->m != A->m)))
        return CHAMELEON_ERR_NOT_SUPPORTED;
    double *a = NULL, *b = NULL;
    int64_t *aoff = NULL, *boff = NULL;
    int *ald = NULL, *bld = NULL, info = 0;
    int rc = tile_tables(A, &a, &aoff, &ald);
    if (!rc && B) rc = tile_tables(B, &b, &boff, &bld);
    if (!rc)
        rc = CHAM_B200_Dag_Run(s->dag, s->uplo, A->m, A->mb, a, aoff, ald, B ? B->n : 0, B ? B->nb : 0, b, boff, bld,
                               &info);
    free(aoff);
    free(ald);
    free(boff);
    free(bld);
    if (!rc && info > 0 && sequence->status == CHAMELEON_SUCCESS) sequence->status = info;
    return rc;
}

int RUNTIME_sequence_wait(CHAM_context_t *ctxt, RUNTIME_sequence_t *sequence) {
    (void)ctxt;
    b200_seq_t *s = (b200_seq_t *)sequence->schedopt;
    if (!s) return CHAMELEON_SUCCESS;
    const int rc = run_sequence(s, sequence);
    CHAM_B200_Dag_Clear(s->dag);
    s->A = s->B = NULL;
    s->unsupported = 0;
    if (rc && sequence->status == CHAMELEON_SUCCESS) sequence->status = rc;
    return rc;
}

void RUNTIME_sequence_flush(CHAM_context_t *ctxt, RUNTIME_sequence_t *sequence, RUNTIME_request_t *request,
                            int status) {
    (void)ctxt;
    sequence->request = request;
    sequence->status = status;
    request->status = status;
}

/* ------------------------------------------------------------------------- */
/* Memory and descriptors                                                    */
/* ------------------------------------------------------------------------- */
void *RUNTIME_malloc(size_t size) {
    void *p = NULL;
    if (g_gpu) {
        if (cudaMallocManaged(&p, size ? size : 1, cudaMemAttachGlobal) != cudaSuccess) {
            cudaGetLastError();
            return NULL;
        }
        return p;
    }
    return malloc(size ? size : 1);
}
void RUNTIME_free(void *ptr, size_t size) {
    (void)size;
    if (!ptr) return;
    if (g_gpu) cudaFree(ptr);
    else free(ptr);
}
void RUNTIME_desc_create(CHAM_desc_t *desc) { (void)desc; }
int RUNTIME_desc_create_flatview(CHAM_desc_t *desc, const CHAM_desc_t *recdesc) {
    (void)desc;
    (void)recdesc;
    return CHAMELEON_ERR_NOT_SUPPORTED;
}
void RUNTIME_desc_register_recursive(CHAM_desc_t *desc, int dist_level) { (void)desc; (void)dist_level; }
void RUNTIME_desc_destroy_submit(CHAM_desc_t *desc, const RUNTIME_sequence_t *sequence) {
    (void)desc;
    (void)sequence;
}
void RUNTIME_desc_destroy(CHAM_desc_t *desc) { (void)desc; }
/* every sequence has completed when its wait returns: the host may read */
int RUNTIME_desc_acquire(const CHAM_desc_t *desc) {
    (void)desc;
    if (g_gpu) cudaDeviceSynchronize();
    return CHAMELEON_SUCCESS;
}
int RUNTIME_desc_release(const CHAM_desc_t *desc) { (void)desc; return CHAMELEON_SUCCESS; }
void RUNTIME_desc_flush(CHAM_desc_t *desc, const RUNTIME_sequence_t *sequence) { (void)desc; (void)sequence; }
void RUNTIME_data_flush(const RUNTIME_sequence_t *sequence, const CHAM_desc_t *A, int Am, int An) {
    (void)sequence;
    (void)A;
    (void)Am;
    (void)An;
}
void RUNTIME_data_unregister(const RUNTIME_sequence_t *sequence, const CHAM_desc_t *A, int Am, int An) {
    (void)sequence;
    (void)A;
    (void)Am;
    (void)An;
}
void *RUNTIME_data_getaddr(const CHAM_desc_t *A, int Am, int An) { return A->get_blktile(A, Am, An); }

/* ------------------------------------------------------------------------- */
/* Options                                                                    */
/* ------------------------------------------------------------------------- */
void RUNTIME_options_init(RUNTIME_option_t *options, const CHAM_context_t *context, RUNTIME_sequence_t *sequence,
                          RUNTIME_request_t *request) {
    memset(options, 0, sizeof(*options));
    options->sequence = sequence;
    options->request = request;
    options->profiling = context ? context->statistics_enabled : 0;
    options->parallel = context ? context->parallel_enabled : 0;
    options->workerid = -1;
}
void RUNTIME_options_finalize(RUNTIME_option_t *options, const CHAM_context_t *context) {
    (void)options;
    (void)context;
}
int RUNTIME_options_ws_alloc(RUNTIME_option_t *options, size_t wsize, size_t hsize) {
    /* the executor keeps its workspaces itself */
    options->ws_wsize = wsize;
    options->ws_hsize = hsize;
    return CHAMELEON_SUCCESS;
}
int RUNTIME_options_ws_free(RUNTIME_option_t *options) {
    options->ws_wsize = options->ws_hsize = 0;
    return CHAMELEON_SUCCESS;
}

/* Locality and profiling displays: nothing to restrict or display */
void RUNTIME_dlocality_allrestore(void) {}
void RUNTIME_dlocality_allrestrict(uint32_t device) { (void)device; }
void RUNTIME_dlocality_onerestrict(cham_tasktype_t task, uint32_t device) { (void)task; (void)device; }
void RUNTIME_dlocality_onerestore(cham_tasktype_t task) { (void)task; }
void RUNTIME_ddisplay_allprofile(void) {}
void RUNTIME_ddisplay_oneprofile(cham_tasktype_t task) { (void)task; }

/* ------------------------------------------------------------------------- */
/* Tile tasks of the Cholesky path (tasks_z.h after z->d generation)          */
/* ------------------------------------------------------------------------- */

/* INSERT_TASK_dpotrf (tasks_z.h:283): factor diagonal tile (Am, Am). */
void INSERT_TASK_dpotrf(const RUNTIME_option_t *options, cham_uplo_t uplo, int n, int nb, const CHAM_desc_t *A,
                        int Am, int An, int iinfo) {
    b200_seq_t *s = seq_state(options);
    (void)n;
    (void)nb;
    (void)iinfo;   /* the executor reports the global order itself */
    if (!s) return;
    if ((s->A && s->A != A) || Am != An) s->unsupported = 1;
    s->A = A;
    s->uplo = uplo;
    record(s, DAG_POTRF, Am, Am, Am, 0);
}

/* INSERT_TASK_dtrsm (tasks_z.h:362): on A's own tiles, the panel solve of
 * chameleon_pdpotrf; on another descriptor, a diagonal solve of
 * chameleon_pdtrsm (Left).  Forward when it applies L^-1 (Lower NoTrans,
 * Upper [Conj]Trans), backward when it applies L^-T. */
void INSERT_TASK_dtrsm(const RUNTIME_option_t *options, cham_side_t side, cham_uplo_t uplo, cham_trans_t transA,
                       cham_diag_t diag, int m, int n, int nb, double alpha, const CHAM_desc_t *A, int Am, int An,
                       const CHAM_desc_t *B, int Bm, int Bn) {
    b200_seq_t *s = seq_state(options);
    (void)m;
    (void)n;
    (void)nb;
    if (!s) return;
    if (diag != ChamNonUnit || alpha != 1.0 || Am != An) {
        s->unsupported = 1;
        return;
    }
    if (!s->A) {
        s->A = A;
        s->uplo = uplo;
    }
    if (A != s->A || uplo != (cham_uplo_t)s->uplo) {
        s->unsupported = 1;
        return;
    }
    if (B == s->A) {   /* panel: Right/Lower A(m,k), or Left/Upper A(k,n) */
        if ((uplo == ChamLower) != (side == ChamRight) || transA == ChamNoTrans) {
            s->unsupported = 1;
            return;
        }
        record(s, DAG_PANEL, uplo == ChamLower ? Bm : Bn, Am, Am, 0);
        return;
    }
    if (side != ChamLeft || (s->B && s->B != B)) {
        s->unsupported = 1;
        return;
    }
    s->B = B;
    const int fwd = (uplo == ChamLower) == (transA == ChamNoTrans);
    record(s, fwd ? DAG_FWD_SOLVE : DAG_BWD_SOLVE, Bm, Bm, Bm, Bn);
}

/* INSERT_TASK_dsyrk (tasks_z.h:312, from zherk): the diagonal-tile update
 * A(n,n) -= A(n,k) A(n,k)^T (Lower) or A(m,m) -= A(k,m)^T A(k,m) (Upper). */
void INSERT_TASK_dsyrk(const RUNTIME_option_t *options, cham_uplo_t uplo, cham_trans_t trans, int n, int k, int nb,
                       double alpha, const CHAM_desc_t *A, int Am, int An, double beta, const CHAM_desc_t *C, int Cm,
                       int Cn) {
    b200_seq_t *s = seq_state(options);
    (void)n;
    (void)k;
    (void)nb;
    (void)trans;
    if (!s) return;
    if (A != s->A || C != s->A || alpha != -1.0 || beta != 1.0 || Cm != Cn || uplo != (cham_uplo_t)s->uplo) {
        s->unsupported = 1;
        return;
    }
    record(s, DAG_UPDATE, Cm, Cm, uplo == ChamLower ? An : Am, 0);
}

/* INSERT_TASK_dgemm (tasks_z.h:64): on A's tiles, the trailing update of
 * chameleon_pdpotrf (Lower: C(m,n) -= A(m,k) A(n,k)^T; Upper: C(m,n) -=
 * A(k,m)^T A(k,n), the logical lower tile (n,m)); on the right-hand sides, the
 * update of chameleon_pdtrsm (B(m) -= op(L)(m,k) B(k)). */
void INSERT_TASK_dgemm(const RUNTIME_option_t *options, cham_trans_t transA, cham_trans_t transB, int m, int n, int k,
                       int nb, double alpha, const CHAM_desc_t *A, int Am, int An, const CHAM_desc_t *B, int Bm,
                       int Bn, double beta, const CHAM_desc_t *C, int Cm, int Cn) {
    b200_seq_t *s = seq_state(options);
    (void)m;
    (void)n;
    (void)k;
    (void)nb;
    if (!s) return;
    if (A != s->A || alpha != -1.0 || beta != 1.0) {
        s->unsupported = 1;
        return;
    }
    if (C == s->A) {
        if (B != s->A) {
            s->unsupported = 1;
            return;
        }
        if (s->uplo == ChamLower) record(s, DAG_UPDATE, Cm, Cn, An, 0);
        else record(s, DAG_UPDATE, Cn, Cm, Am, 0);
        (void)transA;
        (void)transB;
        return;
    }
    if (B != C || (s->B && s->B != C) || Bn != Cn) {
        s->unsupported = 1;
        return;
    }
    s->B = C;
    /* the source row of the right-hand sides is Bm; the updated one is Cm */
    record(s, Cm > Bm ? DAG_FWD_UPDATE : DAG_BWD_UPDATE, Cm, Bm, Bm, Cn);
}
