/*
 * chameleon_b200.h -- public C ABI of the B200-native tiled Cholesky path.
 *
 * Drop-in for Chameleon's d-precision Cholesky factor/solve API
 * (include/chameleon.h, include/chameleon/chameleon_z.h after z->d
 * generation) and for its GPU tile-kernel ABI (gpucublas/include/gpucublas/
 * gpucublas_z.h, gpucublas_zc.h after generation).  Enum values, argument
 * order and error conventions are those of the reference; citations are given
 * per entry point as `file:line` inside the reference project.
 *
 * Memory model: descriptor storage lives in device memory (HBM).  A descriptor
 * created over a host pointer is staged to the device once and copied back
 * after every synchronous call that writes it; one created over a device
 * pointer is used in place.  All computation runs on the GPU; there is no CPU
 * fallback -- every entry point returns CHAMELEON_ERR_NOT_INITIALIZED /
 * CHAMELEON_ERR_UNEXPECTED when no CUDA device is usable.
 */
#ifndef CHAMELEON_B200_H
#define CHAMELEON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------- */
/* Constants (include/chameleon/constants.h:30-445; identical values)         */
/* ------------------------------------------------------------------------- */
typedef enum { Cham8 = 0, ChamHalf = 1, ChamSingle = 2, ChamDouble = 3 } cham_arithmetic_t;
typedef enum { ChamInt = 0, ChamReal = 1, ChamComplex = 2 } cham_ftype_t;
typedef enum {
    ChamRealHalf   = (1 << 2) | 1,
    ChamRealFloat  = (1 << 2) | 2,
    ChamRealDouble = (1 << 2) | 3,
} cham_flttype_t;
typedef enum { ChamCM = 101, ChamRM = 102, ChamCCRB = 103, ChamCRRB = 104 } cham_storage_t;
typedef enum { ChamNoTrans = 111, ChamTrans = 112, ChamConjTrans = 113 } cham_trans_t;
typedef enum { ChamUpper = 121, ChamLower = 122, ChamUpperLower = 123 } cham_uplo_t;
typedef enum { ChamNonUnit = 131, ChamUnit = 132 } cham_diag_t;
typedef enum { ChamLeft = 141, ChamRight = 142 } cham_side_t;
typedef enum {
    ChamOneNorm = 171, ChamFrobeniusNorm = 174, ChamInfNorm = 175, ChamMaxNorm = 177
} cham_normtype_t;

#define CHAMELEON_FALSE 0
#define CHAMELEON_TRUE  1

/* CHAMELEON_Enable / Disable features (constants.h:357-369) */
#define CHAMELEON_WARNINGS   1
#define CHAMELEON_ERRORS     2
#define CHAMELEON_AUTOTUNING 3
/* CHAMELEON_Set / Get parameters (constants.h:374-382) */
#define CHAMELEON_CONCURRENCY      1
#define CHAMELEON_TILE_SIZE        2
#define CHAMELEON_INNER_BLOCK_SIZE 3
#define CHAMELEON_TRANSLATION_MODE 7
#define CHAMELEON_LOOKAHEAD        8
/* B200 additions to CHAMELEON_Set / Get */
#define CHAMELEON_B200_PRECISION      101 /* factorization precision of the mixed solver */
#define CHAMELEON_B200_REFINE_MAXITER 102 /* iterative-refinement iteration cap           */
#define CHAMELEON_B200_WAIT_BUDGET_MS 103 /* bound on any device-side dependency wait     */
#define CHAMELEON_B200_WAIT_BUDGET_US 104 /* the same bound in microseconds              */
#define CHAMELEON_B200_TCGEN05        105 /* 1: tcgen05 trailing updates in BF16x3 (default) */
#define CHAMELEON_B200_REC_TILE       106 /* 1: FP32 factorization with recursive diagonal tiles
                                             and full tile inverses; 0: blocked (default) */
#define CHAMELEON_B200_XINV_SOLVE     107 /* 1: FP32 substitutions apply full inverses of the
                                             diagonal tiles, kept across refinement solves (default) */
#define CHAMELEON_B200_POTRF_CTA      108 /* 1: one executor CTA runs all diagonal-tile
                                             factorizations; 0: any CTA (default) */
#define CHAMELEON_B200_UPD_GROUP_F64  109 /* panels applied per trailing-update task, FP64 path (default 8) */
#define CHAMELEON_B200_UPD_GROUP_F32  110 /* the same, FP32 split products on mma.sync (default 1) */
#define CHAMELEON_B200_UPD_GROUP_TC   111 /* the same, FP32 BF16x3 on tcgen05 (default 8) */
#define CHAMELEON_B200_FACTOR_NB      112 /* tile size of the mixed solver's FP32 factorization;
                                             0: the tile size of A (default 256 when it divides A's) */
#define CHAMELEON_B200_UPD_TAIL_F64   113 /* FP64 path: the last panels of each tile column applied
                                             one per update task (0..8, default 2) */

/* Factorization precisions for CHAMELEON_B200_PRECISION */
#define CHAM_B200_PREC_FP64   0
#define CHAM_B200_PREC_FP32   1
#define CHAM_B200_PREC_BF16X3 2

/* Descriptor allocation modes (constants.h:412-413) */
#define CHAMELEON_MAT_ALLOC_GLOBAL NULL
#define CHAMELEON_MAT_ALLOC_TILE   ((void *)-1)

/* Return codes (constants.h:434-445) */
#define CHAMELEON_SUCCESS               0
#define CHAMELEON_ERR_NOT_INITIALIZED  -101
#define CHAMELEON_ERR_REINITIALIZED    -102
#define CHAMELEON_ERR_NOT_SUPPORTED    -103
#define CHAMELEON_ERR_ILLEGAL_VALUE    -104
#define CHAMELEON_ERR_NOT_FOUND        -105
#define CHAMELEON_ERR_OUT_OF_RESOURCES -106
#define CHAMELEON_ERR_INTERNAL_LIMIT   -107
#define CHAMELEON_ERR_UNALLOCATED      -108
#define CHAMELEON_ERR_FILESYSTEM       -109
#define CHAMELEON_ERR_UNEXPECTED       -110
#define CHAMELEON_ERR_SEQUENCE_FLUSHED -111
/* B200 addition: a device-side dependency wait ran past its budget; the
 * persistent executor drained and returned without faulting the device. */
#define CHAMELEON_ERR_DEVICE_TIMEOUT   -120

/* ------------------------------------------------------------------------- */
/* Descriptor and tile (include/chameleon/struct.h:53-61,179-270)             */
/* ------------------------------------------------------------------------- */
typedef struct chameleon_tile_s {
    void          *mat;     /* device address of the tile                 */
    int            rank, m, n, ld;
    int8_t         format;
    cham_flttype_t flttype;
} CHAM_tile_t;

struct chameleon_desc_s;
typedef struct chameleon_desc_s CHAM_desc_t;

typedef void *(*blkaddr_fct_t)(const CHAM_desc_t *, int, int);
typedef int   (*blkldd_fct_t)(const CHAM_desc_t *, int);

struct chameleon_desc_s {
    char          *name;
    blkaddr_fct_t  get_blkaddr;  /* device address of tile (m, n)         */
    blkldd_fct_t   get_blkldd;   /* leading dimension of tile row m       */
    CHAM_tile_t   *tiles;        /* host array of mt*nt tile views        */
    void          *mat;          /* device base of the tile storage       */
    void          *host_mat;     /* caller host pointer staged in/out, or NULL */
    size_t         A21, A12, A22;
    cham_storage_t styp;
    cham_flttype_t dtyp;
    int mb, nb, bsiz;
    int i, j, m, n, lm, ln;
    int mt, nt, lmt, lnt;
    int llm1, lln1;
    int lda;                     /* ChamCM views only: leading dimension of the user array */
    int alloc_mat;               /* 1 when the library owns `mat`         */
    int id;
    void *schedopt;              /* executor-private state                */
};

/* Sequences (control/async.c:33-85) -- every call here is synchronous on
 * return, sequences carry status only. */
typedef struct runtime_sequence_s {
    int   status;
    void *request;
    void *schedopt;
} RUNTIME_sequence_t;
typedef struct runtime_request_s {
    int status;
} RUNTIME_request_t;
#define RUNTIME_REQUEST_INITIALIZER { 0 }

/* ------------------------------------------------------------------------- */
/* Control (include/chameleon.h:120-200; control/context.c:145-571)           */
/* ------------------------------------------------------------------------- */
int  __chameleon_init(int nworkers, int ncudas);
int  __chameleon_finalize(void);
#define CHAMELEON_Init(_nworkers_, _ncudas_) __chameleon_init((_nworkers_), (_ncudas_))
#define CHAMELEON_Finalize() __chameleon_finalize()
int  CHAMELEON_Initialized(void);
int  CHAMELEON_Set(int param, int value);
int  CHAMELEON_Get(int param, int *value);
int  CHAMELEON_Enable(int option);
int  CHAMELEON_Disable(int option);
const char *CHAMELEON_B200_Strerror(int code);

/* control/descriptor.c:749-756 */
int  CHAMELEON_Desc_Create(CHAM_desc_t **desc, void *mat, cham_flttype_t dtyp, int mb, int nb,
                           int bsiz, int lm, int ln, int i, int j, int m, int n, int p, int q);
int  CHAMELEON_Desc_Destroy(CHAM_desc_t **desc);
int  CHAMELEON_Desc_Flush(const CHAM_desc_t *desc, const RUNTIME_sequence_t *sequence);
int  CHAMELEON_Desc_Acquire(const CHAM_desc_t *desc);
int  CHAMELEON_Desc_Release(const CHAM_desc_t *desc);
/* include/chameleon.h:130-131: column-major host/device array <-> tiles */
int  CHAMELEON_Lap2Desc(cham_uplo_t uplo, void *A, int LDA, CHAM_desc_t *descA);
int  CHAMELEON_Desc2Lap(cham_uplo_t uplo, CHAM_desc_t *descA, void *A, int LDA);
int  CHAMELEON_Sequence_Create(RUNTIME_sequence_t **sequence);
int  CHAMELEON_Sequence_Destroy(RUNTIME_sequence_t *sequence);
int  CHAMELEON_Sequence_Wait(RUNTIME_sequence_t *sequence);

/* ------------------------------------------------------------------------- */
/* Cholesky path (include/chameleon/chameleon_z.h after z->d generation)      */
/* ------------------------------------------------------------------------- */
/* compute/zposv.c:93 (LAPACK layout; A, B host or device column-major)      */
int CHAMELEON_dposv(cham_uplo_t uplo, int N, int NRHS, double *A, int LDA, double *B, int LDB);
/* compute/zposv.c:222 / :276 */
int CHAMELEON_dposv_Tile(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B);
int CHAMELEON_dposv_Tile_Async(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B,
                               RUNTIME_sequence_t *sequence, RUNTIME_request_t *request);
/* compute/zpotrf.c:81 / :192 / :246 */
int CHAMELEON_dpotrf(cham_uplo_t uplo, int N, double *A, int LDA);
int CHAMELEON_dpotrf_Tile(cham_uplo_t uplo, CHAM_desc_t *A);
int CHAMELEON_dpotrf_Tile_Async(cham_uplo_t uplo, CHAM_desc_t *A,
                                RUNTIME_sequence_t *sequence, RUNTIME_request_t *request);
/* compute/zpotrs.c:78 / :198 / :253 */
int CHAMELEON_dpotrs(cham_uplo_t uplo, int N, int NRHS, double *A, int LDA, double *B, int LDB);
int CHAMELEON_dpotrs_Tile(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B);
int CHAMELEON_dpotrs_Tile_Async(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B,
                                RUNTIME_sequence_t *sequence, RUNTIME_request_t *request);
/* compute/zpotrf_batch.c:89 -- every tile of A is an independent matrix */
int CHAMELEON_dpotrf_batch_Tile(cham_uplo_t uplo, CHAM_desc_t *A);
/* compute/ztrsm_batch.c:180 -- tile (m,n) of B solved with tile (m,n) of A */
int CHAMELEON_dtrsm_batch_Tile(cham_side_t side, cham_uplo_t uplo, cham_trans_t trans,
                               cham_diag_t diag, double alpha, CHAM_desc_t *A, CHAM_desc_t *B);
/* compute/zgemm_batch.c:193 / zherk_batch.c:176 (zherk -> dsyrk): one
 * independent product per tile (m, n) of C: gemm C(m,n) <- alpha op(A(m,n))
 * op(B(m,n)) + beta C(m,n); syrk C(m,n) <- alpha op(A(m,n)) op(A(m,n))^T +
 * beta C(m,n) on the uplo triangle of the tile.  C is not read when beta == 0. */
int CHAMELEON_dgemm_batch_Tile(cham_trans_t transA, cham_trans_t transB, double alpha, CHAM_desc_t *A,
                               CHAM_desc_t *B, double beta, CHAM_desc_t *C);
int CHAMELEON_dsyrk_batch_Tile(cham_uplo_t uplo, cham_trans_t trans, double alpha, CHAM_desc_t *A, double beta,
                               CHAM_desc_t *C);
/* compute/zgered.c / pzgered.c:160-260 and pzgerst.c (z -> d): adaptive per-
 * tile precision.  gered rounds each tile of the uplo triangle whose
 * Frobenius norm is small against the matrix's (threshold eps ||A||_F /
 * min(MT, NT), eps = prec or the FP64 unit roundoff when prec < 0) to FP16 or
 * FP32 values and tags it; gerst resets the tags to FP64.  The descriptor
 * keeps its FP64 storage (the reference changes the tile's storage type). */
int CHAMELEON_dgered_Tile(cham_uplo_t uplo, double prec, CHAM_desc_t *A);
int CHAMELEON_dgerst_Tile(cham_uplo_t uplo, CHAM_desc_t *A);
/* The precision tag of tile (m, n): ChamRealDouble, ChamRealFloat or ChamRealHalf. */
int CHAM_B200_Tile_Precision(const CHAM_desc_t *A, int m, int n);
/* Generators: compute/zplgsy.c:276 (pzplgsy.c:29-80), compute/zplrnt.c (pzplrnt.c) */
int CHAMELEON_dplgsy(double bump, cham_uplo_t uplo, int N, double *A, int LDA,
                     unsigned long long int seed);
int CHAMELEON_dplgsy_Tile(double bump, cham_uplo_t uplo, CHAM_desc_t *A,
                          unsigned long long int seed);
int CHAMELEON_dplrnt(int M, int N, double *A, int LDA, unsigned long long int seed);
int CHAMELEON_dplrnt_Tile(CHAM_desc_t *A, unsigned long long int seed);
/* Norms used by the testing checks (compute/zlansy.c, compute/zlange.c) */
double CHAMELEON_dlansy_Tile(cham_normtype_t norm, cham_uplo_t uplo, CHAM_desc_t *A);
double CHAMELEON_dlange_Tile(cham_normtype_t norm, CHAM_desc_t *A);

/* Inverses from the Cholesky factor (compute/ztrtri.c, zlauum.c, zpotri.c:
 * zpotri = pztrtri then pzlauum).  LAPACK semantics: only the uplo triangle of
 * A is read and written; dtrtri returns i > 0 when A(i,i) == 0 (A unchanged);
 * dpotri takes the factor from dpotrf and returns the uplo triangle of A^-1. */
int CHAMELEON_dtrtri(cham_uplo_t uplo, cham_diag_t diag, int N, double *A, int LDA);
int CHAMELEON_dlauum(cham_uplo_t uplo, int N, double *A, int LDA);
int CHAMELEON_dpotri(cham_uplo_t uplo, int N, double *A, int LDA);
int CHAMELEON_dtrtri_Tile(cham_uplo_t uplo, cham_diag_t diag, CHAM_desc_t *A);
/* compute/zpotrimm.c:72,202 (pzpotrimm.c): A (SPD on entry) <- the uplo
 * triangle of A^-1 (potrf, trtri, lauum), then C <- B A^-1; N x N each. */
int CHAMELEON_dpotrimm(cham_uplo_t uplo, int N, double *A, int LDA, double *B, int LDB, double *C, int LDC);
int CHAMELEON_dpotrimm_Tile(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B, CHAM_desc_t *C);
int CHAMELEON_dlauum_Tile(cham_uplo_t uplo, CHAM_desc_t *A);
int CHAMELEON_dpotri_Tile(cham_uplo_t uplo, CHAM_desc_t *A);

/* LAPACKE interface (lapack_api/src/lapack_z{posv,potrf,potrs,potri,lauum,
 * trtri}.c after z->d; include/chameleon/chameleon_zlapack.h:102-119):
 * column-major only (matrix_layout CHAMELEON_LAPACK_COL_MAJOR = CblasColMajor),
 * uplo / diag as LAPACK characters; -1 for another layout. */
#define CHAMELEON_LAPACK_COL_MAJOR 102
int CHAMELEON_lapacke_dposv(int matrix_layout, char uplo, int N, int NRHS, double *A, int lda, double *B, int ldb);
int CHAMELEON_lapacke_dpotrf(int matrix_layout, char uplo, int N, double *A, int lda);
int CHAMELEON_lapacke_dpotrs(int matrix_layout, char uplo, int N, int NRHS, const double *A, int lda, double *B,
                             int ldb);
int CHAMELEON_lapacke_dpotri(int matrix_layout, char uplo, int N, double *A, int lda);
int CHAMELEON_lapacke_dlauum(int matrix_layout, char uplo, int N, double *A, int lda);
int CHAMELEON_lapacke_dtrtri(int matrix_layout, char uplo, char diag, int N, double *A, int lda);
/* Fortran LAPACK interface of the same (lapack_api/src/lapack_zposv.c:25-33
 * and siblings; the reference names them through CMake's Fortran mangling,
 * here the gfortran convention: lower case with a trailing underscore). */
void chameleon_lapack_dposv_(const char *uplo, const int *n, const int *nrhs, double *a, const int *lda, double *b,
                             const int *ldb, int *info);
void chameleon_lapack_dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info);
void chameleon_lapack_dpotrs_(const char *uplo, const int *n, const int *nrhs, const double *a, const int *lda,
                              double *b, const int *ldb, int *info);
void chameleon_lapack_dpotri_(const char *uplo, const int *n, double *a, const int *lda, int *info);
void chameleon_lapack_dlauum_(const char *uplo, const int *n, double *a, const int *lda, int *info);
void chameleon_lapack_dtrtri_(const char *uplo, const char *diag, const int *n, double *a, const int *lda, int *info);

/* ------------------------------------------------------------------------- */
/* Mixed precision (new; in the spirit of the reference's commented-out      */
/* zcposv, include/chameleon/chameleon_zc.h:33-42, and LAPACK dsposv)         */
/* ------------------------------------------------------------------------- */
typedef struct cham_b200_refine_info_s {
    int    iterations;      /* refinement iterations taken (0: direct FP64) */
    int    fallback;        /* 1 when refinement stalled and FP64 was used  */
    int    precision;       /* CHAM_B200_PREC_* of the factorization used   */
    double backward_error;  /* max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf) */
    double seconds;         /* device time of the whole solve               */
} CHAM_b200_refine_info_t;

/* A is FP64 and is not overwritten unless refinement fails (then, as in
 * LAPACK dsposv, A holds the FP64 factor and ITER < 0); X receives the
 * solution of A X = B.  ITER: iterations used (>= 0), -2 cast overflow, -3
 * low-precision factorization failed, -(maxiter+1) no convergence. */
int CHAMELEON_dsposv(cham_uplo_t uplo, int N, int NRHS, double *A, int LDA, double *B, int LDB, double *X,
                     int LDX, int *ITER);
int CHAMELEON_dsposv_Tile(cham_uplo_t uplo, CHAM_desc_t *A, CHAM_desc_t *B, CHAM_desc_t *X,
                          int *iter);
int CHAMELEON_B200_dposv_mixed_Tile(cham_uplo_t uplo, int precision, CHAM_desc_t *A,
                                    CHAM_desc_t *B, CHAM_desc_t *X,
                                    CHAM_b200_refine_info_t *info);

/* ------------------------------------------------------------------------- */
/* GPU tile-kernel ABI (gpucublas/include/gpucublas/gpucublas_z.h:36-61,      */
/* gpucublas_zc.h:22-23 after z->d / zc->ds generation).  The cuBLAS and      */
/* cuSOLVER handle types are opaque handles of this library carrying the      */
/* stream; no cuBLAS or cuSOLVER is linked.                                   */
/* ------------------------------------------------------------------------- */
typedef struct cham_b200_handle_s *cublasHandle_t;
typedef struct cham_b200_handle_s *cusolverDnHandle_t;
int CHAM_B200_Handle_Create(cublasHandle_t *handle, void *cuda_stream);
int CHAM_B200_Handle_Destroy(cublasHandle_t handle);

int CUDA_dgemm(cham_trans_t transa, cham_trans_t transb, int m, int n, int k,
               const double *alpha, const double *A, int lda, const double *B, int ldb,
               const double *beta, double *C, int ldc, cublasHandle_t handle);
int CUDA_dsyrk(cham_uplo_t uplo, cham_trans_t trans, int n, int k, const double *alpha,
               const double *A, int lda, const double *beta, double *C, int ldc,
               cublasHandle_t handle);
int CUDA_dtrsm(cham_side_t side, cham_uplo_t uplo, cham_trans_t transa, cham_diag_t diag,
               int m, int n, const double *alpha, const double *A, int lda, double *B, int ldb,
               cublasHandle_t handle);
/* d_info: device int receiving LAPACK's info; WORK/lwork are accepted and unused */
int CUDA_dpotrf(cham_uplo_t uplo, int n, double *A, int lda, double *WORK, int lwork,
                int *d_info, cusolverDnHandle_t handle);
/* gpucublas_z.h:54 after z->s generation: FP32 tile Cholesky (the mixed
 * solver's diagonal-tile kernel); d_info as CUDA_dpotrf */
int CUDA_spotrf(cham_uplo_t uplo, int n, float *A, int lda, float *WORK, int lwork,
                int *d_info, cusolverDnHandle_t handle);
/* No counterpart in the reference.  CUDA_dpotrf without any device
 * allocation, for callers that cannot allocate: a task runtime that owns the
 * device memory and forbids allocation inside its worker callbacks (StarPU
 * codelets, for instance), or latency-critical code that must not wait on
 * cudaMalloc.  Its scratch is one fixed 512 KiB array in the library's device
 * memory, so n <= 1024 (larger n returns CHAMELEON_ERR_INTERNAL_LIMIT); all
 * calls on a device share that array, so calls that could overlap on the GPU
 * must not be issued.  The first call on a device does a one-time set-up and
 * should come before any stream capture.  Same result and `info` as CUDA_dpotrf. */
int CUDA_dpotrf_noalloc(cham_uplo_t uplo, int n, double *A, int lda, int *d_info, void *cuda_stream);
int CUDA_dplgsy(const double *bump, int m, int n, double *A, int lda, int bigM, int m0, int n0,
                unsigned long long int seed, cublasHandle_t handle);
int CUDA_dplrnt(int m, int n, double *A, int lda, int bigM, int m0, int n0,
                unsigned long long int seed, cublasHandle_t handle);
int CUDA_dlag2s(int m, int n, const double *A, int lda, float *SA, int ldsa,
                cublasHandle_t handle);
int CUDA_slag2d(int m, int n, const float *SA, int ldsa, double *A, int lda,
                cublasHandle_t handle);

/* Tile forms of the kernels above (gpucublas/include/gpucublas/gpucublas_ztile.h
 * :30,46-48,51,55 and gpucublas_zctile.h:22-23 after z->d / zc->ds
 * generation): the operands are CHAM_tile_t (device address + leading
 * dimension), as the runtimes' codelets pass them.  Full-rank tiles only
 * (format CHAMELEON_TILE_FULLRANK); other formats return
 * CHAMELEON_ERR_NOT_SUPPORTED.  Formats: include/chameleon/struct.h:37-39. */
#define CHAMELEON_TILE_FULLRANK (1 << 0)
#define CHAMELEON_TILE_DESC     (1 << 1)
#define CHAMELEON_TILE_HMAT     (1 << 2)
int TCUDA_dgemm(cham_trans_t transA, cham_trans_t transB, int m, int n, int k, const double *alpha,
                const CHAM_tile_t *A, const CHAM_tile_t *B, const double *beta, CHAM_tile_t *C,
                cublasHandle_t handle);
int TCUDA_dsyrk(cham_uplo_t uplo, cham_trans_t trans, int n, int k, const double *alpha, const CHAM_tile_t *A,
                const double *beta, CHAM_tile_t *C, cublasHandle_t handle);
int TCUDA_dtrsm(cham_side_t side, cham_uplo_t uplo, cham_trans_t transA, cham_diag_t diag, int m, int n,
                const double *alpha, const CHAM_tile_t *A, CHAM_tile_t *B, cublasHandle_t handle);
int TCUDA_dpotrf(cham_uplo_t uplo, int n, CHAM_tile_t *A, double *WORK, int lwork, int *d_info,
                 cusolverDnHandle_t handle);
int TCUDA_dplgsy(const double *bump, int m, int n, CHAM_tile_t *A, int bigM, int m0, int n0,
                 unsigned long long int seed, cublasHandle_t handle);
int TCUDA_dplrnt(int m, int n, CHAM_tile_t *A, int bigM, int m0, int n0, unsigned long long int seed,
                 cublasHandle_t handle);
int TCUDA_dlag2s(int m, int n, const CHAM_tile_t *A, CHAM_tile_t *B, cublasHandle_t handle);
int TCUDA_slag2d(int m, int n, const CHAM_tile_t *A, CHAM_tile_t *B, cublasHandle_t handle);

/* ------------------------------------------------------------------------- */
/* Recorded tile DAGs: the runtime-plugin boundary of the reference           */
/* (include/chameleon/tasks_z.h:64-380 INSERT_TASK_*, include/chameleon/      */
/* runtime.h:51-714 RUNTIME_*).  A Chameleon runtime plugin (runtime/b200,    */
/* chameleon_b200/runtime/runtime_b200.c) appends one record per INSERT_TASK  */
/* call of chameleon_pdpotrf / chameleon_pdtrsm (compute/pzpotrf.c:84-194,    */
/* compute/pztrsm.c:58-200, unchanged) and runs the DAG at                    */
/* RUNTIME_sequence_wait.  Records (kind, m, n, k, bn):                       */
/*   POTRF (k, k, k, 0): factor diagonal tile k of A                          */
/*   PANEL (m, k, k, 0): A(m,k) <- A(m,k) L(k,k)^-T                            */
/*   UPDATE (m, n, k, 0): A(m,n) -= A(m,k) A(n,k)^T, m >= n > k (SYRK if m == n)*/
/*   FWD_SOLVE (k, k, k, bn) / BWD_SOLVE: B(k,bn) <- L(k,k)^-1 / ^-T B(k,bn)    */
/*   FWD_UPDATE (m, k, k, bn): B(m,bn) -= L(m,k) B(k,bn), m > k                 */
/*   BWD_UPDATE (m, k, k, bn): B(m,bn) -= L(k,m)^T B(k,bn), m < k               */
/* with tiles of the logical lower triangle (Upper storage: transposed views).*/
/* ------------------------------------------------------------------------- */
#define CHAM_B200_DAG_POTRF      1
#define CHAM_B200_DAG_PANEL      2
#define CHAM_B200_DAG_UPDATE     3
#define CHAM_B200_DAG_FWD_SOLVE  4
#define CHAM_B200_DAG_FWD_UPDATE 5
#define CHAM_B200_DAG_BWD_SOLVE  6
#define CHAM_B200_DAG_BWD_UPDATE 7
typedef struct cham_b200_dag_s *CHAM_b200_dag_t;
int CHAM_B200_Dag_Create(CHAM_b200_dag_t *dag);
int CHAM_B200_Dag_Destroy(CHAM_b200_dag_t dag);
int CHAM_B200_Dag_Clear(CHAM_b200_dag_t dag);
int CHAM_B200_Dag_Record(CHAM_b200_dag_t dag, int kind, int m, int n, int k, int bn);
int CHAM_B200_Dag_Size(CHAM_b200_dag_t dag);
/* the records, 5 ints each, in submission order; returns the count written */
int CHAM_B200_Dag_Get(CHAM_b200_dag_t dag, int *out, int cap);
/* The executor's task list for the recorded DAG (16-byte tasks, as
 * CHAM_B200_Schedule_Build); returns its length, or CHAMELEON_ERR_NOT_SUPPORTED
 * when the executor cannot run the records in their submission order. */
int CHAM_B200_Dag_Schedule(CHAM_b200_dag_t dag, int N, int NB, int nrhs, int NBB, int workers, void *out,
                           int cap);
/* Run the recorded DAG (FP64) on A (order N, NB x NB tiles at A + a_off[m +
 * NT n], leading dimension a_ld[m]; device memory) and B (N x nrhs, NB x NBB
 * tiles likewise; may be NULL with nrhs == 0).  Synchronous; *info receives
 * LAPACK's info of the factorization. */
int CHAM_B200_Dag_Run(CHAM_b200_dag_t dag, cham_uplo_t uplo, int N, int NB, double *A, const int64_t *a_off,
                      const int *a_ld, int nrhs, int NBB, double *B, const int64_t *b_off, const int *b_ld,
                      int *info);
/* CHAMELEON_Init of this library under a name of its own (for runtime plugins
 * linked into a Chameleon build, whose own CHAMELEON_Init is the reference's) */
int CHAM_B200_Init(void);

/* ------------------------------------------------------------------------- */
/* Uneven batch (new; the reference batch API is uniform-size,                */
/* compute/zpotrf_batch.c:66-118).  Matrix i is n[i] x n[i] column-major at   */
/* A + a_off[i] (ld = n[i]); its right-hand sides are n[i] x nrhs[i] at        */
/* B + b_off[i] (ld = n[i]), overwritten by the solution.  All arrays are      */
/* device arrays; info[i] receives the LAPACK info of matrix i.               */
/* ------------------------------------------------------------------------- */
int CHAM_B200_dposv_batch(cham_uplo_t uplo, int count, const int *n, const int *nrhs,
                          double *A, const int64_t *a_off, double *B, const int64_t *b_off,
                          int *info, void *cuda_stream);
/* The same for FP32 systems (FP32 storage and arithmetic). */
int CHAM_B200_sposv_batch(cham_uplo_t uplo, int count, const int *n, const int *nrhs,
                          float *A, const int64_t *a_off, float *B, const int64_t *b_off,
                          int *info, void *cuda_stream);

/* ------------------------------------------------------------------------- */
/* Serving loop (new; the reference solves one system per call).  A server    */
/* owns worker threads and CUDA streams; host threads submit solve requests  */
/* of any order and right-hand-side count and read the results when          */
/* `status` leaves CHAM_B200_REQ_PENDING (or after Serve_Drain).  Small      */
/* systems (N <= small_n) are coalesced into one batched launch per wave of   */
/* arrivals; larger ones run the mixed-precision solver (FP64-accurate) on    */
/* one of `slots` streams.  A request is admitted when its device memory      */
/* fits in the HBM budget (0: 80% of the free memory at creation).           */
/* ------------------------------------------------------------------------- */
#define CHAM_B200_REQ_PENDING (1 << 30)
typedef struct cham_b200_server_s *CHAM_b200_server_t;
typedef struct cham_b200_request_s {
    /* in: column-major host arrays (pinned memory gives asynchronous copies) */
    int N, nrhs;
    int uplo;                   /* ChamLower / ChamUpper: triangle of A read     */
    const double *A; int lda;   /* NULL: solve with the factor kept under key   */
    const double *B; int ldb;   /* N x nrhs                                       */
    double *X;       int ldx;   /* N x nrhs, written on completion               */
    long long factor_key;       /* >= 0 with A: keep the factor under this key
                                   (replaces an older one); >= 0 without A: use
                                   it; < 0: nothing kept                          */
    /* out */
    int status;                 /* PENDING, then 0, > 0 (leading minor not
                                   positive definite) or CHAMELEON_ERR_*;
                                   CHAMELEON_ERR_NOT_FOUND: no factor under key  */
    int iterations;             /* refinement iterations (dsposv ITER; 0 for the
                                   FP64 batched path)                             */
    double t_submit, t_start, t_done;   /* CHAM_B200_Serve_Now() clock          */
} CHAM_b200_request_t;
typedef struct cham_b200_serve_stats_s {
    long long completed, batches, batched_requests, max_batch;
    long long reused_factors, kept_factors;
    double bytes_in_use, budget_bytes;
} CHAM_b200_serve_stats_t;
int    CHAM_B200_Serve_Create(CHAM_b200_server_t *server, int slots, double hbm_budget_bytes, int small_n);
/* The request and its arrays must stay valid until it completes. */
int    CHAM_B200_Serve_Submit(CHAM_b200_server_t server, CHAM_b200_request_t *request);
int    CHAM_B200_Serve_Drain(CHAM_b200_server_t server);       /* wait for all submitted */
int    CHAM_B200_Serve_Stats(CHAM_b200_server_t server, CHAM_b200_serve_stats_t *stats);
int    CHAM_B200_Serve_Destroy(CHAM_b200_server_t server);     /* drains first          */
double CHAM_B200_Serve_Now(void);

/* ------------------------------------------------------------------------- */
/* Multi-GPU dispatch of independent systems (new; host planning only, no    */
/* device call).  Batches and serving requests shard over the GPUs of a node  */
/* with no collective: the plan says which GPU solves which system.          */
/* ------------------------------------------------------------------------- */
/* Estimated device seconds / device bytes of one system of order n with nrhs
 * right-hand sides inside a batch or serving wave. */
double CHAM_B200_Dispatch_Cost(int n, int nrhs);
double CHAM_B200_Dispatch_Bytes(int n, int nrhs);
/* Longest-first list schedule of `count` systems over `nranks` GPUs: owner[i]
 * = the GPU of system i (pin[i] >= 0 forces a live GPU; pin may be NULL),
 * only GPUs with alive[r] != 0, each GPU's systems of one wave fitting in
 * free_bytes[r]; load_s[r] (may be NULL) = seconds of work the GPU already
 * has; wave[i] (may be NULL) = the wave of system i.  Returns the number of
 * waves, CHAMELEON_ERR_OUT_OF_RESOURCES when a system fits on no live GPU,
 * CHAMELEON_ERR_NOT_INITIALIZED when no GPU is alive. */
int CHAM_B200_Dispatch_Plan(int count, const int *n, const int *nrhs, const int *pin, int nranks,
                            const int *alive, const double *free_bytes, const double *load_s, int *owner,
                            int *wave);

#ifdef __cplusplus
}
#endif
#endif /* CHAMELEON_B200_H */
