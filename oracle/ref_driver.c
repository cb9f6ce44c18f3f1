/*
 * Thin C driver around the reference's own library (oracle/_ref/libchamref.so).
 *
 * Test infrastructure only.  The reference's OpenMP runtime submits tasks from
 * inside the `omp parallel` / `omp master` region that its CHAMELEON_Init macro
 * opens (include/chameleon.h:255-276); ctypes cannot open such a region, so
 * each entry point here opens it around one reference call.  Timing follows
 * testing_start/testing_stop (testing/testings.c:125-223): wall time around the
 * call only.
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>
#include "chameleon.h"
#include "chameleon/timer.h"

static int g_ncores = 0;

int chamref_init(int ncores)
{
    if (g_ncores) return 0;
    g_ncores = ncores > 0 ? ncores : omp_get_num_procs();
    int rc = __chameleon_init(g_ncores, 0);
    CHAMELEON_Disable(CHAMELEON_WARNINGS);
    return rc;
}

int chamref_ncores(void) { return g_ncores; }

void chamref_finalize(void)
{
    if (!g_ncores) return;
    __chameleon_finalize();
    g_ncores = 0;
}

static double now(void) { return omp_get_wtime(); }

/* LAPACK-layout generator: CHAMELEON_dplgsy (compute/zplgsy.c). */
int chamref_dplgsy(double bump, int uplo, int N, double *A, int lda, int nb,
                   unsigned long long seed)
{
    int rc = 0;
    CHAMELEON_Set(CHAMELEON_TILE_SIZE, nb);
#pragma omp parallel
#pragma omp master
    rc = CHAMELEON_dplgsy(bump, (cham_uplo_t)uplo, N, A, lda, seed);
    return rc;
}

/* LAPACK-layout generator: CHAMELEON_dplrnt (compute/zplrnt.c). */
int chamref_dplrnt(int M, int N, double *A, int lda, int nb, unsigned long long seed)
{
    int rc = 0;
    CHAMELEON_Set(CHAMELEON_TILE_SIZE, nb);
#pragma omp parallel
#pragma omp master
    rc = CHAMELEON_dplrnt(M, N, A, lda, seed);
    return rc;
}

/* CHAMELEON_dposv (compute/zposv.c:93) on caller arrays. */
int chamref_dposv(int uplo, int N, int nrhs, int nb, double *A, int lda,
                  double *B, int ldb, double *seconds)
{
    int rc = 0;
    double t0 = 0, t1 = 0;
    CHAMELEON_Set(CHAMELEON_TILE_SIZE, nb);
#pragma omp parallel
#pragma omp master
    {
        t0 = now();
        rc = CHAMELEON_dposv((cham_uplo_t)uplo, N, nrhs, A, lda, B, ldb);
        t1 = now();
    }
    if (seconds) *seconds = t1 - t0;
    return rc;
}

int chamref_dpotrf(int uplo, int N, int nb, double *A, int lda, double *seconds)
{
    int rc = 0;
    double t0 = 0, t1 = 0;
    CHAMELEON_Set(CHAMELEON_TILE_SIZE, nb);
#pragma omp parallel
#pragma omp master
    {
        t0 = now();
        rc = CHAMELEON_dpotrf((cham_uplo_t)uplo, N, A, lda);
        t1 = now();
    }
    if (seconds) *seconds = t1 - t0;
    return rc;
}

int chamref_dpotrs(int uplo, int N, int nrhs, int nb, double *A, int lda,
                   double *B, int ldb)
{
    int rc = 0;
    CHAMELEON_Set(CHAMELEON_TILE_SIZE, nb);
#pragma omp parallel
#pragma omp master
    rc = CHAMELEON_dpotrs((cham_uplo_t)uplo, N, nrhs, A, lda, B, ldb);
    return rc;
}

/* CHAMELEON_dpotri / dtrtri / dlauum (compute/zpotri.c, ztrtri.c, zlauum.c)
 * on caller arrays: op 0 = potri, 1 = trtri, 2 = lauum. */
int chamref_dinverse(int op, int uplo, int diag, int N, int nb, double *A, int lda)
{
    int rc = 0;
    CHAMELEON_Set(CHAMELEON_TILE_SIZE, nb);
#pragma omp parallel
#pragma omp master
    {
        if (op == 0)
            rc = CHAMELEON_dpotri((cham_uplo_t)uplo, N, A, lda);
        else if (op == 1)
            rc = CHAMELEON_dtrtri((cham_uplo_t)uplo, (cham_diag_t)diag, N, A, lda);
        else
            rc = CHAMELEON_dlauum((cham_uplo_t)uplo, N, A, lda);
    }
    return rc;
}

/*
 * The testing driver's descriptor path (testing/testing_zposv.c:40-109):
 * tile-allocated descriptors, A from dplgsy(bump = N, uplo, seedA) (only the
 * uplo triangle), B from dplrnt(seedB), timed dposv_Tile.  Outputs (optional)
 * are the factor (uplo triangle, column-major N x N) and the solution.
 */
int chamref_dposv_tile_seeded(int uplo, int N, int nrhs, int nb,
                              unsigned long long seedA, unsigned long long seedB,
                              double *Aout, double *Xout, double *seconds)
{
    CHAM_desc_t *descA = NULL, *descX = NULL;
    int rc = 0;
    double t0 = 0, t1 = 0;
    rc = CHAMELEON_Desc_Create(&descA, CHAMELEON_MAT_ALLOC_TILE, ChamRealDouble, nb, nb, nb * nb,
                               N, N, 0, 0, N, N, 1, 1);
    if (rc) return rc;
    rc = CHAMELEON_Desc_Create(&descX, CHAMELEON_MAT_ALLOC_TILE, ChamRealDouble, nb, nb, nb * nb,
                               N, nrhs, 0, 0, N, nrhs, 1, 1);
    if (rc) { CHAMELEON_Desc_Destroy(&descA); return rc; }
#pragma omp parallel
#pragma omp master
    {
        CHAMELEON_dplgsy_Tile((double)N, (cham_uplo_t)uplo, descA, seedA);
        CHAMELEON_dplrnt_Tile(descX, seedB);
        t0 = now();
        rc = CHAMELEON_dposv_Tile((cham_uplo_t)uplo, descA, descX);
        t1 = now();
        if (Aout) CHAMELEON_Desc2Lap((cham_uplo_t)uplo, descA, Aout, N);
        if (Xout) CHAMELEON_Desc2Lap(ChamUpperLower, descX, Xout, N);
    }
    if (seconds) *seconds = t1 - t0;
    CHAMELEON_Desc_Destroy(&descA);
    CHAMELEON_Desc_Destroy(&descX);
    return rc;
}

/*
 * CHAMELEON_dpotrf_batch_Tile (compute/zpotrf_batch.c:89) over `count` n x n
 * matrices stacked in one column-major (count*n) x n array: a caller matrix
 * is a column-major view (control/descriptor.c:183-199), and with mb = nb = n
 * its tiles A(i,0) are the stacked matrices.
 */
int chamref_dpotrf_batch(int uplo, int n, int count, double *mats, double *seconds)
{
    CHAM_desc_t *descA = NULL;
    int rc;
    double t0 = 0, t1 = 0;
    rc = CHAMELEON_Desc_Create(&descA, mats, ChamRealDouble, n, n, n * n,
                               count * n, n, 0, 0, count * n, n, 1, 1);
    if (rc) return rc;
#pragma omp parallel
#pragma omp master
    {
        t0 = now();
        rc = CHAMELEON_dpotrf_batch_Tile((cham_uplo_t)uplo, descA);
        t1 = now();
    }
    if (seconds) *seconds = t1 - t0;
    CHAMELEON_Desc_Destroy(&descA);
    return rc;
}

/* CHAMELEON_dtrsm_batch_Tile (compute/ztrsm_batch.c:180): stacked column-major
 * A ((count*an) x an) and B ((count*bm) x bn); tile i of B is solved with
 * tile i of A. */
int chamref_dtrsm_batch(int side, int uplo, int trans, int diag, double alpha,
                        int n, int nrhs, int count, double *A, double *B)
{
    CHAM_desc_t *descA = NULL, *descB = NULL;
    int rc;
    int an = (side == ChamLeft) ? n : nrhs;
    int bm = (side == ChamLeft) ? n : nrhs;
    int bn = (side == ChamLeft) ? nrhs : n;
    rc = CHAMELEON_Desc_Create(&descA, A, ChamRealDouble, an, an, an * an,
                               count * an, an, 0, 0, count * an, an, 1, 1);
    if (rc) return rc;
    rc = CHAMELEON_Desc_Create(&descB, B, ChamRealDouble, bm, bn, bm * bn,
                               count * bm, bn, 0, 0, count * bm, bn, 1, 1);
    if (rc) { CHAMELEON_Desc_Destroy(&descA); return rc; }
#pragma omp parallel
#pragma omp master
    rc = CHAMELEON_dtrsm_batch_Tile((cham_side_t)side, (cham_uplo_t)uplo, (cham_trans_t)trans,
                                    (cham_diag_t)diag, alpha, descA, descB);
    CHAMELEON_Desc_Destroy(&descA);
    CHAMELEON_Desc_Destroy(&descB);
    return rc;
}

/* CHAMELEON_dpotrimm (compute/zpotrimm.c:72) on caller arrays. */
int chamref_dpotrimm(int uplo, int N, int nb, double *A, int lda, double *B, int ldb, double *C, int ldc)
{
    int rc = 0;
    CHAMELEON_Set(CHAMELEON_TILE_SIZE, nb);
#pragma omp parallel
#pragma omp master
    rc = CHAMELEON_dpotrimm((cham_uplo_t)uplo, N, A, lda, B, ldb, C, ldc);
    return rc;
}

/* CHAMELEON_dgemm_batch_Tile / dsyrk_batch_Tile (compute/zgemm_batch.c:193,
 * zherk_batch.c:176): `count` tiles stacked in one tile column of a
 * column-major (count am) x an array (likewise B: bm x bn, C: m x n tiles). */
int chamref_dgemm_batch(int transA, int transB, double alpha, double beta, int am, int an, int bm, int bn,
                        int m, int n, int count, double *A, double *B, double *C)
{
    CHAM_desc_t *dA = NULL, *dB = NULL, *dC = NULL;
    int rc = CHAMELEON_Desc_Create(&dA, A, ChamRealDouble, am, an, am * an, count * am, an, 0, 0, count * am, an, 1, 1);
    if (!rc) rc = CHAMELEON_Desc_Create(&dB, B, ChamRealDouble, bm, bn, bm * bn, count * bm, bn, 0, 0, count * bm, bn, 1, 1);
    if (!rc) rc = CHAMELEON_Desc_Create(&dC, C, ChamRealDouble, m, n, m * n, count * m, n, 0, 0, count * m, n, 1, 1);
    if (!rc) {
#pragma omp parallel
#pragma omp master
        rc = CHAMELEON_dgemm_batch_Tile((cham_trans_t)transA, (cham_trans_t)transB, alpha, dA, dB, beta, dC);
    }
    if (dA) CHAMELEON_Desc_Destroy(&dA);
    if (dB) CHAMELEON_Desc_Destroy(&dB);
    if (dC) CHAMELEON_Desc_Destroy(&dC);
    return rc;
}

int chamref_dsyrk_batch(int uplo, int trans, double alpha, double beta, int am, int an, int n, int count,
                        double *A, double *C)
{
    CHAM_desc_t *dA = NULL, *dC = NULL;
    int rc = CHAMELEON_Desc_Create(&dA, A, ChamRealDouble, am, an, am * an, count * am, an, 0, 0, count * am, an, 1, 1);
    if (!rc) rc = CHAMELEON_Desc_Create(&dC, C, ChamRealDouble, n, n, n * n, count * n, n, 0, 0, count * n, n, 1, 1);
    if (!rc) {
#pragma omp parallel
#pragma omp master
        rc = CHAMELEON_dsyrk_batch_Tile((cham_uplo_t)uplo, (cham_trans_t)trans, alpha, dA, beta, dC);
    }
    if (dA) CHAMELEON_Desc_Destroy(&dA);
    if (dC) CHAMELEON_Desc_Destroy(&dC);
    return rc;
}

/* LAPACKE_dsposv from the same OpenBLAS: the CPU mixed-precision comparator. */
extern int scipy_LAPACKE_dsposv(int layout, char uplo, int n, int nrhs, double *a, int lda,
                                double *b, int ldb, double *x, int ldx, int *iter);
int chamref_lapacke_dsposv(int uplo, int N, int nrhs, double *A, int lda, double *B, int ldb,
                           double *X, int ldx, int *iter, double *seconds)
{
    double t0 = now();
    int rc = scipy_LAPACKE_dsposv(102 /* col major */, uplo == ChamUpper ? 'U' : 'L', N, nrhs,
                                  A, lda, B, ldb, X, ldx, iter);
    if (seconds) *seconds = now() - t0;
    return rc;
}
