/*
 * plugin_harness.c -- test driver of the B200 runtime plugin (test
 * infrastructure): the reference's own public API (CHAMELEON_Init,
 * CHAMELEON_Desc_Create, CHAMELEON_dposv_Tile -- compute/zposv.c:222-245,
 * which runs chameleon_pdpotrf and two chameleon_pdtrsm) linked with
 * chameleon_b200/runtime/runtime_b200.c instead of a StarPU/OpenMP runtime.
 * Built by oracle/build_plugin.sh into oracle/_ref/libchamb200rt.so.
 */
#include "control/common.h"

#include <string.h>

int chameleon_b200_runtime_record_only(int on);
int chameleon_b200_runtime_last_dag(int *out, int cap);

/* Copy between a column-major array (ld) and the tiles of a descriptor. */
static void lap_to_tiles(const double *A, int lda, CHAM_desc_t *d, int to_tiles) {
    for (int n = 0; n < d->nt; ++n)
        for (int m = 0; m < d->mt; ++m) {
            double *t = (double *)d->get_blkaddr(d, m, n);
            const int ld = d->get_blkldd(d, m);
            const int rows = (m == d->mt - 1) ? d->m - m * d->mb : d->mb;
            const int cols = (n == d->nt - 1) ? d->n - n * d->nb : d->nb;
            for (int j = 0; j < cols; ++j)
                for (int i = 0; i < rows; ++i) {
                    double *a = (double *)A + (size_t)(m * d->mb + i) + (size_t)(n * d->nb + j) * lda;
                    if (to_tiles) t[i + (size_t)j * ld] = *a;
                    else *a = t[i + (size_t)j * ld];
                }
        }
}

/* One CHAMELEON_dposv_Tile through the plugin.  A (N x N, lda) and B (N x nrhs,
 * ldb) are column-major host arrays (NULL: leave the tiles unset, for
 * record-only runs); on return A holds the factor, B the solution.
 * record_only: keep the recorded DAG instead of running it; the records (5
 * ints each) go to dag (capacity cap), their count to *ndag.  Returns the
 * CHAMELEON_dposv_Tile return code. */
int harness_posv(int uplo, int N, int NB, int nrhs, double *A, int lda, double *B, int ldb, int record_only,
                 int *dag, int cap, int *ndag) {
    chameleon_b200_runtime_record_only(record_only);
    int rc = CHAMELEON_Init(1, 1);
    if (rc) return rc;
    CHAMELEON_Set(CHAMELEON_TILE_SIZE, NB);
    CHAM_desc_t *dA = NULL, *dB = NULL;
    rc = CHAMELEON_Desc_Create(&dA, CHAMELEON_MAT_ALLOC_TILE, ChamRealDouble, NB, NB, NB * NB, N, N, 0, 0, N, N, 1, 1);
    if (!rc)
        rc = CHAMELEON_Desc_Create(&dB, CHAMELEON_MAT_ALLOC_TILE, ChamRealDouble, NB, NB, NB * NB, N, nrhs, 0, 0, N,
                                   nrhs, 1, 1);
    if (!rc && A) lap_to_tiles(A, lda, dA, 1);
    if (!rc && B) lap_to_tiles(B, ldb, dB, 1);
    if (!rc) rc = CHAMELEON_dposv_Tile((cham_uplo_t)uplo, dA, dB);
    if (ndag) *ndag = chameleon_b200_runtime_last_dag(dag, cap);
    if (!record_only) {
        CHAMELEON_Desc_Acquire(dA);
        CHAMELEON_Desc_Acquire(dB);
        if (A) lap_to_tiles(A, lda, dA, 0);
        if (B) lap_to_tiles(B, ldb, dB, 0);
    }
    if (dA) CHAMELEON_Desc_Destroy(&dA);
    if (dB) CHAMELEON_Desc_Destroy(&dB);
    CHAMELEON_Finalize();
    return rc;
}
