/*
 * cham_oracle.c -- CPU restatement of the reference's dposv path.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * bench's CPU baseline as the checker; the product never links it.
 *
 * Parity is pinned two ways: (1) the generators are bit-exact against the
 * reference's own build (oracle/_ref/libchamref.so, built from the reference
 * sources by oracle/build_ref.sh) and against the known-answer values committed
 * in tests/golden/; (2) the factorization and solve are checked with the
 * reference's own residual tests (threshold 60) and compared element-wise, within
 * tolerance, with the reference library's dposv on the same inputs.
 *
 * Each function cites the reference code it restates.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_UPPER 121
#define ORC_LOWER 122

/* coreblas/include/coreblas/random.h:32-56 -- LCG skip-ahead. */
unsigned long long orc_lcg_skip(unsigned long long n, unsigned long long x)
{
    unsigned long long a = 6364136223846793005ULL, c = 1ULL;
    while (n) {
        if (n & 1ULL) x = a * x + c;
        c *= (a + 1ULL);
        a *= a;
        n >>= 1;
    }
    return x;
}

/* random.h:66-73 CORE_dlaran: value of a state, then advance. */
static double orc_laran(unsigned long long *x)
{
    double v = 0.5 - (double)(*x) * 5.4210108624275222e-20;
    *x = 6364136223846793005ULL * (*x) + 1ULL;
    return v;
}

/*
 * coreblas/compute/core_zplgsy.c:38-112 (d precision, NBELEM = 1) applied to the
 * whole matrix: element (i,j), i >= j, takes state i + j*bigM; the upper
 * triangle mirrors the lower; bump is added on the diagonal.  Column j of the
 * lower triangle is one sequential run of the stream starting at state
 * j + j*bigM, exactly as the reference walks it.
 */
void orc_dplgsy(double bump, int N, double *A, int lda, int bigM, int m0, int n0,
                unsigned long long seed)
{
    for (int j = 0; j < N; ++j) {
        unsigned long long x = orc_lcg_skip((unsigned long long)(m0 + j) +
                                            (unsigned long long)(n0 + j) * (unsigned long long)bigM, seed);
        for (int i = j; i < N; ++i) {
            double v = orc_laran(&x);
            A[i + (int64_t)j * lda] = v;
            A[j + (int64_t)i * lda] = v;
        }
        A[j + (int64_t)j * lda] += bump;
    }
}

/* coreblas/compute/core_zplrnt.c:38-54: element (i,j) takes state i + j*bigM. */
void orc_dplrnt(int M, int N, double *A, int lda, int bigM, int m0, int n0, unsigned long long seed)
{
    for (int j = 0; j < N; ++j) {
        unsigned long long x = orc_lcg_skip((unsigned long long)m0 +
                                            (unsigned long long)(n0 + j) * (unsigned long long)bigM, seed);
        for (int i = 0; i < M; ++i) A[i + (int64_t)j * lda] = orc_laran(&x);
    }
}

/* ---- naive tile kernels (the BLAS/LAPACK calls of coreblas) --------------- */
#define AT(p, ld, i, j) (p)[(i) + (int64_t)(j) * (ld)]

/* LAPACK dpotrf semantics (coreblas/compute/core_zpotrf.c:75-81). */
static int k_potrf(int uplo, int n, double *A, int lda)
{
    for (int j = 0; j < n; ++j) {
        double d = (uplo == ORC_LOWER) ? AT(A, lda, j, j) : AT(A, lda, j, j);
        for (int k = 0; k < j; ++k) {
            double l = (uplo == ORC_LOWER) ? AT(A, lda, j, k) : AT(A, lda, k, j);
            d -= l * l;
        }
        if (!(d > 0.0)) return j + 1;
        d = sqrt(d);
        AT(A, lda, j, j) = d;
        for (int i = j + 1; i < n; ++i) {
            double s = (uplo == ORC_LOWER) ? AT(A, lda, i, j) : AT(A, lda, j, i);
            for (int k = 0; k < j; ++k) {
                if (uplo == ORC_LOWER) s -= AT(A, lda, i, k) * AT(A, lda, j, k);
                else s -= AT(A, lda, k, i) * AT(A, lda, k, j);
            }
            if (uplo == ORC_LOWER) AT(A, lda, i, j) = s / d;
            else AT(A, lda, j, i) = s / d;
        }
    }
    return 0;
}

/* element (i,j) of op(X), op = T when t != 0 */
static inline double opel(const double *X, int ld, int t, int i, int j)
{
    return t ? AT(X, ld, j, i) : AT(X, ld, i, j);
}

/* C(m x n) -= op(A)(m x k) * op(B)(k x n) */
static void k_gemm_sub(int ta, int tb, int m, int n, int k, const double *A, int lda, const double *B, int ldb,
                       double *C, int ldc)
{
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double s = 0.0;
            for (int l = 0; l < k; ++l) s += opel(A, lda, ta, i, l) * opel(B, ldb, tb, l, j);
            AT(C, ldc, i, j) -= s;
        }
}

/* Lower triangle of C (n x n) -= op(A) op(A)^T; upper when uplo == Upper. */
static void k_syrk_sub(int uplo, int ta, int n, int k, const double *A, int lda, double *C, int ldc)
{
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            if ((uplo == ORC_LOWER && i < j) || (uplo == ORC_UPPER && i > j)) continue;
            double s = 0.0;
            for (int l = 0; l < k; ++l) s += opel(A, lda, ta, i, l) * opel(A, lda, ta, j, l);
            AT(C, ldc, i, j) -= s;
        }
}

/* B(m x n) <- B * L^{-T}, L lower n x n (Right/Lower/Trans/NonUnit) */
static void k_trsm_rlt(int m, int n, const double *L, int ldl, double *B, int ldb)
{
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            double s = AT(B, ldb, i, j);
            for (int k = 0; k < j; ++k) s -= AT(B, ldb, i, k) * AT(L, ldl, j, k);
            AT(B, ldb, i, j) = s / AT(L, ldl, j, j);
        }
}

/* B(m x n) <- U^{-T} B, U upper m x m (Left/Upper/Trans/NonUnit) */
static void k_trsm_lut(int m, int n, const double *U, int ldu, double *B, int ldb)
{
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double s = AT(B, ldb, i, j);
            for (int k = 0; k < i; ++k) s -= AT(U, ldu, k, i) * AT(B, ldb, k, j);
            AT(B, ldb, i, j) = s / AT(U, ldu, i, i);
        }
}

/* B <- op(T)^{-1} B, T triangular (lower when lower != 0) m x m, op = T when t. */
static void k_trsm_left(int lower, int t, int m, int n, const double *T, int ldt, double *B, int ldb)
{
    /* effective triangle of op(T): lower-forward when (lower && !t) || (!lower && t) */
    const int fwd = (lower && !t) || (!lower && t);
    for (int j = 0; j < n; ++j) {
        if (fwd) {
            for (int i = 0; i < m; ++i) {
                double s = AT(B, ldb, i, j);
                for (int k = 0; k < i; ++k) s -= opel(T, ldt, t, i, k) * AT(B, ldb, k, j);
                AT(B, ldb, i, j) = s / AT(T, ldt, i, i);
            }
        } else {
            for (int i = m - 1; i >= 0; --i) {
                double s = AT(B, ldb, i, j);
                for (int k = i + 1; k < m; ++k) s -= opel(T, ldt, t, i, k) * AT(B, ldb, k, j);
                AT(B, ldb, i, j) = s / AT(T, ldt, i, i);
            }
        }
    }
}

/*
 * compute/pzpotrf.c:84-194 -- right-looking tile Cholesky, same loop order,
 * on a column-major array viewed with NB x NB tiles.  Returns LAPACK info
 * (global 1-based index of the failing minor, compute/pzpotrf.c:94).
 */
int orc_dpotrf_tiled(int uplo, int N, int NB, double *A, int lda)
{
    const int NT = (N + NB - 1) / NB;
#define TD(m) (((m) == NT - 1) ? N - (m) * NB : NB)
#define TP(m, n) (A + (int64_t)(m) * NB + (int64_t)(n) * NB * lda)
    for (int k = 0; k < NT; ++k) {
        const int tk = TD(k);
        int info = k_potrf(uplo, tk, TP(k, k), lda);
        if (info) return k * NB + info;
        if (uplo == ORC_LOWER) {
            for (int m = k + 1; m < NT; ++m) k_trsm_rlt(TD(m), tk, TP(k, k), lda, TP(m, k), lda);
            for (int n = k + 1; n < NT; ++n) {
                k_syrk_sub(ORC_LOWER, 0, TD(n), tk, TP(n, k), lda, TP(n, n), lda);
                for (int m = n + 1; m < NT; ++m)
                    k_gemm_sub(0, 1, TD(m), TD(n), tk, TP(m, k), lda, TP(n, k), lda, TP(m, n), lda);
            }
        } else {
            for (int n = k + 1; n < NT; ++n) k_trsm_lut(tk, TD(n), TP(k, k), lda, TP(k, n), lda);
            for (int m = k + 1; m < NT; ++m) {
                k_syrk_sub(ORC_UPPER, 1, TD(m), tk, TP(k, m), lda, TP(m, m), lda);
                for (int n = m + 1; n < NT; ++n)
                    k_gemm_sub(1, 0, TD(m), TD(n), tk, TP(k, m), lda, TP(k, n), lda, TP(m, n), lda);
            }
        }
    }
    return 0;
}

/*
 * compute/zpotrs.c:302-304 -> compute/pztrsm.c:58-200: two blocked left
 * triangular solves with the factor (Upper: U^T then U; Lower: L then L^T).
 */
void orc_dpotrs_tiled(int uplo, int N, int nrhs, int NB, const double *A, int lda, double *B, int ldb)
{
    const int NT = (N + NB - 1) / NB;
#define BP(m) (B + (int64_t)(m) * NB)
    const int lower = (uplo == ORC_LOWER);
    /* forward: op(T) lower-effective (L or U^T) */
    for (int k = 0; k < NT; ++k) {
        k_trsm_left(lower, !lower, TD(k), nrhs, TP(k, k), lda, BP(k), ldb);
        for (int m = k + 1; m < NT; ++m) {
            if (lower) k_gemm_sub(0, 0, TD(m), nrhs, TD(k), TP(m, k), lda, BP(k), ldb, BP(m), ldb);
            else k_gemm_sub(1, 0, TD(m), nrhs, TD(k), TP(k, m), lda, BP(k), ldb, BP(m), ldb);
        }
    }
    /* backward: op(T) upper-effective (L^T or U) */
    for (int k = NT - 1; k >= 0; --k) {
        k_trsm_left(lower, lower, TD(k), nrhs, TP(k, k), lda, BP(k), ldb);
        for (int m = k - 1; m >= 0; --m) {
            if (lower) k_gemm_sub(1, 0, TD(m), nrhs, TD(k), TP(k, m), lda, BP(k), ldb, BP(m), ldb);
            else k_gemm_sub(0, 0, TD(m), nrhs, TD(k), TP(m, k), lda, BP(k), ldb, BP(m), ldb);
        }
    }
#undef BP
#undef TP
#undef TD
}

/* ---- checks (testing/testing_zcheck_facto.c) ------------------------------ */

/* LAPACK dlamch('e') as used by the testing driver (control/lamch.c:48-56). */
double orc_eps(void) { return 1.1102230246251565e-16; }

static double one_norm(int M, int N, const double *A, int lda)
{
    double r = 0.0;
    for (int j = 0; j < N; ++j) {
        double s = 0.0;
        for (int i = 0; i < M; ++i) s += fabs(AT(A, lda, i, j));
        if (s > r) r = s;
    }
    return r;
}

/*
 * check_zxxtrf (testing_zcheck_facto.c:198-300), symmetric case:
 * ||A0 - op(F)op(F)^T||_1 / (||A0||_1 N eps), F the uplo triangle of the
 * factor.  A0 is the full symmetric matrix.
 */
double orc_check_factorization(int uplo, int N, const double *A0, int lda, const double *F, int ldf)
{
    double *R = (double *)malloc(sizeof(double) * (size_t)N * N);
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
            double s = 0.0;
            const int kmax = i < j ? i : j;
            for (int k = 0; k <= kmax; ++k) {
                if (uplo == ORC_LOWER) s += AT(F, ldf, i, k) * AT(F, ldf, j, k);
                else s += AT(F, ldf, k, i) * AT(F, ldf, k, j);
            }
            R[i + (int64_t)j * N] = AT(A0, lda, i, j) - s;
        }
    const double anorm = one_norm(N, N, A0, lda);
    const double rnorm = one_norm(N, N, R, N);
    free(R);
    return rnorm / (anorm * N * orc_eps());
}

/*
 * check_zsolve (testing_zcheck_facto.c:392-460), symmetric case:
 * ||B - A0 X||_1 / (||A0||_1 ||X||_1 N eps).
 */
double orc_check_solve(int N, int nrhs, const double *A0, int lda, const double *X, int ldx,
                       const double *B, int ldb)
{
    double *R = (double *)malloc(sizeof(double) * (size_t)N * nrhs);
    for (int j = 0; j < nrhs; ++j)
        for (int i = 0; i < N; ++i) {
            double s = AT(B, ldb, i, j);
            for (int k = 0; k < N; ++k) s -= AT(A0, lda, i, k) * AT(X, ldx, k, j);
            R[i + (int64_t)j * N] = s;
        }
    const double anorm = one_norm(N, N, A0, lda);
    const double xnorm = one_norm(N, nrhs, X, ldx);
    const double rnorm = one_norm(N, nrhs, R, N);
    free(R);
    return rnorm / (anorm * xnorm * N * orc_eps());
}
