// executor.cuh -- device-resident tile-DAG executor (shared declarations).
//
// The reference runs chameleon_pdpotrf / chameleon_pdtrsm (compute/pzpotrf.c:
// 84-194, compute/pztrsm.c:58-200) by submitting one runtime task per tile
// kernel to StarPU/OpenMP (runtime/*/codelets/codelet_z{potrf,trsm,syrk,gemm}.c).
// Here the same DAG is recorded once on the host as a list of sub-tile tasks in
// a topological order and run by ONE persistent kernel: each CTA takes the
// next task index with an atomic, waits (bounded) on per-tile dependency
// counters, runs the tile operation and releases its counter.  A task only
// waits on tasks that precede it in the list, and a CTA only takes a task while
// it is resident, so the launch cannot deadlock whatever the grid size.
#pragma once
#include <stdint.h>

namespace chb {

enum TaskKind : int16_t {
    TK_POTRF = 1,     // factor diagonal tile k, invert its inner diagonal blocks
    TK_TRSM = 2,      // panel row block: A(m,k) <- A(m,k) L(k,k)^{-T}
    TK_UPD = 3,       // trailing sub-block: A(m,n) -= sum_{k in group} A(m,k) A(n,k)^T (SYRK when m == n)
    TK_FWD_TRSM = 4,  // B(k) <- L(k,k)^{-1} B(k)
    TK_FWD_UPD = 5,   // B(m) -= L(m,k) B(k)            (m > k)
    TK_BWD_TRSM = 6,  // B(k) <- L(k,k)^{-T} B(k)
    TK_BWD_UPD = 7,   // B(m) -= L(k,m)^T B(k)          (m < k)
    TK_INV = 8,       // invert inner diagonal blocks of an existing factor (potrs alone)
    TK_XINV = 9,      // full inverse of diagonal tile k (FP32 substitution steps)
    TK_CAST = 10,     // (MODE_CAST) FP64 -> FP32 copy of tile (m,n) once its columns have
                      // arrived from the host, with its share of ||A||_inf
};

// TK_UPD applies the panels k .. k + bn - 1 of one k group (one accumulator,
// one write of the sub-block); `grp` is the group's position among the update
// groups of tile column n (upd_group_of), i.e. how many groups precede it.
struct Task {
    int16_t kind, sub;   // sub: row block (TRSM / *_UPD on B) or (bi | bj << 8) (TK_UPD)
    int16_t m, n, k, bn; // bn: right-hand-side tile column, or (TK_UPD) the group's panel count
    int32_t grp;         // TK_UPD: index of the group in tile column n
};

// Update groups of tile column n: the panels k < n that update tile (m, n),
// m >= n, are applied in groups.  The last `tail` panels (default UPD_TAIL:
// n-2, n-1) are groups of their own: they are on the critical path of steps
// n-1 and n.  The panels before them form groups of G aligned at the end (the
// first group takes the remainder), so that every step completes a group for
// 1/G of the columns and the update work arrives evenly instead of in bursts.
constexpr int UPD_TAIL = 2;
__host__ __device__ __forceinline__ int upd_ngroups(int n, int G, int tail) {
    if (n <= tail) return n > 0 ? n : 0;
    return (n - tail + G - 1) / G + tail;
}
// The group of column n (n > k) that panel k belongs to: first panel, panel
// count and index.
__host__ __device__ __forceinline__ void upd_group_of(int n, int k, int G, int tail, int *k0, int *cnt, int *idx) {
    const int m = n > tail ? n - tail : 0;   // panels in groups of G
    if (k >= m) {
        *k0 = k;
        *cnt = 1;
        *idx = (m + G - 1) / G + (k - m);
        return;
    }
    const int r = m % G;   // size of the first (partial) group, 0 if none
    if (r > 0 && k < r) {
        *k0 = 0;
        *cnt = r;
        *idx = 0;
    } else {
        const int g = (k - r) / G;
        *k0 = r + g * G;
        *cnt = G;
        *idx = g + (r > 0 ? 1 : 0);
    }
}
static_assert(sizeof(Task) == 16, "Task is 16 bytes");

// MODE_XINV: the substitution steps apply full inverses of the diagonal tiles
// (one GEMM per tile), computed by TK_XINV tasks; with MODE_NOINV (solve only)
// the inverses are already in place from an earlier launch on the same factor.
// MODE_CAST: the FP32 tiles of A are produced inside the launch by TK_CAST
// tasks from an FP64 column-major copy of A that is still arriving from the
// host: each tile's first consumer waits for its cast.
enum ExecMode : int { MODE_FACT = 1, MODE_SOLVE = 2, MODE_XINV = 4, MODE_NOINV = 8, MODE_CAST = 16 };

constexpr int SUBB = 128;      // sub-block edge of trailing updates / row blocks
// Row block of the substitution tasks (FWD/BWD TRSM and UPD) with full
// diagonal-tile inverses (MODE_XINV): the forward and backward solves are a
// chain of 2 NT dependent steps, and 64-row tasks halve each step's latency.
constexpr int SOLB = 64;
// Row block of the substitution tasks of a launch mode.
__host__ __device__ constexpr int solve_rows(int mode) { return (mode & 4 /*MODE_XINV*/) ? SOLB : SUBB; }

struct ExecState {
    int next;          // dispatch cursor (alone in its 128-byte line: the contended atomic)
    int pad0[31];
    int abort;         // set on failure: remaining tasks are skipped
    int info;          // min global 1-based index of a non-positive pivot (INT_MAX: none)
    int error;         // 0 or a CHAMELEON_ERR_* code (device timeout)
    int done;          // tasks completed (each CTA adds its count when it exits)
    int stuck_task;    // task index whose wait ran out (-1)
    int pad[2];
};

struct TraceRec {
    int32_t task, smid;
    uint64_t t0, t1;   // globaltimer after the dependency wait, at the end of the task
    uint32_t wait_ns;  // time from taking the task to its dependencies being met
    uint32_t ph[3];    // clock cycles: POTRF in (block-column update, leaf, panel); tcgen05
                       // update from its start to (C staged, accumulator ready, end)
};

struct ExecParams {
    const Task *tasks;
    int ntasks;
    // npotrf > 0: CTA 0 runs exactly the POTRF tasks potrf_idx[0..npotrf) in
    // order and the other CTAs skip them (both are sub-orders of one
    // topological order, so the launch still always progresses)
    int npotrf;
    const int *potrf_idx;
    int mode;
    int upper;
    int NT, N, NB;          // A: NT x NT tiles, order N, tile size NB (square tiles)
    void *A;                // double or float tiles
    const int64_t *a_off;   // element offset of tile (m,n) at a_off[m + NT*n]
    const int *a_ld;        // leading dimension of tile row m
    int NTB, nrhs, NBB;     // B: NT x NTB tiles of NB x NBB
    void *B;
    const int64_t *b_off;   // b_off[m + NT*bn]
    const int *b_ld;
    int *updA, *panA, *fwdB, *fwdDone, *bwdB, *bwdDone;
    void *invd;             // full_inv: NT inverted NB x NB diagonal tiles (ld NB);
                            // else NT * NIB inverted IB x IB blocks (element type of A)
    int NIB;
    int full_inv;           // FP32 path: recursive tile factorization with full tile inverses
    void *xinv;             // MODE_XINV: NT full inverses of the diagonal tiles (ld NB)
    void *Y;                // MODE_XINV: forward results (layout of B): the substitutions
                            // read B and write Y (forward), read Y and write B (backward)
    int *xinvDone;          // MODE_XINV: TK_XINV(k) done
    ExecState *st;
    TraceRec *trace;        // optional per-task trace (nullptr: off)
    // tcgen05 trailing update of the FP32 factorization (split-BF16 operands):
    // split chunks of panel tile (m,k), m > k, at split + (m(m-1)/2 + k) * tile_split_bytes
    uint8_t *split;
    int split_nrb, split_nkc;   // 128-row blocks and 64-wide k chunks per panel tile
    int kgroup;                 // update group size G (upd_ngroups / upd_group_of)
    int utail;                  // single-panel update groups at the end of each column
    // MODE_CAST: the FP64 source (column-major, ld csrc_ld) of the stored
    // triangle; tile column q of it has arrived once carrive[q] >= cepoch
    // (written by the copy engine after the column's data); castDone counts
    // the casts per tile; colsum receives the absolute row sums of the
    // symmetric matrix (its infinity norm), covf is set on a value beyond FP32
    const double *csrc;
    int64_t csrc_ld;
    const int *carrive;
    int cepoch;
    int *castDone;
    double *colsum;
    int *covf;
    unsigned long long wait_budget_ns;
};

}  // namespace chb
